"""GPU table builder (csrc/lattice_build.cu through lbm.build_lattice) against the reference's own tables:
bit-exact on every small fixture and, by SHA-256, on the full-size validation and benchmark lattices."""
import hashlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from cerebrosim_b200 import _lib, cases, lbm  # noqa: E402


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_small_fixtures_bit_exact(golden):
    for name in golden.small_names():
        meta, arr = golden.small_case(name)
        lat = lbm.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=meta["openings"],
                                periodic=meta["periodic"], opening_slack=meta["slack"])
        for k in ("nbr", "q", "uin", "coords"):
            assert lat[k].dtype == arr[k].dtype and lat[k].shape == arr[k].shape, (name, k)
            assert np.array_equal(lat[k].view(np.uint32) if k in ("q", "uin") else lat[k],
                                  arr[k].view(np.uint32) if k in ("q", "uin") else arr[k]), (name, k)
        assert lat["counts"] == meta["counts"], name
        assert lat["shape"] == arr["phi"].shape


@pytest.mark.parametrize("name", ["periodic_pipe_D10", "periodic_pipe_D20", "periodic_pipe_D40",
                                  "poiseuille_R10_L64", "open_pipe_straight_D20", "open_pipe_tilted_D20",
                                  "stenosis70_D20", "open_pipe_R24_L192"])
def test_full_size_tables_by_hash(golden, name):
    h = golden.hashes[name]
    lat = lbm.build_lattice(**cases.lattice_args(cases.case(name)))
    assert lat["nbr"].shape[1] == h["N"] and lat["counts"] == h["counts"]
    for k in ("nbr", "q", "uin", "coords"):
        assert sha(lat[k]) == h[k], k


def test_link_encoding_roundtrip(golden):
    """The step's packed link table expands back to exactly the reference's (nbr, q)."""
    import ctypes
    for name in ("box_openings_slack1", "noise_nan_inf", "stenosis70_D8"):
        meta, arr = golden.small_case(name)
        lat = lbm.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=meta["openings"],
                                periodic=meta["periodic"], opening_slack=meta["slack"])
        s = lbm.Solver(lat, 0.05, model="regularised")
        links = s.link_table()                       # expanded from the compressed connectivity
        nbr = torch.empty_like(links)
        q = torch.empty(links.shape, dtype=torch.float32, device=s.dev)
        _lib.check(_lib.load().cs_links_decode(ctypes.c_void_p(links.data_ptr()),
                                               ctypes.c_void_p(s.ginfo.data_ptr()), ctypes.c_void_p(s.gq.data_ptr()),
                                               s.N, s.gmax, ctypes.c_void_p(nbr.data_ptr()),
                                               ctypes.c_void_p(q.data_ptr()), ctypes.c_void_p(s.stream.cuda_stream)))
        s.synchronize()
        assert s.ghosts == [int((arr["nbr"][i] < 0).sum()) for i in range(27)]
        assert s.npad == s.N + max(s.ghosts)
        assert np.array_equal(nbr.cpu().numpy(), arr["nbr"])
        qd = q.cpu().numpy()
        wall = arr["nbr"] == lbm.WALL
        assert np.array_equal(qd[wall].view(np.uint32), arr["q"][wall].view(np.uint32))
        assert np.all(qd[~wall] == 0.5)


@pytest.mark.parametrize("name", ["open_pipe_R24_L192", "open_pipe_tilted_D20", "stenosis70_D20"])
def test_compressed_connectivity(name):
    """Regular nodes share segment delta vectors; the compressed form expands back to the full pull table."""
    lat = lbm.build_lattice(**cases.lattice_args(cases.case(name)))
    s = lbm.Solver(lat, 0.05, model="regularised")
    links = s.link_table().cpu().numpy()
    nbr = lat["nbr"]
    fluid = nbr >= 0
    assert np.array_equal(links[fluid], nbr[fluid])
    assert np.all(links[~fluid] >= s.N)
    irregular = (~fluid).any(0)
    assert s.n_irr == int(irregular.sum())
    assert s.n_seg < 0.05 * s.N                       # a few segments per row, not per node
    print(name, s.N, "irregular", s.n_irr, "segments", s.n_seg)


def test_invalid_tables_are_rejected(golden):
    meta, arr = golden.small_case("stenosis70_D8")
    lat = lbm.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=meta["openings"])
    bad = dict(lat)
    bad.pop("_dev")
    nbr = lat["nbr"].copy()
    nbr[3, 17] = lat["nbr"].shape[1] + 5           # pull source beyond N
    bad["nbr"] = nbr
    with pytest.raises(_lib.CerebroSimError, match="invalid entries"):
        lbm.Solver(bad, 0.05)
    nbr = lat["nbr"].copy()
    nbr[5, 3] = lbm.OUTLET0 - 4                     # outlet 4 of a lattice with one outlet
    bad["nbr"] = nbr
    with pytest.raises(_lib.CerebroSimError):
        lbm.Solver(bad, 0.05)
    q = lat["q"].copy()
    w = np.argwhere(lat["nbr"] == lbm.WALL)[0]
    q[w[0], w[1]] = np.nan                          # a wall link without a finite q
    bad["nbr"], bad["q"] = lat["nbr"], q
    with pytest.raises(_lib.CerebroSimError):
        lbm.Solver(bad, 0.05)


def test_builder_limits():
    phi = np.full((4, 4, 4), -1.0, np.float32)
    ops = [{"kind": "outlet", "centre": [0, 0, 0], "normal": [1, 0, 0], "radius": 1.0}] * 33
    with pytest.raises(_lib.CerebroSimError, match="openings"):
        lbm.build_lattice(phi, [0, 0, 0], 1.0, openings=ops)
    with pytest.raises(ValueError):
        lbm.build_lattice(phi, [0, 0, 0], 1.0, periodic=(3,))
    with pytest.raises(ValueError):
        lbm.build_lattice(phi[0], [0, 0, 0], 1.0)


def test_sponge_on_the_device_equals_the_reference(golden):
    """Solver.set_sponge evaluates the sponge on the device (k_sponge): per-cell tau and the float32 1 / tau equal
    the reference's own set_sponge output (tests/golden/sponge.npz) bit for bit, for inlet and outlet sponges of
    several lengths; C order and a renumbered order give the same cells."""
    import json
    meta, arr = golden.small_case("open_pipe_tilted_R4")
    lat = lbm.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=meta["openings"])
    for order in ("c", "boundary-first"):
        for tag in ("a", "b", "c"):
            args = json.loads(str(golden.sponge[f"{tag}/args"]))
            s = lbm.Solver(lat, 0.02, model="regularised", order=order)
            s.tau = args["tau"]                       # the reference's tau itself, not 3 nu + 0.5 recomputed
            s.set_sponge(args["length"], args["tau_max"], tuple(args["kinds"]))
            assert np.array_equal(s.tau_cell, golden.sponge[f"{tag}/tau_cell"]), tag
            om = s.om.abs()
            if s.inv is not None:
                om = om[s.inv]
            assert np.array_equal(om.cpu().numpy(), golden.sponge[f"{tag}/om"]), tag
