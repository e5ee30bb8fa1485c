"""The table oracle (oracle/lattice_ref.py) and the host-side geometry against the reference's own outputs.

tests/golden/ was written by running the reference's lbm.build_lattice / Solver.set_sponge / Units (see
tests/golden/make_golden.py); the link counts of the full-size lattices also equal the ones the reference
published in geometry/solver.json:73-120 (75600 nodes, links 137890 / 2818 / [2818] for the straight open pipe...).
"""
import hashlib
import json

import numpy as np
import pytest

from cerebrosim_b200 import cases
from oracle import lattice_ref as L


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


PUBLISHED_COUNTS = {  # geometry/solver.json:73-120 of the reference
    "open_pipe_straight_D20": (75600, {"wall": 137890, "inlet": 2818, "outlet": [2818]}),
    "open_pipe_tilted_D20": (75280, {"wall": 136979, "inlet": 2832, "outlet": [2779]}),
    "stenosis70_D20": (144678, None),
}


def test_small_fixtures_bit_exact(golden):
    for name in golden.small_names():
        meta, arr = golden.small_case(name)
        lat = L.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=meta["openings"],
                              periodic=meta["periodic"], opening_slack=meta["slack"])
        for k in ("nbr", "q", "uin", "coords"):
            assert lat[k].dtype == arr[k].dtype and np.array_equal(lat[k], arr[k]), (name, k)
        assert lat["counts"] == meta["counts"], name
        assert lat["n_outlets"] == len([o for o in meta["openings"] if o["kind"] == "outlet"])


@pytest.mark.parametrize("name", ["periodic_pipe_D10", "periodic_pipe_D20", "periodic_pipe_D40",
                                  "poiseuille_R10_L64", "open_pipe_straight_D20", "open_pipe_tilted_D20",
                                  "stenosis70_D20", "open_pipe_R24_L192"])
def test_full_size_tables_by_hash(golden, name):
    h = golden.hashes[name]
    c = cases.case(name)
    assert sha(c["phi"]) == h["phi"], "geometry differs from the reference's validate.py"
    lat = L.build_lattice(**cases.lattice_args(c))
    assert lat["nbr"].shape[1] == h["N"]
    assert lat["counts"] == h["counts"]
    for k in ("nbr", "q", "uin", "coords"):
        assert sha(lat[k]) == h[k], k
    if name in PUBLISHED_COUNTS:
        n, cnt = PUBLISHED_COUNTS[name]
        assert lat["nbr"].shape[1] == n
        if cnt:
            assert lat["counts"] == cnt


def test_sponge_matches_reference(golden):
    meta, arr = golden.small_case("open_pipe_tilted_R4")
    lat = L.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=meta["openings"])
    from cerebrosim_b200 import lbm as product
    for tag in ("a", "b", "c"):
        args = json.loads(str(golden.sponge[f"{tag}/args"]))
        ref_tau = golden.sponge[f"{tag}/tau_cell"]
        tau = L.sponge_tau(lat, args["tau"], args["length"], args["tau_max"], tuple(args["kinds"]))
        assert np.array_equal(tau, ref_tau)
        tau_p = product.sponge_tau(lat, args["tau"], args["length"], args["tau_max"], tuple(args["kinds"]))
        assert np.array_equal(tau_p, ref_tau)
        assert np.array_equal((1.0 / tau_p).astype(np.float32), golden.sponge[f"{tag}/om"])


def test_units_and_constants(golden):
    from cerebrosim_b200 import lbm as product
    for key, u in golden.units.items():
        if key == "constants":
            for mod in (L, product):
                assert np.array_equal(mod.C, np.array(u["C"])) and np.array_equal(mod.OPP, np.array(u["OPP"]))
                assert np.array_equal(mod.W, np.array(u["W"]))
                assert (mod.WALL, mod.INLET, mod.OUTLET0) == (u["WALL"], u["INLET"], u["OUTLET0"])
            continue
        for mod in (L, product):
            x = mod.Units(u["dx"], u["dt"], 1060.0, 3.5e-3 / 1060.0)
            assert x.nu_lu == u["nu_lu"] and x.tau == u["tau"] and x.c == u["c"]
            assert float(x.u(0.02)) == u["u_of_0.02"] and float(x.p(1e-4)) == u["p_of_1e-4"]
            assert float(x.u_lu(0.6)) == u["u_lu_of_0.6"] and float(x.p_lu(1000.0)) == u["p_lu_of_1000"]


def test_scatter_roundtrip(golden):
    from cerebrosim_b200 import lbm as product
    meta, arr = golden.small_case("stenosis70_D8")
    lat = {"shape": arr["phi"].shape, "coords": arr["coords"]}
    vals = np.arange(len(arr["coords"]), dtype=np.float32)
    g = product.scatter(lat, vals)
    assert np.array_equal(g[tuple(arr["coords"].T)], vals)
    assert np.isnan(g).sum() == g.size - len(vals)
    gi = product.scatter(lat, np.arange(len(vals)), fill=-1)
    assert gi.dtype == float and gi[tuple(arr["coords"][3])] == 3
