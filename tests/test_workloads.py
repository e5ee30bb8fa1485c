"""The synthetic workloads: generated vessels, inflow waveform, sweep and request stream (host side)."""
import numpy as np
import pytest

from cerebrosim_b200 import vessel, workloads as W
from oracle import sdf_ref


def test_vessel_geometry():
    g = W.stenosed_vessel(3)
    t, b = g["branches"]["trunk"], g["branches"]["branch"]
    # parent spans the 20 mm along x within the jitter, radius 1.5 mm; 70 % area reduction at the throat
    assert abs(t["C"][0, 0]) < 1e-9 and abs(t["C"][-1, 0] - 20.0) < 1e-9
    assert np.abs(t["C"][:, 1:]).max() <= 2.0 + 0.5
    assert np.isclose((t["R"].min() / 1.5) ** 2, 0.3, atol=2e-3)
    assert np.allclose(t["R0"], 1.5) and np.allclose(b["R"], 1.0)
    # the branch leaves the parent's centreline at 40 degrees to its tangent
    k = int(np.argmin(np.linalg.norm(t["C"] - b["C"][0], axis=1)))
    tk = t["C"][k + 1] - t["C"][k - 1]
    d = b["C"][-1] - b["C"][0]
    ang = np.degrees(np.arccos(tk @ d / np.linalg.norm(tk) / np.linalg.norm(d)))
    assert abs(ang - 40.0) < 1.0
    assert b["caps"]["start"] is None and b["caps"]["end"] is not None
    # caps point outwards along the centreline
    assert t["caps"]["start"][1] @ (t["C"][1] - t["C"][0]) < 0 and t["caps"]["end"][1] @ (t["C"][-1] - t["C"][-2]) > 0


def test_openings_and_occlusion():
    assert [(o["kind"], o["branch"]) for o in W.openings(W.stenosed_vessel(3))] == [
        ("inlet", "trunk"), ("outlet", "trunk"), ("outlet", "branch")]
    go = W.stenosed_vessel(3, stenosis=1.0)
    assert [(o["kind"], o["branch"]) for o in W.openings(go)] == [
        ("inlet", "branch"), ("outlet", "trunk"), ("outlet", "trunk_distal")]
    # the clot: the field is positive (solid) across the whole gap between the faces, negative on either side
    pk = vessel.packed(go)
    prox, dist = go["branches"]["trunk"]["C"], go["branches"]["trunk_distal"]["C"]
    a, b = prox[-1], dist[0]
    assert np.isclose(np.linalg.norm(b - a), 3.0, atol=0.15)
    gap = a[None, :] + np.linspace(0.02, 0.98, 25)[:, None] * (b - a)[None, :]
    assert (sdf_ref.sdf_points(gap, *pk.arrays()) > 0).all()
    assert (sdf_ref.sdf_points(np.vstack([prox[-5], dist[5]]), *pk.arrays()) < 0).all()


def test_fourier_drive():
    for seed in (3, 100, 1000):
        c = W.fourier_drive(seed)
        assert len(c) == 9
        phi = np.linspace(0, 2 * np.pi, 8192, endpoint=False)
        w = c[0] + sum(c[1 + 2 * k] * np.cos((k + 1) * phi) + c[2 + 2 * k] * np.sin((k + 1) * phi) for k in range(4))
        assert np.isclose(w.mean(), 0.03, rtol=1e-9)
        assert np.isclose(w.max() / w.mean(), 1.8, rtol=2e-3)
        assert w.min() / w.mean() >= 0.2 - 1e-6


def test_sizes_and_inflow():
    g = W.stenosed_vessel(3)
    n = W.estimated_nodes(g, 0.05)
    assert 1.3e6 < n < 1.8e6
    dx = W.dx_for_nodes(0.5e6, n, 0.05)
    assert np.isclose(W.estimated_nodes(g, dx), 0.5e6)
    assert np.isclose(W.inflow_scale(95.0, 0.0), 0.03)
    assert np.isclose(W.inflow_scale(145.0, 0.95), 0.1 * 0.05 / 1.8)
    assert np.isclose(W.inflow_scale(145.0, 1.0), 0.03 * 145 / 95)


def test_request_stream_and_sweep_specs():
    rs = W.request_stream(20, seed=5)
    assert [r["id"] for r in rs] == list(range(20))
    assert all(np.diff([r["arrival"] for r in rs]) > 0)
    assert all(1 <= r["beats"] <= 4 and 0 <= r["stenosis"] <= 1 and 70 <= r["pressure"] <= 145 for r in rs)
    assert all(0.2e6 <= r["nodes"] <= 4e6 for r in rs)
    assert rs == W.request_stream(20, seed=5)
    sw = W.sweep()
    assert len(sw) == 16
    assert sorted(s["stenosis"] for s in sw[:12]) == [0.0, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9, 0.95, 1.0]
    assert np.isclose(min(s["nodes"] for s in sw), 0.3e6) and np.isclose(max(s["nodes"] for s in sw), 3e6)
    assert [s["pressure"] for s in sw] == [70.0 + 5 * k for k in range(16)]


def test_node_orders_are_permutations():
    from cerebrosim_b200 import lbm
    rng = np.random.default_rng(1)
    coords = np.unique(rng.integers(0, 40, size=(3000, 3)), axis=0)
    coords = coords[np.lexsort((coords[:, 2], coords[:, 1], coords[:, 0]))]        # C order
    lat = {"coords": coords, "nbr": np.zeros((27, len(coords)), np.int32)}
    assert lbm.node_order(lat, "c") is None
    for order in ("axis", "morton"):
        perm = lbm.node_order(lat, order)
        assert perm is None or np.array_equal(np.sort(perm), np.arange(len(coords)))
    # a lattice longest along z is already in "axis" order
    long_z = coords.copy()
    long_z[:, 2] *= 10
    assert lbm.node_order({"coords": long_z, "nbr": lat["nbr"]}, "axis") is None
    # along x: the x coordinate varies fastest
    long_x = coords[:, [2, 1, 0]] * np.array([10, 1, 1])
    long_x = long_x[np.lexsort((long_x[:, 2], long_x[:, 1], long_x[:, 0]))]
    perm = lbm.node_order({"coords": long_x, "nbr": lat["nbr"]}, "axis")
    c = long_x[perm]
    assert np.all(np.diff(c[:, 0])[(np.diff(c[:, 2]) == 0) & (np.diff(c[:, 1]) == 0)] > 0)


def test_split_order_puts_boundary_nodes_last():
    from cerebrosim_b200 import cases, lbm
    from oracle import lattice_ref as L
    lat = L.build_lattice(**cases.lattice_args(cases.case("open_pipe_straight_D20")))
    bnd = (lat["nbr"] < 0).any(0)
    perm = lbm.node_order(lat, "split")
    assert np.array_equal(np.sort(perm), np.arange(len(perm)))
    k = int((~bnd).sum())
    assert not bnd[perm[:k]].any() and bnd[perm[k:]].all()
    assert np.all(np.diff(perm[:k]) > 0) and np.all(np.diff(perm[k:]) > 0)      # C order within each part


def test_boundary_first_order_puts_boundary_nodes_first():
    from cerebrosim_b200 import cases, lbm
    from oracle import lattice_ref as L
    lat = L.build_lattice(**cases.lattice_args(cases.case("open_pipe_straight_D20")))
    bnd = (lat["nbr"] < 0).any(0)
    k = int(bnd.sum())
    perm = lbm.node_order(lat, "boundary-first")
    assert np.array_equal(np.sort(perm), np.arange(len(perm)))
    assert bnd[perm[:k]].all() and not bnd[perm[k:]].any()
    assert np.all(np.diff(perm[:k]) > 0) and np.all(np.diff(perm[k:]) > 0)      # C order within each part
    axis = lbm.node_order(lat, "axis")
    axis = np.arange(len(bnd)) if axis is None else axis              # None: the axis order is the C order
    perm = lbm.node_order(lat, "axis-boundary-first")
    assert np.array_equal(perm, np.concatenate([axis[bnd[axis]], axis[~bnd[axis]]]))


def test_lattice_host_tables_are_copied_on_first_read():
    """lbm.Lattice (build_lattice(..., host=False)): a host table missing from the dict is copied from its device copy
    the first time it is read and then kept; other missing keys raise KeyError; n_nodes reads no host table."""
    import torch
    from cerebrosim_b200 import lbm
    nbr = torch.arange(27 * 5, dtype=torch.int32).reshape(27, 5)
    dev = {"nbr": nbr, "q": nbr.float(), "uin": torch.zeros(5, 3), "coords": torch.zeros(5, 3)}
    lat = lbm.Lattice(dx=1.0, _dev=dev)
    assert lbm.n_nodes(lat) == 5 and "nbr" not in dict.keys(lat)
    got = lat["nbr"]
    assert isinstance(got, np.ndarray) and np.array_equal(got, nbr.numpy()) and "nbr" in dict.keys(lat)
    assert lat["nbr"] is got
    assert "q" not in dict.keys(lat)
    with pytest.raises(KeyError):
        lat["nothing"]
    assert lbm.n_nodes({"nbr": np.zeros((27, 7), np.int32)}) == 7


def test_device_node_orders_equal_host_orders_on_cpu_tensors():
    """The solver's device computation of the axis and split orders (lbm._device_order: an argsort of one integer key
    per node, stable partitions by the boundary mask) gives node_order's permutations; run here on CPU tensors, on a
    pipe along x (its longest axis is not the C order's fastest) with an inlet and an outlet."""
    import torch
    from cerebrosim_b200 import lbm
    from oracle import lattice_ref as L
    x, y, z = np.meshgrid(np.arange(60), np.arange(14), np.arange(16), indexing="ij")
    phi = (np.sqrt((y - 6.5) ** 2 + (z - 7.2) ** 2) - 5.0).astype(np.float32)
    ops = [{"kind": "inlet", "centre": [0.5, 6.5, 7.2], "normal": [1, 0, 0], "radius": 6.0},
           {"kind": "outlet", "centre": [58.5, 6.5, 7.2], "normal": [-1, 0, 0], "radius": 6.0}]
    lat = L.build_lattice(phi, [0, 0, 0], 1.0, openings=ops)
    nbr = torch.as_tensor(lat["nbr"])
    for order in lbm._DEVICE_ORDERS:
        host = lbm.node_order(lat, order)
        dev = lbm._device_order(lat, nbr, order, torch.device("cpu"))
        assert host is not None and dev is not None and np.array_equal(dev.numpy(), host), order
