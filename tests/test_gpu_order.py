"""Internal node orders and the autotuner: a solver on a renumbered lattice gives the same fields, in the lattice's
order, as on the lattice's own C order (each node's update reads the same values whatever its number)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from cerebrosim_b200 import autotune, lbm  # noqa: E402
from cerebrosim_b200.simulate import ArterySolver  # noqa: E402


def lattice(golden, name):
    meta, arr = golden.small_case(name)
    return lbm.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=meta["openings"],
                             periodic=meta["periodic"], opening_slack=meta["slack"])


def configure(s):
    s.set_sponge(4, 0.6)
    s.set_outlet_pressure([0.0] * max(1, s.lat["n_outlets"]))
    s.set_drive([0.03, 0.01, 0.0], period=200, ramp=50)


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_orders_give_identical_fields(golden, storage):
    lat = lattice(golden, "stenosis70_D8")
    ref = lbm.Solver(lat, 0.02, model="regularised", storage=storage)
    configure(ref)
    ref.run(301)
    p0, u0 = ref.fields()
    for order in ("axis", "morton", "split", "axis-split", "boundary-first", "axis-boundary-first"):
        s = lbm.Solver(lat, 0.02, model="regularised", storage=storage, order=order)
        assert order == "axis" or s.perm is not None
        configure(s)
        s.run(301)
        p, u = s.fields()
        assert s.ok()
        assert np.array_equal(p, p0) and np.array_equal(u, u0), order


def test_artery_coupling_in_another_order(golden):
    meta, arr = golden.small_case("open_pipe_straight_R4")
    lat0 = lattice(golden, "open_pipe_straight_R4")
    ops = [dict(o, kind="outlet") for o in lat0["openings"]]
    lat = lbm.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=ops)
    z = lat["coords"][:, 2]
    idx = np.flatnonzero(((z >= 3) & (z < 5)) | ((z >= z.max() - 5) & (z < z.max() - 3)))
    flux = {"idx": idx, "w": np.tile(np.array([[0, 0, 0.5]], np.float32), (len(idx), 1)),
            "slot": (z[idx] > 10).astype(int)}
    runs = []
    for order in ("c", "split"):
        s = ArterySolver(lat, 0.01, flux, [0.0, 0.05], 1e-4, 0.01, model="regularised", order=order)
        s.set_outlet_pressure([0.0, -1e-4])
        s.set_sponge(4, 0.55, kinds=("outlet",))
        s.set_drive([2e-4, 1e-4, 0.0], period=300, ramp=100)
        s.run(400)
        runs.append((s.fields(), s.Qlast.numpy()))
    (p0, u0), q0 = runs[0]
    (p1, u1), q1 = runs[1]
    # the flux partial sums add in another grouping: FP64 last-bit differences only
    np.testing.assert_allclose(q1, q0, rtol=1e-9, atol=1e-15)
    assert np.abs(u1 - u0).max() <= 1e-6 * np.abs(u0).max()


def test_autotune_picks_a_measured_candidate(golden):
    lat = lattice(golden, "stenosis70_D8")
    best, table = autotune.tune(lat, 0.02, configure=configure, blocks=(128, 256), steps=100, warmup=20,
                                model="regularised")
    assert len(table) >= 4 and best in table
    assert best["us_per_step"] == min(r["us_per_step"] for r in table)
