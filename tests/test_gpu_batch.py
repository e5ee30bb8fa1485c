"""BatchSolver: several vessels in one persistent launch per step.

- Alone and in the mix: an instance in a batch of its own and the same instance in a batch with other vessels
  evolve bit for bit alike (same kernels, each instance on its own buffers, slab fluxes reduced in a fixed order
  without atomics), whatever the mix and whenever instances join or leave.
- Batched and dedicated kernels: the batched kernels and the single-lattice kernels are compiled separately and
  may round differently in the last bit; they agree within the path's tolerance, relative L2 <= 1e-5.
- Both batched forms: the persistent grid (blocks claim work items) and one block per work item (the 9-blocks-per-SM
  kernel of the regularised step without body force).
- The by-instance schedule runs each member with its own single-lattice kernels: bit for bit the member's solo run,
  joins and leaves included, and within 1e-5 of the fused schedule.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from cerebrosim_b200 import lbm  # noqa: E402
from cerebrosim_b200.batch import BatchSolver  # noqa: E402
from cerebrosim_b200.simulate import ArterySolver  # noqa: E402


def lattice(golden, name):
    meta, arr = golden.small_case(name)
    return lbm.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=meta["openings"],
                             periodic=meta["periodic"], opening_slack=meta["slack"])


def flux_for(lat):
    z = lat["coords"][:, 2]
    lo = np.flatnonzero((z >= 3) & (z < 5))
    hi = np.flatnonzero((z >= z.max() - 5) & (z < z.max() - 3))
    idx = np.concatenate([lo, hi])
    slot = np.concatenate([np.zeros(len(lo), int), np.ones(len(hi), int)])
    w = np.tile(np.array([[0.0, 0.0, 0.5]], np.float32), (len(idx), 1))
    return {"idx": idx, "w": w, "slot": slot}


SPECS = [("stenosis70_D8", dict(drive=([0.03], 1, 300), p=[0.0]), "plain"),
         ("open_pipe_tilted_R4", dict(drive=([0.02, 0.004, -0.003], 250, 100), p=[1e-4]), "plain"),
         ("box_openings_slack1", dict(drive=([0.01], 1, 100), p=[0.0, 2e-4, -1e-4]), "plain"),
         ("open_pipe_straight_R4", dict(drive=([2e-4, 1e-4, 0.0], 300, 100), p=None), "artery")]


def make(golden, name, cfg, kind, storage="f32"):
    lat = lattice(golden, name)
    if kind == "artery":
        ops = [dict(o, kind="outlet") for o in lat["openings"]]
        meta, arr = golden.small_case(name)
        lat = lbm.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=ops)
        s = ArterySolver(lat, 0.01, flux_for(lat), [0.0, 0.05], 1e-4, 0.01, model="regularised", storage=storage,
                         block=256)
        s.set_outlet_pressure([0.0, -1e-4])
        s.set_sponge(4, 0.55, kinds=("outlet",))
    else:
        s = lbm.Solver(lat, 0.02, model="regularised", storage=storage, block=256)
        s.set_sponge(4, 0.6)
        s.set_outlet_pressure(cfg["p"])
    coef, period, ramp = cfg["drive"]
    s.set_drive(coef, period=period, ramp=ramp)
    return s


def same(a, b):
    pa, ua = a.fields()
    pb, ub = b.fields()
    assert a.ok() and b.ok()
    assert np.array_equal(pa, pb) and np.array_equal(ua, ub)
    assert a.tick_value() == b.tick_value()
    if isinstance(a, ArterySolver):
        assert np.array_equal(a.Qlast.numpy(), b.Qlast.numpy())
        assert np.array_equal(a.p_out.cpu().numpy(), b.p_out.cpu().numpy())


def close(a, b, tol=1e-5):
    pa, ua = a.fields()
    pb, ub = b.fields()
    assert a.ok() and b.ok()
    e_u = np.sqrt(((ua - ub) ** 2).sum() / (ub ** 2).sum())
    e_r = np.sqrt(((3 * pa.astype(np.float64) - 3 * pb) ** 2).sum() / ((1 + 3 * pb.astype(np.float64)) ** 2).sum())
    assert e_u <= tol and e_r <= tol, (e_u, e_r)
    assert a.tick_value() == b.tick_value()


def run_alone(s, steps, chunk, persistent=True):
    """An instance in a batch of its own."""
    b = BatchSolver([s], persistent=persistent)
    b.run(steps, chunk=chunk)
    return b


@pytest.mark.parametrize("persistent", [True, False])
@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_batch_alone_and_in_the_mix(golden, storage, persistent):
    alone = [make(golden, n, c, k, storage) for n, c, k in SPECS]
    mixed = [make(golden, n, c, k, storage) for n, c, k in SPECS]
    for s in alone:
        run_alone(s, 501, 100, persistent)
    b = BatchSolver(mixed, persistent=persistent)
    b.run(501, chunk=100)
    assert b.steps == 501 and all(m.steps == 501 for m in mixed)
    for a, m in zip(alone, mixed):
        same(a, m)


@pytest.mark.parametrize("persistent", [True, False])
def test_batched_kernels_match_dedicated_kernels(golden, persistent):
    dedicated = [make(golden, n, c, k) for n, c, k in SPECS]
    batched = [make(golden, n, c, k) for n, c, k in SPECS]
    for s in dedicated:
        s.run(501, chunk=100)
    BatchSolver(batched, persistent=persistent).run(501, chunk=100)
    for a, m in zip(dedicated, batched):
        close(a, m)


def test_batch_members_join_and_leave(golden):
    """Continuous batching: instances join with their own parity and step count and leave mid-run."""
    alone = [make(golden, n, c, k) for n, c, k in SPECS]
    mixed = [make(golden, n, c, k) for n, c, k in SPECS]
    run_alone(mixed[1], 7, 40)                        # an odd head start: the member joins with parity 1
    b = BatchSolver(mixed[:2])
    b.run(100, chunk=40)
    b.add(mixed[2])
    b.run(130, chunk=40)
    b.remove(mixed[0])
    b.add(mixed[3])
    b.run(61, chunk=40)
    steps = [100 + 130, 7 + 100 + 130 + 61, 130 + 61, 61]
    for s, k in zip(alone, steps):
        run_alone(s, k, 40)
    for a, m in zip(alone, mixed):
        same(a, m)


@pytest.mark.parametrize("schedule", ["by-instance", "concurrent:2", "concurrent:4"])
def test_by_instance_schedule_is_the_solo_run(golden, schedule):
    """Member after member on the batch stream, or in groups on concurrent streams: each member's run is its solo
    run, bit for bit, joins and leaves included."""
    solo = [make(golden, n, c, k) for n, c, k in SPECS]
    mixed = [make(golden, n, c, k) for n, c, k in SPECS]
    fused = [make(golden, n, c, k) for n, c, k in SPECS]
    b = BatchSolver(mixed[:3], schedule=schedule)
    b.run(101, chunk=40)
    b.remove(mixed[1])
    b.add(mixed[3])
    b.run(60, chunk=40)
    steps = [161, 101, 161, 60]
    for s, k in zip(solo, steps):
        s.block = 128            # the batch's block size, which the members take on joining
        if hasattr(s, "_set_flux_blocks"):
            s._set_flux_blocks()
        s.run(k, chunk=40)
    for a, m in zip(solo, mixed):
        same(a, m)
    bf = BatchSolver(fused[:3])
    bf.run(101, chunk=40)
    bf.remove(fused[1])
    bf.add(fused[3])
    bf.run(60, chunk=40)
    for a, m in zip(fused, mixed):
        close(a, m)


def test_schedule_tuning_times_each_and_keeps_the_fastest(golden):
    from cerebrosim_b200 import autotune
    from cerebrosim_b200.batch import SCHEDULES
    members = [make(golden, n, c, k) for n, c, k in SPECS[:2]]
    b = BatchSolver(members)
    best, table = autotune.tune_schedule(b, steps=20, chunk=10, warmup=10)
    assert [r["schedule"] for r in table] == list(SCHEDULES)
    assert best["schedule"] == b.schedule == min(table, key=lambda r: r["us_per_step"])["schedule"]
    assert all(r["us_per_step"] > 0 for r in table)
    k = 30 * len(SCHEDULES)
    assert b.steps == k and all(m.steps == k and m.ok() for m in members)


def test_coupled_runs_are_reproducible(golden):
    """The resistance coupling reduces its flux without atomics: two runs agree bit for bit."""
    n, c, k = SPECS[3]
    r1, r2 = make(golden, n, c, k), make(golden, n, c, k)
    for s in (r1, r2):
        s.run(700, chunk=100)
    same(r1, r2)
    assert np.abs(r1.Qlast.numpy()).max() > 0
    assert torch.equal(r1.f[r1.cur], r2.f[r2.cur])


@pytest.mark.parametrize("schedule", ["fused", "by-instance", "concurrent:2"])
def test_graph_per_heartbeat_prepared_ahead(golden, schedule):
    """A heartbeat's steps as one CUDA graph per member (or per 400 steps for the fused schedule), captured by
    prepare() before the run: the same fields, bit for bit, as the same steps in graphs of 40."""
    beat = 600
    ref = [make(golden, n, c, k) for n, c, k in SPECS]
    got = [make(golden, n, c, k) for n, c, k in SPECS]
    BatchSolver(ref, schedule=schedule).run(2 * beat, chunk=40)
    b = BatchSolver(got, schedule=schedule)
    b.prepare(beat)
    b.run(2 * beat, chunk=beat)
    for a, m in zip(ref, got):
        same(a, m)
