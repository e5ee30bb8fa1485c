"""Parity of the fused GPU step (csrc/step.cu) with the CPU oracle (oracle/lbm_ref.cpp, the reference's k_clock +
k_step + k_flux + k_bc restated in FP32) on identical inputs.

Tolerance (the target the path is held to): after 1000 FP32 steps the relative L2 difference of the velocity and of
the density rho = 1 + delta_rho is at most 1e-5. The GPU reorders the collision's sums (moments instead of
link-by-link projections) and contracts multiply-adds differently, so bits differ; the fields must not.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from cerebrosim_b200 import cases, lbm  # noqa: E402
from cerebrosim_b200.simulate import ArterySolver  # noqa: E402
from oracle import lattice_ref as L  # noqa: E402
from oracle.step_ref import OracleSolver  # noqa: E402

TOL = 1e-5
STEPS = 1000


def rel_l2(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def compare(s_gpu, s_ref, tol=TOL):
    p_g, u_g = s_gpu.fields()
    p_r, u_r = s_ref.fields()
    assert s_gpu.ok() and s_ref.ok()
    e_u = rel_l2(u_g, u_r)
    e_rho = rel_l2(1.0 + 3.0 * p_g.astype(np.float64), 1.0 + 3.0 * p_r.astype(np.float64))
    assert np.abs(u_r).max() > 0, "the case does not move"
    assert e_u <= tol, f"velocity rel L2 {e_u:.3e}"
    assert e_rho <= tol, f"density rel L2 {e_rho:.3e}"
    assert s_gpu.tick_value() == int(s_ref.tick[0])
    assert float(s_gpu.drv.item()) == pytest.approx(float(s_ref.drv[0]), rel=1e-6, abs=1e-12)
    return e_u, e_rho


def lattice_from_golden(golden, name):
    meta, arr = golden.small_case(name)
    kw = dict(openings=meta["openings"], periodic=meta["periodic"], opening_slack=meta["slack"])
    return (lbm.build_lattice(arr["phi"], meta["origin"], meta["dx"], **kw),
            L.build_lattice(arr["phi"], meta["origin"], meta["dx"], **kw))


def both(lat_g, lat_r, nu, setup, **kw):
    g = lbm.Solver(lat_g, nu, **kw)
    r = OracleSolver(lat_r, nu, **kw)
    for s in (g, r):
        setup(s)
    return g, r


def test_periodic_pipe_body_force():
    c = cases.case("periodic_pipe_D10")
    lg, lr = lbm.build_lattice(**cases.lattice_args(c)), L.build_lattice(**cases.lattice_args(c))
    g, r = both(lg, lr, 0.02, lambda s: s.set_force([0, 0, 2e-5]), model="regularised")
    for s in (g, r):
        s.run(STEPS)
    compare(g, r)


def test_headline_pipe_at_full_size():
    """The bench's workload itself — the pulsatile pipe: open pipe R = 24, L = 192 (347,328 nodes) with the plug
    inlet, its Fourier drive and the pressure outlet, tau 0.55 — for 1000 steps against the oracle on the same
    tables."""
    c = cases.case("open_pipe_R24_L192")
    lg = cases.plug_inlet(lbm.build_lattice(**cases.lattice_args(c)))
    lr = cases.plug_inlet(L.build_lattice(**cases.lattice_args(c)))
    assert lg["nbr"].shape[1] == 347328
    for k in ("nbr", "q", "uin"):
        assert np.array_equal(lg[k], lr[k]), k

    def setup(s):
        s.set_drive([0.02, 0.0, 0.01], period=4000)
        s.set_outlet_pressure([0.0])
    g, r = both(lg, lr, (0.55 - 0.5) / 3.0, setup, model="regularised")
    for s in (g, r):
        s.run(STEPS)
    compare(g, r)


@pytest.mark.parametrize("storage,bound", [("f16", 3e-3), ("bf16", 3e-2)])
def test_headline_pipe_16bit_at_full_size(storage, bound):
    """The bench's 347,328-node pipe with 16-bit shifted storage, 300 steps, against the FP64 oracle of the same
    scheme: the bounds of the small-lattice 16-bit check hold at full size."""
    c = cases.case("open_pipe_R24_L192")
    lg = cases.plug_inlet(lbm.build_lattice(**cases.lattice_args(c)))
    lr = cases.plug_inlet(L.build_lattice(**cases.lattice_args(c)))
    g = lbm.Solver(lg, (0.55 - 0.5) / 3.0, model="regularised", storage=storage)
    r = OracleSolver(lr, (0.55 - 0.5) / 3.0, model="regularised", dtype=np.float64)
    for s in (g, r):
        s.set_drive([0.02, 0.0, 0.01], period=4000)
        s.set_outlet_pressure([0.0])
        s.run(300)
    _, u_g = g.fields()
    _, u_r = r.fields()
    assert g.ok()
    assert rel_l2(u_g.astype(np.float64), u_r) <= bound


def test_stenosed_artery_at_full_size():
    """The batched / served workloads' vessel at its full size: the generated stenosed artery of seed 3 at 0.05 mm
    (1,567,027 nodes; Bouzidi walls, Fourier velocity inlet, two pressure outlets, sponge), 1000 FP32 steps against
    the oracle on the same tables, in the lattice's C order and in the vessel-axis orders the autotuner picks."""
    from cerebrosim_b200 import workloads
    spec = {"seed": 3, "stenosis": 0.7, "pressure": 95.0}
    lat = workloads.lattice(workloads.stenosed_vessel(3), 0.05)
    assert lat["nbr"].shape[1] == 1567027
    r = OracleSolver(lat, (0.52 - 0.5) / 3.0, model="regularised")
    workloads.configure(r, spec, lat, period=8000)
    r.run(STEPS)
    for order in ("c", "axis-split", "axis-boundary-first"):
        g = workloads.make_solver(spec, lat, period=8000, order=order)
        g.run(STEPS)
        compare(g, r)


def test_poiseuille_cylinder_tau08():
    """The small Poiseuille cylinder: R = 10, 24 x 24 x 64 periodic, tau = 0.8, g = 1e-6."""
    c = cases.case("poiseuille_R10_L64")
    lg, lr = lbm.build_lattice(**cases.lattice_args(c)), L.build_lattice(**cases.lattice_args(c))
    g, r = both(lg, lr, 0.1, lambda s: s.set_force([0, 0, 1e-6]), model="regularised")
    for s in (g, r):
        s.run(STEPS)
    compare(g, r)


@pytest.mark.parametrize("model,sigma,gal,bouzidi", [("regularised", 1.0, None, True),
                                                     ("regularised", 0.6, None, True),
                                                     ("regularised", 1.0, False, False),
                                                     ("trt", 1.0, None, True)])
def test_open_pipe_inlet_outlet_sponge(golden, model, sigma, gal, bouzidi):
    lg, lr = lattice_from_golden(golden, "open_pipe_tilted_R4")

    def setup(s):
        s.set_sponge(4, 0.6)
        s.set_drive([0.02, 0.004, -0.003, 0.002, 0.001], period=300, ramp=150)
        s.set_outlet_pressure([1e-4])
    g, r = both(lg, lr, 0.02, setup, model=model, sigma=sigma, galilean=gal, bouzidi=bouzidi)
    for s in (g, r):
        s.run(STEPS)
    compare(g, r)


def test_block_sizes_agree(golden):
    """Every bulk block size gives the oracle's fields; the sizes of at most 128 threads run one build of the kernel
    (9 blocks of 128 per SM) and agree bit for bit."""
    lg, lr = lattice_from_golden(golden, "open_pipe_tilted_R4")

    def setup(s):
        s.set_sponge(4, 0.6)
        s.set_drive([0.02, 0.004, -0.003], period=300, ramp=150)
        s.set_outlet_pressure([1e-4])
    r = OracleSolver(lr, 0.02, model="regularised")
    setup(r)
    r.run(STEPS)
    dense = []
    for block in (32, 64, 96, 128, 192, 256):
        g = lbm.Solver(lg, 0.02, model="regularised", block=block)
        setup(g)
        g.run(STEPS)
        compare(g, r)
        if block <= 128:
            dense.append(g.fields())
    for p, u in dense[1:]:
        assert np.array_equal(p, dense[0][0]) and np.array_equal(u, dense[0][1])


def test_stenosis_small(golden):
    lg, lr = lattice_from_golden(golden, "stenosis70_D8")

    def setup(s):
        s.set_sponge(8, 0.55)
        s.set_drive([0.03], ramp=300)
        s.set_outlet_pressure([0.0])
    g, r = both(lg, lr, 0.01, setup, model="regularised")
    for s in (g, r):
        s.run(STEPS)
    compare(g, r)


def test_several_openings_and_irregular_walls(golden):
    """Two inlets, three outlets with their own pressures, q < 0.5 and q >= 0.5 walls."""
    lg, lr = lattice_from_golden(golden, "box_openings_slack1")

    def setup(s):
        s.set_sponge(3, 0.7)
        s.set_drive([0.01], ramp=100)
        s.set_outlet_pressure([0.0, 2e-4, -1e-4])
    g, r = both(lg, lr, 0.05, setup, model="regularised")
    for s in (g, r):
        s.run(STEPS)
    compare(g, r)


def test_artery_solver_flux_and_outlet_resistance(golden):
    """simulate.py's coupling: slab fluxes reduced in the step, outlet pressures relaxed towards R Q - pref."""
    meta, arr = golden.small_case("stenosis70_D8")
    ops = [dict(o, kind="outlet") for o in meta["openings"]]     # simulate.py declares every end an outlet
    lg = lbm.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=ops)
    lr = L.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=ops)
    coords = lr["coords"]
    z = coords[:, 2]
    idx = np.concatenate([np.flatnonzero((z >= 6) & (z < 8)), np.flatnonzero((z >= z.max() - 8) & (z < z.max() - 6))])
    slot = np.concatenate([np.zeros(((z >= 6) & (z < 8)).sum(), int), np.ones(((z >= z.max() - 8) & (z < z.max() - 6)).sum(), int)])
    w = np.where(slot[:, None] == 0, [[0, 0, 0.5]], [[0, 0, 0.5]]).astype(np.float32)
    flux = {"idx": idx[::-1].copy(), "w": w[::-1].copy(), "slot": slot[::-1].copy()}   # unsorted on purpose
    R, pref, alpha = [0.0, 0.05], 1e-4, 0.01
    g = ArterySolver(lg, 0.01, flux, R, pref, alpha, model="regularised")
    r = OracleSolver(lr, 0.01, model="regularised", flux=flux, R_lu=R, pref_lu=pref, alpha=alpha)
    for s in (g, r):
        s.set_outlet_pressure([0.0, -pref])
        s.set_sponge(6, 0.55, kinds=("outlet",))
        s.set_drive([2e-4, 1e-4, 0.0], period=500, ramp=200)
    for s in (g, r):
        s.run(STEPS)
    compare(g, r)
    q_g, q_r = g.Qlast.numpy(), r.Qlast
    assert np.abs(q_r).max() > 0
    assert rel_l2(q_g, q_r) <= 1e-5
    p_g, p_r = g.p_out.cpu().numpy(), r.p_out
    assert rel_l2(p_g.astype(np.float64), p_r.astype(np.float64)) <= 1e-5
    assert np.all(g.Qacc.numpy() == 0)


def test_graph_and_single_launches_identical(golden):
    lg, _ = lattice_from_golden(golden, "open_pipe_straight_R4")
    a = lbm.Solver(lg, 0.02, model="regularised")
    b = lbm.Solver(lg, 0.02, model="regularised")
    c = lbm.Solver(lg, 0.02, model="regularised")
    for s in (a, b, c):
        s.set_sponge(4, 0.6)
        s.set_drive([0.02], ramp=100)
    a.run(1001, chunk=100)
    for _ in range(1001):
        b._launch(b.cur)
        b.cur = 1 - b.cur
    b.steps = 1001
    c.run(1001, chunk=2000)          # no full chunk: the 1001 leftover steps in one library call
    pa, ua = a.fields()
    pb, ub = b.fields()
    pc, uc = c.fields()
    assert a.cur == b.cur == c.cur == 1 and c.steps == 1001 and c.tick_value() == b.tick_value()
    assert np.array_equal(pa, pb) and np.array_equal(ua, ub)
    assert np.array_equal(pc, pb) and np.array_equal(uc, ub)
    assert torch.equal(a.f[a.cur], b.f[b.cur]) and torch.equal(c.f[c.cur], b.f[b.cur])


def test_subclass_launch_hook_is_captured(golden):
    """A subclass that extends _launch (as simulate.ArterySolver does in the reference) still runs in graphs."""
    lg, _ = lattice_from_golden(golden, "open_pipe_straight_R4")

    class Counting(lbm.Solver):
        def _launch(self, a):
            super()._launch(a)
            self.rho.add_(0.0)
            self.counter += 1

    s = Counting.__new__(Counting)
    s.counter = 0
    lbm.Solver.__init__(s, lg, 0.02, model="regularised")
    ref = lbm.Solver(lg, 0.02, model="regularised")
    for x in (s, ref):
        x.set_sponge(4, 0.6)
        x.set_drive([0.02], ramp=100)
        x.run(400, chunk=100)
    assert s.counter == 100                        # captured once, replayed 4 times
    assert s.ok() and np.array_equal(s.fields()[1], ref.fields()[1])


@pytest.mark.parametrize("storage,bound", [("f16", 3e-3), ("bf16", 3e-2)])
def test_16bit_storage_error_vs_fp64_oracle(golden, storage, bound):
    """16-bit shifted storage with FP32 arithmetic, against the FP64 oracle of the same scheme."""
    lg, lr = lattice_from_golden(golden, "stenosis70_D8")

    def setup(s):
        s.set_sponge(8, 0.55)
        s.set_drive([0.03], ramp=300)
        s.set_outlet_pressure([0.0])
    g = lbm.Solver(lg, 0.01, model="regularised", storage=storage)
    r = OracleSolver(lr, 0.01, model="regularised", dtype=np.float64)
    for s in (g, r):
        setup(s)
        s.run(STEPS)
    _, u_g = g.fields()
    _, u_r = r.fields()
    assert g.ok()
    assert rel_l2(u_g.astype(np.float64), u_r) <= bound


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_checkpoint_resume_is_bit_exact(golden, tmp_path, storage):
    """A run checkpointed after an odd number of steps (the state in the second buffer) and resumed on a fresh
    solver from the saved file ends bit for bit where the uninterrupted run ends; the coupled artery solver's flows
    and outlet pressures too."""
    lg, _ = lattice_from_golden(golden, "open_pipe_tilted_R4")

    def setup(s):
        s.set_sponge(4, 0.6)
        s.set_drive([0.02, 0.004, -0.003], period=300, ramp=150)
        s.set_outlet_pressure([1e-4])
    a = lbm.Solver(lg, 0.02, model="regularised", storage=storage)
    setup(a)
    a.run(333, chunk=100)
    a.save(tmp_path / "ck.pt")
    a.run(200, chunk=100)
    b = lbm.Solver(lg, 0.02, model="regularised", storage=storage)
    b.load(tmp_path / "ck.pt")
    assert b.steps == 333 and b.tick_value() == 333
    b.run(200, chunk=100)
    (pa, ua), (pb, ub) = a.fields(), b.fields()
    assert np.array_equal(pa, pb) and np.array_equal(ua, ub) and a.tick_value() == b.tick_value() == 533
    with pytest.raises(ValueError):
        lbm.Solver(lg, 0.02, model="regularised", storage="f16" if storage != "f16" else "f32").restore(a.checkpoint())


def test_checkpoint_resume_artery_solver(golden):
    lg, _ = lattice_from_golden(golden, "open_pipe_tilted_R4")
    z = lg["coords"][:, 2]
    idx = np.flatnonzero((z >= 6) & (z < 8))
    flux = {"idx": idx, "w": np.tile([0.0, 0.0, 0.5], (len(idx), 1)), "slot": np.zeros(len(idx), np.int32)}

    def make():
        s = ArterySolver(lg, 0.02, flux, [0.0], 1e-4, 0.01, model="regularised")
        s.set_drive([0.0, 1e-3], period=200)
        return s
    a = make()
    a.run(101, chunk=50)
    st = a.checkpoint()
    a.run(100, chunk=50)
    b = make()
    b.restore(st)
    b.run(100, chunk=50)
    assert np.array_equal(a.fields()[1], b.fields()[1])
    assert np.array_equal(a.Qlast.numpy(), b.Qlast.numpy()) and np.array_equal(a.p_out64.cpu().numpy(),
                                                                                b.p_out64.cpu().numpy())
