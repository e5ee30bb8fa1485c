"""The step oracle (oracle/lbm_ref.cpp) pinned against the reference's published validation results.

The reference's GPU code cannot run here, so no stored populations exist; its published errors
(reports/step3_report.md:20-33, geometry/solver.json:20-84) pin the restated step instead. With multiply-add
contraction (as the reference's GPU compiler does) the FP32 restatement reproduces them to 4-6 digits.
"""
import numpy as np
import pytest

from oracle import validation as V
from oracle import lattice_ref as L
from oracle.step_ref import OracleSolver


def test_poiseuille_d10_matches_published():
    r = V.poiseuille(L.build_lattice, OracleSolver, 10, True)
    l2_ref, flow_ref = V.PUBLISHED["poiseuille"][(10, True)]
    assert r["ok"]
    assert r["l2"] == pytest.approx(l2_ref, rel=1e-4)
    assert r["flow_err"] == pytest.approx(flow_ref, rel=1e-4)


def test_poiseuille_d20_halfway_matches_published():
    r = V.poiseuille(L.build_lattice, OracleSolver, 20, False)
    l2_ref, flow_ref = V.PUBLISHED["poiseuille"][(20, False)]
    assert r["l2"] == pytest.approx(l2_ref, rel=5e-4)
    assert r["flow_err"] == pytest.approx(flow_ref, rel=5e-4)


def test_womersley_wo56_matches_published():
    r = V.womersley(L.build_lattice, OracleSolver, 5.6)
    T, l2_ref = V.PUBLISHED["womersley"][5.6]
    assert r["period_steps"] == T
    assert r["l2"] == pytest.approx(l2_ref, rel=1e-5)


def test_fp64_oracle_close_to_fp32():
    """The FP64 oracle of the same scheme: same steady state to the FP32 rounding level (~1e-3 at tau 0.505)."""
    r32 = V.poiseuille(L.build_lattice, OracleSolver, 10, True)
    r64 = V.poiseuille(L.build_lattice, lambda *a, **k: OracleSolver(*a, dtype=np.float64, **k), 10, True)
    assert r64["l2"] == pytest.approx(r32["l2"], rel=2e-3)


def test_open_boundaries_short_run_is_stable(golden):
    """Velocity inlet + pressure outlet + sponge + TRT / regularised on a small tilted pipe: finite and flowing."""
    meta, arr = golden.small_case("open_pipe_tilted_R4")
    lat = L.build_lattice(arr["phi"], meta["origin"], meta["dx"], openings=meta["openings"])
    for model in ("regularised", "trt"):
        s = OracleSolver(lat, 0.01, model=model)
        s.set_sponge(4, 0.6)
        s.set_drive([0.02], ramp=200)
        s.set_outlet_pressure([0.0])
        s.run(600)
        p, u = s.fields()
        assert s.ok() and np.abs(u).max() > 1e-3 and np.abs(u).max() < 0.1
