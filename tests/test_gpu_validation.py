"""The reference's own validation suite (validate.py checks 1-4) run on the GPU solver, against the results the
reference published (geometry/solver.json:20-175, reports/step3_report.md:20-50).

Tolerances: at tau ~ 0.502-0.505 an FP32 steady state depends on rounding at the 1e-3 level. For the D = 20
Poiseuille error the FP64 oracle of the scheme gives 3.4398 %, the FP32 CPU restatement 3.4379 % without and
3.4295 % with multiply-add contraction, the reference's FP32 GPU run 3.4291 %: FP32 results scatter by +-0.3 %
around FP64. So Poiseuille and Womersley errors must agree with the published ones to 1 % relative; the open-pipe
numbers to 0.3 percentage points; the steady stenosis pressure drop to 1 % and the unsteady Re 200 jet (whose last
flow-through varies by 0.7-1.4 %) to 3 %.
"""
import pytest
import torch

pytestmark = pytest.mark.gpu

from cerebrosim_b200 import lbm  # noqa: E402
from oracle import validation as V  # noqa: E402

P = V.PUBLISHED


# D = 40, interpolated walls: the FP64 oracle of the scheme (oracle/lbm_ref.cpp in double, run on the host) gives
# L2 0.93585 % and flow error -1.04945 %. The reference's FP32 run published 0.91874 % (1.8 % below it); FP32 CPU
# restatements land at 0.91888 % (reference order, contracted) and this GPU path at 0.9534 % (1.9 % above). With a
# body force of 3.3e-7 balanced over 586,851 steps at tau 0.505 every FP32 evaluation order rounds its own way, so
# this case is checked against the FP64 value within 3 %.
FP64_D40 = (0.009358519314586382, -0.010494494415846045)


@pytest.mark.parametrize("D,bz", [(10, True), (20, True), (40, True), (20, False)])
def test_poiseuille(D, bz):
    r = V.poiseuille(lbm.build_lattice, lbm.Solver, D, bz)
    print("poiseuille", D, bz, r)
    l2_ref, flow_ref = P["poiseuille"][(D, bz)]
    assert r["ok"]
    if D == 40:
        assert r["l2"] == pytest.approx(FP64_D40[0], rel=3e-2)
        assert r["flow_err"] == pytest.approx(FP64_D40[1], rel=3e-2)
        assert r["l2"] == pytest.approx(l2_ref, rel=5e-2)
        return
    assert r["l2"] == pytest.approx(l2_ref, rel=1e-2)
    assert r["flow_err"] == pytest.approx(flow_ref, rel=1e-2)


@pytest.mark.parametrize("Wo", [1.4, 2.8, 5.6])
def test_womersley(Wo):
    r = V.womersley(lbm.build_lattice, lbm.Solver, Wo)
    print("womersley", Wo, r)
    T, l2_ref = P["womersley"][Wo]
    assert r["ok"] and r["period_steps"] == T
    assert r["l2"] == pytest.approx(l2_ref, rel=1e-2)


@pytest.mark.parametrize("name", ["straight", "tilted"])
def test_open_pipe(name):
    r = V.open_pipe(lbm.build_lattice, lbm.Solver, name)
    print("open_pipe", name, r)
    ref = P["open_pipe"][name]
    assert r["ok"]
    assert r["grad_err"] == pytest.approx(ref["grad_err"], abs=3e-3)
    assert r["profile_l2"] == pytest.approx(ref["profile_l2"], abs=3e-3)
    assert r["flow_vs_inlet"] == pytest.approx(ref["flow_vs_inlet"], abs=3e-3)


@pytest.mark.parametrize("key,Re,rel", [("narrow70", 100, 1e-2), ("narrow70", 200, 3e-2),
                                        ("narrow70_fine", 200, 3e-2)])
def test_stenosis(key, Re, rel):
    r = V.stenosis(lbm.build_lattice, lbm.Solver, key, Re, sync=torch.cuda.synchronize)
    print("stenosis", key, Re, r)
    ref = P["stenosis"][(key, Re)]
    assert r["ok"]
    assert r["dp_Pa"] == pytest.approx(ref["dp_Pa"], rel=rel)
    assert r["mlups"] > ref["mlups"]               # faster than the reference's RTX 3090 run
