"""The reference's own drivers, unmodified, on this package (cerebrosim_b200.refshim).

REFERENCE_DIR names a checkout of CerebroSim (its validate.py, vessel.py and simulate.py are imported from there,
not copied); without it every test here is skipped. On the host: the scripts import through the stand-in modules and
bind to this package. On the GPU: validate.py's own Poiseuille and open-pipe checks run through cerebrosim_b200.lbm
and reproduce the results the reference published (geometry/solver.json:20-120), within the tolerances of
tests/test_gpu_validation.py.
"""
import os

import pytest

from oracle import validation as V

REF = os.environ.get("REFERENCE_DIR")
pytestmark = pytest.mark.skipif(not (REF and os.path.exists(os.path.join(REF, "validate.py"))),
                                reason="REFERENCE_DIR (a CerebroSim checkout) not set")


@pytest.fixture
def ref_modules():
    from cerebrosim_b200 import refshim
    saved = refshim.install(REF)
    try:
        yield refshim
    finally:
        refshim.uninstall(saved)


def test_reference_scripts_bind_to_this_package(ref_modules):
    from cerebrosim_b200 import lbm, simulate as ours
    validate = ref_modules.load("validate")
    assert validate.lbm is lbm and validate.__file__.startswith(os.path.abspath(REF))
    assert validate.V.sdf_grid.__module__ == "cerebrosim_b200.refshim"
    simulate = ref_modules.load("simulate")
    assert simulate.lbm is lbm and simulate.ArterySolver is ours.ArterySolver
    # the reference's host-side helpers run as they are
    assert simulate.circuit(0.0)["R_eq"] > 0
    with pytest.raises(NotImplementedError, match="cerebrosim_b200"):
        validate.wp.launch(None, dim=1)


@pytest.mark.gpu
def test_reference_validate_poiseuille_and_open_pipe(ref_modules):
    validate = ref_modules.load("validate")
    un = validate.units("healthy")
    for o in validate.test_poiseuille(un.nu_lu):
        l2_ref, flow_ref = V.PUBLISHED["poiseuille"][(o["D"], o["bouzidi"])]
        assert o["ok"]
        tol = 5e-2 if o["D"] == 40 else 1e-2        # D = 40: FP32 rounding over 586,851 steps
        assert o["l2"] == pytest.approx(l2_ref, rel=tol) and o["flow_err"] == pytest.approx(flow_ref, rel=tol)
    for o in validate.test_open_pipe():
        ref = V.PUBLISHED["open_pipe"][o["name"]]
        assert o["ok"]
        for k in ("grad_err", "profile_l2", "flow_vs_inlet"):
            assert o[k] == pytest.approx(ref[k], abs=3e-3), k
