"""Host side of the heartbeat loop: the lumped circuit and its calibration, the Fourier helpers, coarse bins."""
import numpy as np
import pytest

from cerebrosim_b200 import simulate as S


def test_fourier_round_trip():
    t = np.arange(400) / 400
    y = 1.0 + 0.3 * np.cos(2 * np.pi * t) - 0.2 * np.sin(4 * np.pi * t) + 0.05 * np.cos(10 * np.pi * t)
    c = S.fourier(y, nh=10)
    assert len(c) == 21
    np.testing.assert_allclose(S.from_fourier(c, t), y, atol=1e-12)
    np.testing.assert_allclose(c[:5], [1.0, 0.3, 0.0, 0.0, -0.2], atol=1e-12)


def test_circuit_and_recalibration():
    shape = 1.0 + 0.4 * np.sin(2 * np.pi * np.arange(400) / 400)
    cal = S.circuit(0.0, shape, 240.0, 135.0, 80.0)
    q_in, q_t, p = 240e-6 / 60, 135e-6 / 60, 80.0 * S.MMHG
    assert cal["R_out"][1] == pytest.approx(p / q_t) and cal["R_out"][2] == pytest.approx(p / (q_in - q_t))
    assert cal["R_eq"] == pytest.approx(p / q_in)
    # the mean inlet pressure draws the mean inflow through R_eq: a0 = R_eq q_in = p
    assert cal["P_in_coef"][0] == pytest.approx(p)
    # a beat that needed 10 % more pressure for the same flow adds that resistance to the segment
    cal2 = S.recalibrate(cal, 1.1 * p, 240.0, shape, 240.0, 135.0, 80.0)
    assert cal2["R_seg"] == pytest.approx(0.1 * p / q_in)
    assert cal2["P_in_coef"][0] == pytest.approx(1.1 * p)
    assert S.recalibrate(cal, 0.9 * p, 240.0, shape, 240.0, 135.0, 80.0)["R_seg"] == 0.0


def test_circuit_matches_the_reference_golden():
    """The circuit and the calibrate branch against the reference's own simulate.circuit (tests/golden/circuit.json,
    written by make_golden.py from the reference's code and its flow targets and inflow waveform)."""
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "circuit.json")))
    a = g["inputs"]
    args = (np.asarray(a["shape"]), a["q_in_ml_min"], a["q_target_ml_min"], a["p_out_mmhg"])
    for ref in g["circuit"]:
        cal = S.circuit(ref["R_seg"], *args, nh=a["harmonics"])
        np.testing.assert_allclose(cal["R_out"], ref["R_out"], rtol=1e-13)
        np.testing.assert_allclose(cal["P_in_coef"], ref["P_in_coef"], rtol=1e-11, atol=1e-9)
        assert cal["R_eq"] == pytest.approx(ref["R_eq"], rel=1e-13)
    cal0 = S.circuit(0.0, *args, nh=a["harmonics"])
    for ref in g["recalibrate"]:
        cal = S.recalibrate(cal0, ref["p_in_pa"], ref["q_in_ml_min"], *args)
        assert cal["R_seg"] == pytest.approx(ref["R_seg"], rel=1e-13)
        np.testing.assert_allclose(cal["P_in_coef"], ref["P_in_coef"], rtol=1e-11, atol=1e-9)


def test_coarse_bins():
    rng = np.random.default_rng(0)
    coords = np.unique(rng.integers(0, 20, size=(500, 3)), axis=0)
    uk, inv, cnt, f = S.coarse_bins({"coords": coords}, 0.05, 0.1)
    assert f == 2 and cnt.sum() == len(coords)
    np.testing.assert_array_equal(uk[inv], coords // 2)
    uk1, inv1, cnt1, f1 = S.coarse_bins({"coords": coords}, 0.1, 0.1)
    assert f1 == 1 and np.all(cnt1 == 1) and len(uk1) == len(coords)
