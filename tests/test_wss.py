"""Wall shear stress: the package's fit against the reference's own wss.py on the reference's method check.

tests/golden/make_wss_golden.py ran the reference's `weights` and `shear` (wss.py:35-57) on the cylinders of its
`--test` (radius 0.4 - 2.0 mm on a 0.1 mm grid, Poiseuille and blunt profiles); `pipe_cases` there rebuilds the
same inputs. The fit coefficients must agree to float32 rounding, the shear to 1e-5, and the Poiseuille cases keep
the reference's known answer 2 mu u_max / R.
"""
import json
import os
import sys

import numpy as np
import pytest

from cerebrosim_b200 import wss

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_wss_golden import pipe_cases  # noqa: E402

G = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(G, "wss.npz")), json.load(open(os.path.join(G, "wss.json")))


@pytest.fixture(scope="module")
def cases():
    return pipe_cases()


def host_shear(U, normals, idx, c, mu=wss.MU):
    """wss.py:50-55 restated on the host, for the CPU check of the fit coefficients."""
    u = U[idx]
    ut = u - np.einsum("vkc,vc->vk", u, normals)[..., None] * normals[:, None, :]
    return mu * 1e3 * (c[..., None].astype(float) * ut).sum(1)


def test_constants_match_reference(golden):
    _, meta = golden
    assert meta["mu_pa_s"] == wss.MU and meta["K"] == wss.K
    assert (meta["d_min"], meta["d_max"], meta["sigma"]) == (wss.D_MIN, wss.D_MAX, wss.SIGMA)


def test_fit_matches_reference(golden, cases):
    arr, meta = golden
    for k, (R, pw, cells, depth, U, verts, normals) in enumerate(cases):
        idx, c, quad, any_ = wss.weights(verts, normals, cells, depth)
        assert np.array_equal(quad, arr[f"{k}/quad"]) and np.array_equal(any_, arr[f"{k}/any"])
        if f"{k}/c" in arr.files:
            assert np.array_equal(idx, arr[f"{k}/idx"])
            np.testing.assert_allclose(c, arr[f"{k}/c"], rtol=2e-6, atol=1e-9)
        tau = host_shear(U, normals, idx, c)
        np.testing.assert_allclose(tau, arr[f"{k}/tau"], rtol=1e-5, atol=1e-9)
        mag = np.linalg.norm(tau, axis=1).mean()
        if pw == 2:                                    # exact for the parabola: 2 mu u_max / R
            assert mag == pytest.approx(meta["cases"][k]["exact_pa"], rel=1e-6)
        assert mag == pytest.approx(meta["cases"][k]["mean_pa"], rel=1e-6)


@pytest.mark.gpu
def test_gpu_shear_matches_reference(golden, cases):
    arr, _ = golden
    for k, (R, pw, cells, depth, U, verts, normals) in enumerate(cases):
        idx, c, quad, any_ = wss.weights(verts, normals, cells, depth)
        sh = wss.Shear(normals, idx, c, len(cells))
        tau = sh(U.astype(np.float32)).cpu().numpy()
        np.testing.assert_allclose(tau, arr[f"{k}/tau"], rtol=1e-5, atol=1e-6)
