"""GPU vessel signed distance and the artery lattice built from it (vessel.py:178-245, validate.py:294-308).

- Against the oracle: the kernel's field equals the NumPy restatement's within a few float32 ulps of the distance
  (both evaluate the same float32 expressions; the compilers may fuse multiply-adds differently).
- Against the reference's published artery: the healthy vessel at dx 0.1 mm gives the reference's lattice exactly,
  620,028 fluid cells with 747,143 wall, 11,400 inlet and 2,649 / 2,682 outlet links (geometry/solver.json).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from cerebrosim_b200 import vessel  # noqa: E402
from oracle import sdf_ref  # noqa: E402

PUBLISHED_HEALTHY = {"cells": 620028, "counts": {"wall": 747143, "inlet": 11400, "outlet": [2649, 2682]}}


def packed(v):
    m = v["meta"]
    return vessel.Packed(m["names"], v["pts"], v["rad"], v["start"], v["count"], v["cap_p"], v["cap_n"], v["cap_r"],
                         m["blend"])


def openings(v):
    return [dict(o, centre=np.asarray(o["centre"]), normal=np.asarray(o["normal"])) for o in v["meta"]["openings"]]


@pytest.mark.parametrize("case", ["healthy", "occluded"])
def test_sdf_matches_oracle(golden, case):
    v = golden.vessel(case)
    pk = packed(v)
    dx = 0.7
    gpu, origin = vessel.sdf_grid(pk, dx, v["lo"], v["hi"])
    ref = sdf_ref.sdf_grid(pk.arrays(), v["lo"], v["hi"], dx)
    assert gpu.shape == ref.shape and gpu.dtype == np.float32
    np.testing.assert_array_equal(origin, v["lo"])
    err = np.abs(gpu.astype(np.float64) - ref)
    assert err.max() <= 2e-5 * max(1.0, np.abs(ref).max()), err.max()
    near = np.abs(ref) < 1e-4
    assert ((gpu < 0) == (ref < 0))[~near].all()


def test_healthy_artery_matches_published_lattice(golden):
    v = golden.vessel("healthy")
    lat = vessel.artery_lattice(packed(v), 0.1, openings=openings(v), lo=v["lo"], hi=v["hi"])
    assert lat["shape"] == (544, 229, 372)
    assert lat["nbr"].shape[1] == PUBLISHED_HEALTHY["cells"]
    assert lat["counts"] == PUBLISHED_HEALTHY["counts"]
    assert [o["kind"] for o in lat["openings"]] == ["inlet", "outlet", "outlet"]


def test_empty_and_invalid_vessels(golden):
    v = golden.vessel("healthy")
    with pytest.raises(ValueError):
        vessel.Packed(["a"], v["pts"][:3], v["rad"][:3], [0], [5], np.zeros((2, 3)), np.zeros((2, 3)), [0, 0])
    # no branch at all: the field is the initial 1e9 everywhere, so no fluid
    empty = vessel.Packed([], np.zeros((0, 3)), np.zeros(0), [], [], np.zeros((0, 3)), np.zeros((0, 3)), [])
    phi, _ = vessel.sdf_grid(empty, 1.0, [0, 0, 0], [2, 3, 4])
    assert phi.shape == (3, 4, 5) and (phi == np.float32(1e9)).all()
