"""The oracle's vessel signed distance (vessel.py:178-245) on the reference's own centrelines.

The reference's kernel cannot run here; its field is pinned on the GPU through the published healthy-artery lattice
(tests/test_gpu_vessel.py). These checks hold the restatement to what the construction implies: the field is minus
the radius on the centreline away from junctions and ends, positive outside the box the radii span, and the smooth
minimum reduces to the plain minimum away from the blend band.
"""
import numpy as np

from oracle import sdf_ref


def pk_of(v):
    return (v["pts"], v["rad"], v["start"], v["count"], v["cap_p"], v["cap_n"], v["cap_r"], v["meta"]["blend"])


def test_packed_layout(golden):
    for case in ("healthy", "narrow70", "occluded"):
        v = golden.vessel(case)
        assert v["meta"]["names"] == ["trunk", "blocked", "sibling"]
        assert v["start"][0] == 0 and (np.diff(v["start"]) == v["count"][:-1]).all()
        assert v["start"][-1] + v["count"][-1] == len(v["pts"]) == len(v["rad"])
        # an open end has a cap radius equal to the end radius; inlet first among the openings
        ops = v["meta"]["openings"]
        assert [o["kind"] for o in ops] == ["inlet", "outlet", "outlet"]
        assert (v["cap_r"] > 0).sum() == len(ops)
        assert sdf_ref.grid_shape(v["lo"], v["hi"], 0.1) == (544, 229, 372)


def test_smin():
    a = np.array([0.0, 1.0, -2.0, 5.0], np.float32)
    b = np.array([3.0, 1.0, -2.1, -5.0], np.float32)
    got = sdf_ref.smin(a, b, 0.6)
    assert got[0] == 0.0 and got[3] == -5.0                  # |a - b| >= k: the plain minimum
    assert got[1] == np.float32(1.0) - np.float32(0.15)      # a == b: h = 1/2, min - k/4
    assert got[2] < -2.1


def test_centreline_is_minus_radius(golden):
    v = golden.vessel("healthy")
    pk = pk_of(v)
    s0, c0 = int(v["start"][0]), int(v["count"][0])
    idx = np.arange(s0 + 10, s0 + c0 - 10, 7)               # trunk interior, away from the inlet cap
    p = v["pts"][idx].astype(np.float32)
    # keep points farther than the blend band plus the other branches' radii from every other branch
    other = np.concatenate([v["pts"][int(s):int(s) + int(c)] for s, c in zip(v["start"][1:], v["count"][1:])])
    far = np.min(np.linalg.norm(p[:, None, :] - other[None, :, :], axis=2), axis=1) > 3.0 + v["rad"].max()
    assert far.sum() >= 5
    d = sdf_ref.sdf_points(p[far], *pk)
    np.testing.assert_allclose(d, -v["rad"][idx][far], rtol=0, atol=1e-5)


def test_box_corners_outside(golden):
    v = golden.vessel("narrow70")
    lo, hi = v["lo"], v["hi"]
    corners = np.array([[x, y, z] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])])
    assert (sdf_ref.sdf_points(corners, *pk_of(v)) > 0).all()


def test_coarse_grid_inside_fraction(golden):
    """At 1 mm the lumen holds a few hundred voxels; the clotted case holds fewer than the healthy one."""
    vols = {}
    for case in ("healthy", "occluded"):
        v = golden.vessel(case)
        phi = sdf_ref.sdf_grid(pk_of(v), v["lo"], v["hi"], 1.0)
        assert phi.dtype == np.float32 and phi.shape == sdf_ref.grid_shape(v["lo"], v["hi"], 1.0)
        vols[case] = int((phi < 0).sum())
    # the healthy lumen: about 620,028 voxels of 1e-3 mm^3 at 0.1 mm, i.e. about 620 mm^3
    assert 450 < vols["healthy"] < 800
    assert vols["occluded"] < vols["healthy"]
