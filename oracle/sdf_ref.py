"""NumPy restatement of CerebroSim's vessel signed distance — TEST INFRASTRUCTURE (the oracle), never the product path.

Follows vessel.py:178-181 (`_smin`), vessel.py:184-207 (`k_sdf`), vessel.py:210-221 (`_packed`), vessel.py:224-227
(`bounds`) and vessel.py:230-245 (`sdf_grid`), in float32 like the reference's kernel, vectorised over voxels.
The reference evaluates the field with a GPU kernel (Warp) that is not importable here; its output is pinned through
the artery it builds: the published healthy-artery lattice (geometry/solver.json: 620,028 cells at dx 0.1 mm, link
counts wall 747,143 / inlet 11,400 / outlets 2,649 and 2,682), which the GPU path must reproduce exactly.
"""
import numpy as np

F = np.float32


def smin(a, b, k):
    """vessel.py:178-181: polynomial smooth minimum."""
    h = np.clip(F(0.5) + F(0.5) * (b - a) / F(k), F(0.0), F(1.0)).astype(F)
    return (b + (a - b) * h - F(k) * h * (F(1.0) - h)).astype(F)


def sdf_points(p, pts, rad, start, count, cap_p, cap_n, cap_r, blend):
    """vessel.py:184-207 at the points p (M, 3) float32 -> (M,) float32."""
    p = np.asarray(p, F)
    pts, rad = np.asarray(pts, F), np.asarray(rad, F)
    cap_p, cap_n, cap_r = np.asarray(cap_p, F), np.asarray(cap_n, F), np.asarray(cap_r, F)
    d = np.full(len(p), F(1.0e9), F)
    for b in range(len(start)):
        db = np.full(len(p), F(1.0e9), F)
        s0 = int(start[b])
        for s in range(s0, s0 + int(count[b]) - 1):
            a = pts[s]
            ab = pts[s + 1] - a
            t = np.clip(((p - a) @ ab) / max(F(ab @ ab), F(1.0e-12)), F(0.0), F(1.0)).astype(F)
            r = rad[s] + (rad[s + 1] - rad[s]) * t
            e = p - (a + ab[None, :] * t[:, None])
            db = np.minimum(db, np.sqrt((e * e).sum(1)) - r)
        for e in range(2):
            c = b * 2 + e
            if cap_r[c] > 0.0:
                q = p - cap_p[c]
                near = np.sqrt((q * q).sum(1)) < F(2.5) * cap_r[c]
                db = np.where(near, np.maximum(db, q @ cap_n[c]), db).astype(F)
        d = smin(d, db, blend)
    return d


def grid_shape(lo, hi, dx):
    """vessel.py:235-236: voxel counts of the box [lo, hi] at spacing dx."""
    return tuple(int(x) for x in np.ceil((np.asarray(hi) - np.asarray(lo)) / dx).astype(int) + 1)


def sdf_grid(pk, lo, hi, dx):
    """vessel.py:230-245 on a packed vessel (pts, rad, start, count, cap_p, cap_n, cap_r, blend): the field on the
    voxel centres lo + (i, j, k) dx, float32 (nx, ny, nz)."""
    n = grid_shape(lo, hi, dx)
    org = np.asarray(lo, F)
    ii = np.indices(n, dtype=F).reshape(3, -1).T
    p = org[None, :] + ii * F(dx)
    return sdf_points(p, *pk).reshape(n)
