"""Signed-distance fields of the validation and benchmark vessels (NumPy, host side).

These restate the geometry of CerebroSim's validation suite so that the same lattices can be built here:
  - `periodic_pipe(D)`        validate.py:59-66   (Poiseuille / Womersley pipes, periodic along z)
  - `open_pipe(axis, L, radius)` validate.py:125-148 (velocity inlet + pressure outlet pipes, any orientation)
  - `stenosis_radius(...)`    validate.py:226-237 (cosine narrowing)
  - `poiseuille_cylinder()`   a circular cylinder R = 10 on a 24 x 24 x 64 grid, periodic along z, axis off the
                              grid's symmetry lines by validate.py:42's offset (about 20 k fluid nodes)
Every function returns float32 SDF values, negative inside the lumen, exactly as the reference passes them to
`build_lattice` (the float64 -> float32 cast happens at lbm.py:272); tests pin them by hash against the reference.
"""
import math

import numpy as np

# pipe axes off the grid's symmetry lines; straight pipes' ends between nodes (validate.py:42)
OFFSET = np.array([0.31, 0.17, 0.5])


def periodic_pipe(D):
    """Pipe of diameter D (cells) on an (n, n, 2) grid, periodic along z. Returns (phi, r per grid node, R)."""
    R = D / 2.0
    n = int(math.ceil(D)) + 4
    centre = np.array([n / 2 - 0.5, n / 2 - 0.5]) + OFFSET[:2]
    gi, gj, _ = np.meshgrid(np.arange(n), np.arange(n), np.arange(2), indexing="ij")
    r = np.hypot(gi - centre[0], gj - centre[1])
    return (r - R).astype(np.float32), r, R


def poiseuille_cylinder(R=10.0, n=24, length=64):
    """Cylinder of radius R on an (n, n, length) grid, periodic along z. Returns (phi, r per grid node)."""
    centre = np.array([n / 2 - 0.5, n / 2 - 0.5]) + OFFSET[:2]
    gi, gj, _ = np.meshgrid(np.arange(n), np.arange(n), np.arange(length), indexing="ij")
    r = np.hypot(gi - centre[0], gj - centre[1])
    return (r - R).astype(np.float32), r


def open_pipe(axis, L, radius, pad=3):
    """Straight pipe from its start A along unit `axis`, length L cells, radius(s) along the axis.

    Returns (phi, openings, A, axis): phi float32 on the bounding grid; openings = [inlet at A facing -axis,
    outlet at A + L axis facing +axis] with the end radii; A the pipe start in grid coordinates."""
    axis = np.asarray(axis, float)
    axis = axis / np.linalg.norm(axis)
    rmax = float(max(radius(np.linspace(0, L, 400))))
    ends = np.array([np.zeros(3), axis * L])
    ext = rmax * np.sqrt(np.clip(1 - axis ** 2, 0, 1)) + pad
    lo = ends.min(0) - ext
    hi = ends.max(0) + ext
    dims = np.ceil(hi - lo).astype(int) + 1
    start = -lo + OFFSET
    g = np.stack(np.meshgrid(*[np.arange(k) for k in dims], indexing="ij"), -1).reshape(-1, 3) - start
    s = g @ axis
    rad = np.linalg.norm(g - s[:, None] * axis, axis=1)
    phi = np.maximum(np.maximum(rad - radius(s), -s), s - L).reshape(dims)
    r0, r1 = float(radius(np.array([0.0]))[0]), float(radius(np.array([L]))[0])
    openings = [{"kind": "inlet", "centre": start, "normal": -axis, "radius": r0},
                {"kind": "outlet", "centre": start + axis * L, "normal": axis, "radius": r1}]
    return phi.astype(np.float32), openings, start, axis


def axial_radial(coords, start, axis):
    """Axial and radial coordinate of lattice nodes relative to a pipe's start and axis (validate.py:145-147)."""
    p = coords - start
    s = p @ axis
    return s, np.linalg.norm(p - s[:, None] * axis, axis=1)


def stenosis_radius(D, severity=0.7, length_d=2.0, up_d=4, down_d=18):
    """Cosine narrowing of a pipe of diameter D cells (validate.py:226-237 with Ls = length_d x D).
    Returns (radius(s), total length L, narrowing start s0, narrowing length Ls)."""
    R0, Ls, s0 = D / 2, length_d * D, up_d * D

    def radius(s):
        s = np.asarray(s, float)
        x = np.clip((s - s0) / Ls, 0, 1)
        return R0 * (1 - severity * 0.5 * (1 - np.cos(2 * math.pi * x)))
    return radius, (up_d + down_d) * D + Ls, s0, Ls
