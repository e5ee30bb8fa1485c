"""Vessel signed distance on the GPU, the voxeliser that feeds `lbm.build_lattice` (vessel.py:178-245).

A vessel is the reference's geometry dict (`vessel.build(case)`: {"branches": {name: {"C": (P, 3) centreline mm,
"R": (P,) radii, "R0": unclotted radii, "caps": {"start": (centre, normal) | None, "end": ...}}}}) or the packed
arrays `packed(g)` makes of it. `sdf_grid` evaluates the field with the library's k_sdf kernel and keeps it on the
device, so that `artery_lattice` goes from centrelines to the lattice tables without the grid crossing PCIe.
"""
import ctypes

import numpy as np
import torch

from . import _lib, lbm
from ._lib import check

JUNCTION_BLEND = 0.6     # mm, smooth-union blend radius at the junction (vessel.py:36)


class Packed:
    """Centrelines packed for the kernel (vessel.py:210-221): pts (n_pts, 3), rad (n_pts,), per branch start / count,
    per branch end (start, end) cap_p / cap_n (2 nbranch, 3) and cap_r (2 nbranch,) (0 = closed end)."""

    def __init__(self, names, pts, rad, start, count, cap_p, cap_n, cap_r, blend=JUNCTION_BLEND):
        self.names = list(names)
        self.pts = np.ascontiguousarray(np.asarray(pts, np.float64).reshape(-1, 3))
        self.rad = np.ascontiguousarray(np.asarray(rad, np.float64).reshape(-1))
        self.start = np.asarray(start, np.int32).reshape(-1)
        self.count = np.asarray(count, np.int32).reshape(-1)
        nb = len(self.start)
        self.cap_p = np.asarray(cap_p, np.float64).reshape(2 * nb, 3) if nb else np.zeros((0, 3))
        self.cap_n = np.asarray(cap_n, np.float64).reshape(2 * nb, 3) if nb else np.zeros((0, 3))
        self.cap_r = np.asarray(cap_r, np.float64).reshape(2 * nb) if nb else np.zeros(0)
        self.blend = float(blend)
        if len(self.count) != nb or len(self.rad) != len(self.pts):
            raise ValueError("packed vessel: start/count or pts/rad lengths differ")
        if nb and ((self.count < 1).any() or (self.start < 0).any()
                   or (self.start.astype(np.int64) + self.count > len(self.pts)).any()):
            raise ValueError("packed vessel: a branch runs outside pts")

    def arrays(self):
        return (self.pts, self.rad, self.start, self.count, self.cap_p, self.cap_n, self.cap_r, self.blend)


def packed(g, blend=JUNCTION_BLEND):
    """vessel.py:210-221: branches back to back, a cap per branch end (radius 0 where the end is closed)."""
    names = list(g["branches"])
    pts, rad, start, count, cp, cn, cr = [], [], [], [], [], [], []
    k = 0
    for name in names:
        b = g["branches"][name]
        C, R = np.asarray(b["C"], float), np.asarray(b["R"], float)
        start.append(k)
        count.append(len(C))
        k += len(C)
        pts.append(C)
        rad.append(R)
        for key, r in (("start", R[0]), ("end", R[-1])):
            cap = b["caps"][key]
            cp.append(np.asarray(cap[0], float) if cap else np.zeros(3))
            cn.append(np.asarray(cap[1], float) if cap else np.zeros(3))
            cr.append(float(r) if cap else 0.0)
    return Packed(names, np.vstack(pts), np.concatenate(rad), start, count, np.array(cp), np.array(cn),
                  np.array(cr), blend)


def bounds(g, margin=0.5):
    """vessel.py:224-227: the centrelines' box grown by the largest unclotted radius and a margin."""
    allp = np.vstack([np.asarray(b["C"], float) for b in g["branches"].values()])
    rmax = max(float(np.max(b["R0"])) for b in g["branches"].values())
    return allp.min(0) - rmax - margin, allp.max(0) + rmax + margin


def grid_shape(lo, hi, dx):
    """vessel.py:235: voxels along each axis of the box [lo, hi] at spacing dx."""
    return tuple(int(x) for x in np.ceil((np.asarray(hi, float) - np.asarray(lo, float)) / dx).astype(int) + 1)


def sdf_device(pk, lo, hi, dx, device=None):
    """The field of the packed vessel `pk` on the voxel centres lo + (i, j, k) dx, as a float32 CUDA tensor
    (nx, ny, nz). The kernel runs on the current stream of `device`."""
    lib = _lib.load()
    dev = lbm._device(device)
    n = grid_shape(lo, hi, dx)
    if min(n) <= 0:
        raise ValueError(f"empty grid {n}")
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev)
        up = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev)
              for k, v in (("pts", pk.pts.astype(np.float32)), ("rad", pk.rad.astype(np.float32)),
                           ("start", pk.start), ("count", pk.count), ("cap_p", pk.cap_p.astype(np.float32)),
                           ("cap_n", pk.cap_n.astype(np.float32)), ("cap_r", pk.cap_r.astype(np.float32)))}
        out = torch.empty(n, dtype=torch.float32, device=dev)
        org = (ctypes.c_float * 3)(*np.asarray(lo, float).astype(np.float32).tolist())

        def p(t):
            return ctypes.c_void_p(t.data_ptr() if t.numel() else 0)
        check(lib.cs_sdf_vessel(p(up["pts"]), p(up["rad"]), p(up["start"]), p(up["count"]), len(pk.start),
                                p(up["cap_p"]), p(up["cap_n"]), p(up["cap_r"]), float(pk.blend), org, float(dx),
                                n[0], n[1], n[2], p(out), ctypes.c_void_p(stream.cuda_stream)))
        stream.synchronize()    # the uploads are freed on return
    return out


def sdf_grid(g, dx, lo=None, hi=None, device=None, host=True):
    """vessel.py:230-245: signed distance (mm, negative inside) on voxel centres origin + (i, j, k) dx ->
    (array (nx, ny, nz), origin). `g` is a geometry dict or a `Packed`; host=False returns the CUDA tensor."""
    pk = g if isinstance(g, Packed) else packed(g)
    if lo is None:
        if isinstance(g, Packed):
            raise ValueError("a packed vessel needs explicit bounds lo, hi")
        lo, hi = bounds(g)
    out = sdf_device(pk, lo, hi, dx, device)
    return (out.cpu().numpy() if host else out), np.asarray(lo, float)


def openings_of(g):
    """validate.py:297-305: an inlet at every capped branch start, an outlet at every capped end, inlets first.
    A cap given as (centre, normal, "closed") cuts the vessel flat like the others but is a wall, not an opening
    (the faces of a clot that splits a vessel)."""
    ops = []
    for name, b in g["branches"].items():
        for key, kind in (("start", "inlet"), ("end", "outlet")):
            cap = b["caps"][key]
            if cap is not None and not (len(cap) > 2 and cap[2] == "closed"):
                r = b["R"][0] if key == "start" else b["R"][-1]
                ops.append({"kind": kind, "centre": np.asarray(cap[0], float), "normal": np.asarray(cap[1], float),
                            "radius": float(r), "branch": name})
    ops.sort(key=lambda o: o["kind"] != "inlet")
    return ops


def artery_lattice(g, dx_mm, openings=None, lo=None, hi=None, device=None, host=True):
    """validate.py:294-308: the vessel's lattice at dx_mm, field and tables built on the device.
    `g` is a geometry dict, or a `Packed` with explicit `openings`, `lo` and `hi`; host=False: host tables copied
    only when read (lbm.Lattice)."""
    if isinstance(g, Packed):
        if openings is None or lo is None:
            raise ValueError("a packed vessel needs its openings and bounds")
    else:
        openings = openings_of(g) if openings is None else openings
    phi, origin = sdf_grid(g, dx_mm, lo, hi, device=device, host=False)
    ops = sorted(openings, key=lambda o: o["kind"] != "inlet")
    lat = lbm.build_lattice(phi, origin, dx_mm, openings=ops, device=phi.device, host=host)
    del phi
    lat["openings"] = ops
    return lat
