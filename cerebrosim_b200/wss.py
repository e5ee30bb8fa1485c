"""Wall shear stress from a solver's velocity field, by the reference's weighted near-wall fit (wss.py:35-57).

At each wall vertex (a point on the wall with its unit normal pointing into the lumen) the velocity of the nearby
lumen cells, minus its part along the normal, is fitted against the distance d to the wall as u_t(d) = a d + b d^2
(no slip at the wall; weighted towards cells straight below the vertex), and tau = mu a. The fit is linear in the
velocities, so it reduces to one coefficient per (vertex, neighbour cell): `weights` finds them once per geometry on
the host (a k-d tree query and 2 x 2 least squares per vertex); `Shear` applies them to any number of velocity
fields on the GPU (`cs_wss_shear`).

The constants are the reference's: 48 nearest cells within 0.8 mm, cells between 0.02 and 0.45 mm from the wall,
sideways Gaussian weight of 0.15 mm, blood viscosity 3.5 mPa s (geometry/physics.json). Lengths in mm, velocities
in m/s, stresses in Pa.

`lattice_wall(lat, phi)` gives a vertex set for a sparse lattice: the points where its wall links cross the wall
(x - q c dx), with normals from the signed distance's gradient.
"""
import ctypes

import numpy as np
import torch
from scipy.spatial import cKDTree

from . import _lib, lbm
from ._lib import check

MU = 0.0035            # Pa s (geometry/physics.json: blood viscosity)
K = 48                 # nearest lumen cells per vertex
D_MIN, D_MAX = 0.02, 0.45
SIGMA = 0.15
REACH = 0.8            # mm: farthest neighbour considered


def weights(verts, normals, cells, depth, k=K, d_min=D_MIN, d_max=D_MAX, sigma=SIGMA, reach=REACH):
    """Fit coefficients (wss.py:35-48): for each vertex its k nearest cells `idx` (V, k) and coefficients `c`
    (V, k, float32) with a = sum_j c_j u_t,j (per mm); `quad` marks vertices fitted with a d + b d^2 (enough
    weighted cells), the others use u_t = a d; `any` marks vertices with some cell in the fit."""
    verts = np.asarray(verts, float)
    normals = np.asarray(normals, float)
    cells = np.asarray(cells, float)
    depth = np.asarray(depth, float)
    dist, idx = cKDTree(cells).query(verts, k=k, distance_upper_bound=reach)
    found = np.isfinite(dist)
    idx = np.where(found, idx, 0)
    d = depth[idx]
    rel = cells[idx] - verts[:, None, :]
    along = np.einsum("vkc,vc->vk", rel, normals)
    side = np.linalg.norm(rel - along[..., None] * normals[:, None, :], axis=-1)
    w = np.exp(-(side / sigma) ** 2) * found * (d > d_min) * (d < d_max)
    # weighted least squares of u = a d + b d^2: normal equations [s2 s3; s3 s4] [a b] = [sum w d u, sum w d^2 u]
    s2 = (w * d ** 2).sum(1)
    s3 = (w * d ** 3).sum(1)
    s4 = (w * d ** 4).sum(1)
    det = s2 * s4 - s3 ** 2
    quad = (det > 1e-12 * np.maximum(s2 * s4, 1e-30)) & ((w > 0.05).sum(1) >= 6)
    c_quad = w * (s4[:, None] * d - s3[:, None] * d ** 2) / np.where(quad, det, 1.0)[:, None]
    c_lin = w * d / np.maximum(s2, 1e-30)[:, None]
    c = np.where(quad[:, None], c_quad, c_lin)
    c[s2 <= 0] = 0.0
    return idx.astype(np.int32), c.astype(np.float32), quad, s2 > 0


class Shear:
    """Shear at fixed vertices for velocity fields of the same cells, on the GPU (cs_wss_shear)."""

    def __init__(self, normals, idx, c, n_cells, mu=MU, device=None):
        self.dev = lbm._device(device)
        self.n_cells = int(n_cells)
        self.normals = torch.as_tensor(np.ascontiguousarray(normals, np.float32)).to(self.dev)
        self.idx = torch.as_tensor(np.ascontiguousarray(idx, np.int32)).to(self.dev)
        self.c = torch.as_tensor(np.ascontiguousarray(c, np.float32)).to(self.dev)
        self.k = int(self.idx.shape[1])
        self.scale = float(mu) * 1e3           # (m/s)/mm -> 1/s, times mu

    def __call__(self, U):
        """tau (V, 3) float32 CUDA tensor (Pa) for the cells' velocity U ((n_cells, 3), m/s, host or device)."""
        U = torch.as_tensor(U, dtype=torch.float32).to(self.dev).contiguous()
        if U.shape != (self.n_cells, 3):
            raise ValueError(f"velocity of shape {tuple(U.shape)}, expected ({self.n_cells}, 3)")
        tau = torch.empty((self.idx.shape[0], 3), dtype=torch.float32, device=self.dev)
        stream = torch.cuda.current_stream(self.dev)

        def p(t):
            return ctypes.c_void_p(t.data_ptr() if t.numel() else 0)
        check(_lib.load().cs_wss_shear(p(U), self.n_cells, p(self.idx), p(self.c), p(self.normals),
                                       int(self.idx.shape[0]), self.k, self.scale, p(tau),
                                       ctypes.c_void_p(stream.cuda_stream)))
        return tau


def lattice_wall(lat, phi, origin=None, dx=None, stride=1):
    """Wall vertices of a sparse lattice (mm): where each wall link of an axis or edge direction crosses the wall,
    x_node - q c dx, one per (node, direction), every `stride`-th kept; normals (into the lumen) from the central
    differences of phi (float32 grid on the lattice's nodes, negative inside) at the nearest grid node.
    Returns (verts, normals, cells, depth): cells are the fluid nodes' positions and depth their distance to the wall
    (-phi)."""
    phi = np.asarray(phi, np.float32)
    origin = np.asarray(lat["origin"] if origin is None else origin, float)
    dx = float(lat["dx"] if dx is None else dx)
    coords = lat["coords"]
    cells = origin + coords * dx
    depth = -phi[tuple(coords.T)].astype(float)
    nbr, q = lat["nbr"], lat["q"]
    pts = []
    for i in range(1, 19):
        nodes = np.flatnonzero(nbr[i] == lbm.WALL)
        if len(nodes):
            pts.append(cells[nodes] - q[i, nodes, None].astype(float) * lbm.C[i][None, :] * dx)
    verts = np.vstack(pts)[::max(1, int(stride))]
    g = np.stack(np.gradient(phi.astype(float), dx), axis=-1)        # d phi / d x, per grid node
    ijk = np.clip(np.rint((verts - origin) / dx).astype(int), 0, np.array(phi.shape) - 1)
    n = -g[tuple(ijk.T)]
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-12)
    return verts, n, cells, depth
