"""Golden vectors for the wall-shear-stress method, from the reference's own wss.py.

    python tests/golden/make_wss_golden.py /path/to/CerebroSim

The reference's method check (`wss.py --test`, wss.py:61-84) fits the shear on cylinders of radius 0.4 - 2.0 mm
sampled on a 0.1 mm grid with a Poiseuille profile (power 2) and a blunt one (power 4). This script builds the
same inputs (`pipe_case`, with the same seeded draws in the same order), runs the reference's `weights` and `shear`
(wss.py:35-57) on them and stores, per case, the per-vertex shear vectors, the quadratic-fit flags, and for the
first cases the fit coefficients and neighbour indices. tests/test_wss.py regenerates the inputs with `pipe_case`
and compares the package's method with these outputs.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [(r, p) for p in (2, 4) for r in (0.4, 0.65, 1.0, 1.5, 2.0)]
H = 0.1
U_MAX = 0.5


def pipe_cases(seed=0):
    """The cylinders of the reference's method check, in its order, from one seeded generator: per case (R, power,
    cells, depth, U, verts, normals)."""
    rng = np.random.default_rng(seed)
    out = []
    for R, pw in CASES:
        g = np.arange(-R - H, R + H + 1e-9, H)
        x, y, z = np.meshgrid(g + rng.uniform(0, H), g + rng.uniform(0, H), np.arange(0, 3, H), indexing="ij")
        r = np.hypot(x, y)
        m = r < R
        cells = np.column_stack([x[m], y[m], z[m]])
        depth = R - r[m]
        U = np.zeros_like(cells)
        U[:, 2] = U_MAX * (1 - (r[m] / R) ** pw)
        th = rng.uniform(0, 2 * np.pi, 400)
        verts = np.column_stack([R * np.cos(th), R * np.sin(th), rng.uniform(1, 2, 400)])
        normals = -np.column_stack([np.cos(th), np.sin(th), np.zeros_like(th)])
        out.append((R, pw, cells, depth, U, verts, normals))
    return out


def main(ref):
    sys.path.insert(0, ref)
    import wss as W
    arrays, meta = {}, {"mu_pa_s": float(W.MU), "K": int(W.K), "d_min": float(W.D_MIN), "d_max": float(W.D_MAX),
                        "sigma": float(W.SIGMA), "cases": []}
    for k, (R, pw, cells, depth, U, verts, normals) in enumerate(pipe_cases()):
        idx, c, quad, any_ = W.weights(verts, normals, cells, depth)
        tau = W.shear(U, normals, idx, c)
        arrays[f"{k}/tau"] = tau
        arrays[f"{k}/quad"] = quad
        arrays[f"{k}/any"] = any_
        if k < 2:
            arrays[f"{k}/idx"] = idx.astype(np.int32)
            arrays[f"{k}/c"] = c
        mag = np.linalg.norm(tau, axis=1)
        exact = pw * W.MU * U_MAX / (R * 1e-3)
        meta["cases"].append({"R": R, "power": pw, "exact_pa": exact, "mean_pa": float(mag.mean()),
                              "quad_pct": float(100 * quad.mean())})
    np.savez_compressed(os.path.join(HERE, "wss.npz"), **arrays)
    json.dump(meta, open(os.path.join(HERE, "wss.json"), "w"), indent=1)
    for c in meta["cases"]:
        print(c)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CEREBROSIM_REF", "."))
