"""Generate the FP64 fixture of the full-size precision check (the seed-3 stenosed artery at 0.05 mm).

An FP64 run of the step at this size takes about 1.5 hours on 8 host cores, too long for a test, so it is made once
and its results are kept as a fixture, `precision_artery_dx0.05.npz`. The fixture's lattice must be the one the GPU
builds: the GPU voxeliser and the NumPy one agree to float32 rounding, which moves a couple of wall voxels at this
size, so the field is taken from the GPU near the wall. Two steps:

    # on a machine with the GPU: the GPU's signed distance within 0.2 mm of the wall, and its lattice's hashes
    python tests/golden/make_precision_golden.py band band.npz
    # on any host (no GPU needed): the NumPy field elsewhere, the lattice (bit-exact builder restatement), the
    # FP64 run of two 8000-step beats, and the fixture
    python tests/golden/make_precision_golden.py fp64 band.npz [--phi-cache phi.npy]

The fixture holds the lattice's hashes (nbr, q), the node count, the FP64 velocity at every 16th node (seeded
sample), the pressure drop (mean pressure on the inlet cells minus the mean on the parent's outlet cells), and the
wall shear stress of the FP64 field at every 16th wall point of `wss.lattice_wall`, with the fit of `wss.weights`
and mu = 1 (the same as the test evaluates).
"""
import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "precision_artery_dx0.05.npz")
SEED, DX, TAU, PERIOD, BEATS = 3, 0.05, 0.52, 8000, 2
SPEC = {"seed": SEED, "stenosis": 0.7, "pressure": 95.0}
BAND = 0.2           # mm: the GPU field is kept where |phi| < BAND
NODE_STRIDE = 16     # one node in 16 (seeded sample) for the velocity comparison
WALL_STRIDE = 16     # every 16th wall point for the shear comparison


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def sample_nodes(n):
    """The seeded node sample of the fixture."""
    rng = np.random.default_rng(12345)
    return np.sort(rng.choice(n, size=n // NODE_STRIDE, replace=False)).astype(np.int64)


def shear_host(u, normals, idx, c, scale=1e3):
    """tau_v = scale * sum_j c_vj (u_j - (u_j . n_v) n_v), FP64 (the formula of cs_wss_shear)."""
    uj = u[idx].astype(float)                                  # (V, K, 3)
    n = normals.astype(float)[:, None, :]
    ut = uj - (uj * n).sum(-1, keepdims=True) * n
    return scale * (c.astype(float)[..., None] * ut).sum(1)


def cmd_band(path):
    import torch

    from cerebrosim_b200 import vessel, workloads
    g = workloads.stenosed_vessel(SEED)
    phi, origin = vessel.sdf_grid(g, DX)
    lat = workloads.lattice(g, DX)
    flat = np.flatnonzero(np.abs(phi.reshape(-1)) < BAND).astype(np.int64)
    np.savez_compressed(path, shape=np.array(phi.shape), origin=origin, idx=flat, val=phi.reshape(-1)[flat],
                        nbr_sha=sha(lat["nbr"]), q_sha=sha(lat["q"]), n=lat["nbr"].shape[1])
    print(f"band: {len(flat)} voxels of {phi.size}; lattice {lat['nbr'].shape[1]} nodes, counts {lat['counts']}; "
          f"GPU {torch.cuda.get_device_name()}")


def cmd_fp64(band_path, phi_cache=None):
    from cerebrosim_b200 import lbm, vessel, workloads, wss
    from oracle import lattice_ref as L
    from oracle import sdf_ref
    from oracle.step_ref import OracleSolver
    band = np.load(band_path)
    g = workloads.stenosed_vessel(SEED)
    lo, hi = vessel.bounds(g)
    if phi_cache and os.path.exists(phi_cache):
        phi = np.load(phi_cache)
    else:
        t = time.time()
        phi = sdf_ref.sdf_grid(vessel.packed(g).arrays(), lo, hi, DX)
        print(f"NumPy field {phi.shape} in {time.time() - t:.0f} s", flush=True)
        if phi_cache:
            np.save(phi_cache, phi)
    assert tuple(phi.shape) == tuple(band["shape"]), (phi.shape, band["shape"])
    flat = phi.reshape(-1).copy()
    far = np.ones(flat.size, bool)
    far[band["idx"]] = False
    # outside the band both fields are at least BAND from zero: the overlay changes no sign there
    assert np.all(np.abs(flat[far]) >= 0.5 * BAND)
    flat[band["idx"]] = band["val"]
    phi = flat.reshape(phi.shape)
    lat = L.build_lattice(phi, np.asarray(lo, float), DX, openings=workloads.openings(g))
    assert sha(lat["nbr"]) == str(band["nbr_sha"]) and sha(lat["q"]) == str(band["q_sha"]), "lattice differs from GPU"
    N = lat["nbr"].shape[1]
    print(f"lattice {N} nodes, counts {lat['counts']} (hashes equal the GPU's)", flush=True)
    ref = OracleSolver(lat, (TAU - 0.5) / 3.0, model="regularised", dtype=np.float64)
    workloads.configure(ref, SPEC, lat, period=PERIOD)
    t = time.time()
    for b in range(BEATS * 8):
        ref.run(PERIOD // 8)
        print(f"  {(b + 1) * PERIOD // 8} steps, {time.time() - t:.0f} s", flush=True)
    assert ref.ok()
    p, u = ref.fields()
    p, u = np.asarray(p, float), np.asarray(u, float)
    inlet = (lat["nbr"] == lbm.INLET).any(0)
    outlet = (lat["nbr"] == lbm.OUTLET0).any(0)
    dp = float(p[inlet].mean() - p[outlet].mean())
    nodes = sample_nodes(N)
    verts, normals, cells, depth = wss.lattice_wall(lat, phi, stride=WALL_STRIDE)
    idx, c, _, _ = wss.weights(verts, normals, cells * 1.0, depth)
    tau = shear_host(u.astype(np.float32), normals, idx, c)
    np.savez_compressed(OUT, nbr_sha=str(band["nbr_sha"]), q_sha=str(band["q_sha"]), n=N, steps=BEATS * PERIOD,
                        nodes=nodes, u=u[nodes].astype(np.float32), dp=dp, tau=tau.astype(np.float32),
                        p_mean=float(p.mean()))
    print(f"wrote {OUT}: dp {dp:.6e}, {len(nodes)} nodes, {len(tau)} wall points")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["band", "fp64"])
    ap.add_argument("band")
    ap.add_argument("--phi-cache")
    a = ap.parse_args()
    cmd_band(a.band) if a.what == "band" else cmd_fp64(a.band, a.phi_cache)
