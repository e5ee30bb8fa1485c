"""Storage precision against an FP64 run of the same scheme: velocity, pressure drop and wall shear stress.

The generated stenosed artery (seed 3: 70 % stenosis, side branch, Fourier inflow of period 8000 steps, tau 0.52)
at a coarse voxel size runs two beats with FP32, FP16-shifted and BF16-shifted populations on the GPU and in FP64
on the CPU oracle (oracle/lbm_ref.cpp, the same scheme in double). Compared at the end of the second beat:
- velocity: relative L2 over all nodes;
- pressure drop: mean pressure on the inlet cells minus the mean on the parent's outlet cells, relative error;
- wall shear stress: at the wall points of the lattice's wall links, by the weighted near-wall fit (wss.py:35-57;
  the same fit coefficients for every run), relative L2 of the shear vectors and relative error of the mean
  magnitude.
The voxel size and beats can be raised with CS_PRECISION_DX (mm) and CS_PRECISION_BEATS; the bounds below hold at
the default 0.2 mm. At finer voxels the flow per cell is slower relative to the stored deviations and BF16's 8-bit
mantissa falls behind (see the recorded study); FP16 holds velocity and WSS within 1 %.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from cerebrosim_b200 import lbm, vessel, workloads, wss  # noqa: E402
from oracle.step_ref import OracleSolver  # noqa: E402

DX = float(os.environ.get("CS_PRECISION_DX", "0.2"))
BEATS = int(os.environ.get("CS_PRECISION_BEATS", "2"))
PERIOD = 8000
TAU = 0.52
# relative-error limits per storage: velocity and WSS; the pressure drop (a difference of two small means, so the
# 16-bit rounding of the density shows in it more) is stated beside them with a looser bound
LIMITS = {"f32": 1e-3, "f16": 1e-2, "bf16": 5e-2}
DP_LIMITS = {"f32": 1e-3, "f16": 1e-1, "bf16": 1e-1}


def metrics(p, u, ref_p, ref_u, inlet, outlet, shear, tau_ref):
    e_u = float(np.linalg.norm(u - ref_u) / np.linalg.norm(ref_u))
    dp = float(p[inlet].mean() - p[outlet].mean())
    dp_ref = float(ref_p[inlet].mean() - ref_p[outlet].mean())
    tau = shear(u.astype(np.float32)).cpu().numpy().astype(float)
    e_tau = float(np.linalg.norm(tau - tau_ref) / np.linalg.norm(tau_ref))
    m, m_ref = np.linalg.norm(tau, axis=1).mean(), np.linalg.norm(tau_ref, axis=1).mean()
    return {"velocity_rel_l2": e_u, "pressure_drop_rel": abs(dp - dp_ref) / abs(dp_ref), "wss_rel_l2": e_tau,
            "wss_mean_rel": float(abs(m - m_ref) / m_ref), "dp": dp, "dp_fp64": dp_ref}


def test_storage_error_vs_fp64_oracle():
    spec = {"seed": 3, "stenosis": 0.7, "pressure": 95.0}
    g = workloads.stenosed_vessel(3)
    lat = workloads.lattice(g, DX)
    phi, _ = vessel.sdf_grid(g, DX)
    steps = BEATS * PERIOD
    # FP64 reference run of the same scheme on the host
    ref = OracleSolver(lat, (TAU - 0.5) / 3.0, model="regularised", dtype=np.float64)
    workloads.configure(ref, spec, lat, period=PERIOD)
    ref.run(steps)
    assert ref.ok()
    ref_p, ref_u = ref.fields()
    ref_p, ref_u = ref_p.astype(float), ref_u.astype(float)
    inlet = (lat["nbr"] == lbm.INLET).any(0)
    outlet = (lat["nbr"] == lbm.OUTLET0).any(0)
    verts, normals, cells, depth = wss.lattice_wall(lat, phi)
    idx, c, quad, any_ = wss.weights(verts, normals, cells * 1.0, depth)
    shear = wss.Shear(normals, idx, c, len(cells), mu=1.0)
    tau_ref = shear(ref_u.astype(np.float32)).cpu().numpy().astype(float)
    report = {"dx_mm": DX, "nodes": int(lat["nbr"].shape[1]), "steps": steps, "wall_points": int(len(verts))}
    for st in ("f32", "f16", "bf16"):
        s = workloads.make_solver(spec, lat, tau=TAU, period=PERIOD, storage=st)
        s.run(steps, chunk=1000)
        assert s.ok()
        p, u = s.fields()
        report[st] = metrics(p.astype(float), u.astype(float), ref_p, ref_u, inlet, outlet, shear, tau_ref)
    print("PRECISION", json.dumps(report))
    for st, r in report.items():
        if st not in LIMITS:
            continue
        lim = LIMITS[st]
        assert r["velocity_rel_l2"] <= lim and r["pressure_drop_rel"] <= DP_LIMITS[st], (st, r)
        assert r["wss_rel_l2"] <= lim and r["wss_mean_rel"] <= lim, (st, r)
