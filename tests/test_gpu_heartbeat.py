"""The heartbeat loop on the device: probes and coarse frames reduced on the GPU agree with the same quantities
computed on the host from the solver's fields; the result files have the reference's layout (simulate.py:361-380)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from cerebrosim_b200 import simulate as S, vessel, workloads as W  # noqa: E402


def artery(order="c"):
    # every open end an outlet, the parent's start pressure-driven through p_out[0] (as simulate.setup does)
    g = W.stenosed_vessel(seed=11, stenosis=0.5)
    dx = W.dx_for_nodes(30e3, W.estimated_nodes(g, 0.05), 0.05)
    lat = vessel.artery_lattice(g, dx, openings=[dict(o, kind="outlet") for o in W.openings(g)])
    P = lat["origin"] + lat["coords"] * dx
    idx, w, slot = [], [], []
    for k, o in enumerate(lat["openings"]):
        rel = P - o["centre"]
        depth = -(rel @ o["normal"]) / dx
        side = np.linalg.norm(rel + (depth * dx)[:, None] * o["normal"], axis=1) < 1.3 * o["radius"]
        m = np.flatnonzero(side & (depth >= 4) & (depth < 6))
        idx.append(m)
        slot.append(np.full(len(m), k))
        w.append(np.tile((-1.0 if k == 0 else 1.0) * o["normal"] / 2.0, (len(m), 1)))
    flux = {"idx": np.concatenate(idx), "w": np.vstack(w).astype(np.float32), "slot": np.concatenate(slot)}
    n_open = len(lat["openings"])
    s = S.ArterySolver(lat, (0.52 - 0.5) / 3, flux, [0.0] + [0.05] * (n_open - 1), 0.0, 0.01, model="regularised",
                       order=order)
    s.set_sponge(4, 0.55, kinds=("outlet",))
    s.set_outlet_pressure([0.0] * n_open)
    s.set_drive([1e-3, 5e-4, 0.0], period=200, ramp=20)
    # probes: three points along the parent's centreline
    C = g["branches"]["trunk"]["C"]
    pidx, pslot = [], []
    for k, f in enumerate((0.2, 0.5, 0.8)):
        pt = C[int(f * (len(C) - 1))]
        m = np.flatnonzero(np.linalg.norm(P - pt, axis=1) < 0.6)
        pidx.append(m)
        pslot.append(np.full(len(m), k))
    return s, lat, dx, np.concatenate(pidx), np.concatenate(pslot)


@pytest.mark.parametrize("order", ["c", "axis"])
def test_heartbeat_loop(tmp_path, order):
    s, lat, dx, pidx, pslot = artery(order)
    probes = S.Probes(s, pidx, pslot, 3)
    cmap = S.CoarseMap(s, lat, dx, target_mm=2 * dx)
    beats_seen = []
    series, frames = S.run_beats(s, 200, 2, 20, probes=probes, cmap=cmap, frames=5,
                                 on_beat=lambda s_, b, ser: beats_seen.append(b))
    assert beats_seen == [1, 2] and s.ok()
    assert series["step"].tolist() == list(range(20, 401, 20))
    assert series["Q"].shape == (20, s.n_open) and series["p_open"].shape == (20, s.n_open)
    assert series["p_probe"].shape == (20, 3) and np.isfinite(series["p_probe"]).all()
    assert frames["t_step"].tolist() == [40, 80, 120, 160, 200] and frames["p"].shape == (5, cmap.n_bins)
    # device reductions against the host, on the final state
    p, u = s.fields()
    pp, um = probes.sample()
    ref = np.array([p[pidx[pslot == k]].astype(float).mean() for k in range(3)])
    np.testing.assert_allclose(pp, ref, rtol=1e-6, atol=1e-9)
    assert um == pytest.approx(float(np.linalg.norm(u[pidx], axis=1).max()), rel=1e-6)
    cp, cu = cmap.frame()
    np.testing.assert_allclose(cp, np.bincount(cmap.inv, weights=p.astype(float)) / cmap.cnt, rtol=1e-5, atol=1e-9)
    np.testing.assert_allclose(cu[:, 2], np.bincount(cmap.inv, weights=u[:, 2].astype(float)) / cmap.cnt, rtol=1e-5,
                               atol=1e-9)
    np.testing.assert_array_equal(frames["p"][-1], cp)       # the last frame is the final state
    # result files in the reference's layout
    d = str(tmp_path / "run")
    S.save(d, {"case": "test", "steps_per_beat": 200}, series,
           {"t": frames["t_step"], "p_mmhg": frames["p"], "u_m_s": frames["u"]}, cmap=cmap, lat=lat,
           wall_mm=np.zeros(s.N), dx_mm=dx)
    ser = np.load(os.path.join(d, "series.npz"))
    assert set(ser.files) == {"step", "Q", "p_open", "p_probe", "umax"}
    fl = np.load(os.path.join(d, "fields.npz"))
    assert set(fl.files) == {"coords", "origin", "dx_mm", "wall_mm", "t", "p_mmhg", "u_m_s"}
    assert fl["p_mmhg"].dtype == np.float16 and fl["u_m_s"].shape == (5, cmap.n_bins, 3)
    assert json.load(open(os.path.join(d, "meta.json")))["steps_per_beat"] == 200
