"""The artery solver of CerebroSim's simulate.py on the B200 library: `ArterySolver` (simulate.py:93-114).

`ArterySolver(lat, nu_lu, flux, R_lu, pref_lu, alpha, **kw)` keeps the reference constructor. Per step, after the
collision, the slab flux Q_k = sum u . w over each open end's flux cells is reduced and the outlet pressures are
relaxed towards R_k Q_k - pref (simulate.py:65-82). Here the flux is reduced inside the bulk kernel by the blocks
that hold slab cells and k_bc adds the blocks' partial sums, both in FP64 and in a fixed order, so a run is
bit-reproducible; Qlast / p_out64 are double, p_out (read by the outlet links) is the float32 image of p_out64, and
Qacc (the reference's accumulator, zero between steps) is kept as a zero array.

Device state is exposed through `DeviceArray`, which keeps the reference's `.numpy()` / `.zero_()` / `.assign()`
access pattern on top of a torch tensor.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check
from .lbm import Solver, ctypes_void


class DeviceArray:
    """A torch CUDA tensor with the array methods simulate.py uses on the reference's device arrays."""

    def __init__(self, tensor, stream=None):
        self.tensor = tensor
        self._stream = stream

    def numpy(self):
        if self._stream is not None:
            self._stream.synchronize()
        return self.tensor.cpu().numpy()

    def zero_(self):
        self.tensor.zero_()

    def assign(self, values):
        self.tensor.copy_(torch.as_tensor(np.asarray(values)).to(self.tensor.device, self.tensor.dtype))

    def __len__(self):
        return len(self.tensor)

    @property
    def shape(self):
        return tuple(self.tensor.shape)


class ArterySolver(Solver):
    """lbm.Solver + resistance outlets and flow measurement inside each step (simulate.py:93-114).

    flux: {"idx": (M,) node of each slab cell, "w": (M, 3) weight vector, "slot": (M,) open end}; R_lu: resistance
    per open end (R_lu[0] is unused: p_out[0] follows the drive); pref_lu: reference pressure; alpha: relaxation."""

    MAX_OPEN = 8

    def __init__(self, lat, nu_lu, flux, R_lu, pref_lu, alpha, **kw):
        super().__init__(lat, nu_lu, **kw)
        idx = np.asarray(flux["idx"], np.int64).reshape(-1)
        w = np.asarray(flux["w"], np.float32).reshape(-1, 3)
        slot = np.asarray(flux["slot"], np.int64).reshape(-1)
        self.n_open = n_open = len(R_lu)
        if not (len(idx) == len(w) == len(slot)):
            raise ValueError("flux idx / w / slot lengths differ")
        if n_open < 1 or n_open > self.MAX_OPEN or n_open > len(self.p_out):
            raise ValueError(f"{n_open} open ends: 1..{self.MAX_OPEN} and at most the {len(self.p_out)} outlet "
                             "pressures of the lattice")
        if len(idx) and (idx.min() < 0 or idx.max() >= self.N):
            raise ValueError("flux idx outside the lattice")
        if len(slot) and (slot.min() < 0 or slot.max() >= n_open):
            raise ValueError("flux slot outside the open ends")
        if self.inv is not None:                          # the lattice's node ids -> the internal numbering
            idx = self.inv.cpu().numpy()[idx]
        order = np.argsort(idx, kind="stable")            # the fused reduction reads entries block by block
        dev = self.dev
        with torch.cuda.device(dev), torch.cuda.stream(self.stream):
            self.f_idx = torch.as_tensor(idx[order].astype(np.int32)).to(dev)
            self.f_w = torch.as_tensor(np.ascontiguousarray(w[order])).to(dev)
            self.f_slot = torch.as_tensor(slot[order].astype(np.int32)).to(dev)
            self._qacc = torch.zeros(n_open, dtype=torch.float64, device=dev)
            self._qlast = torch.zeros(n_open, dtype=torch.float64, device=dev)
            self._r = torch.as_tensor(np.asarray(R_lu, np.float32)).to(dev)
            # running sums of the open ends' pressure and flow over the current beat, and the step count
            self._beat_acc = torch.zeros(2 * self.MAX_OPEN + 1, dtype=torch.float64, device=dev)
        self.pref = float(pref_lu)
        self.alpha = float(alpha)
        self.Qacc = DeviceArray(self._qacc, self.stream)
        self.Qlast = DeviceArray(self._qlast, self.stream)
        self.R = DeviceArray(self._r, self.stream)
        self._set_flux_blocks()

    def _set_flux_blocks(self):
        """Partition the sorted flux list by bulk block (for the current block size): each block that holds flux
        entries writes its partial sums to its own row of q_part; fb_list names those blocks in ascending order."""
        nb = max(1, -(-self.N // self.block))
        idx = self.f_idx.cpu().numpy()
        fb = np.unique(idx // self.block).astype(np.int32) if len(idx) else np.zeros(0, np.int32)
        with torch.cuda.device(self.dev), torch.cuda.stream(self.stream):
            self._flux_block = torch.empty(nb + 1, dtype=torch.int32, device=self.dev)
            check(_lib.load().cs_flux_blocks(ctypes.c_void_p(self.f_idx.data_ptr() if len(self.f_idx) else 0),
                                             len(self.f_idx), self.N, self.block,
                                             ctypes.c_void_p(self._flux_block.data_ptr()),
                                             ctypes_void(self.stream.cuda_stream)))
            self._fb_list = torch.as_tensor(fb if len(fb) else np.zeros(1, np.int32)).to(self.dev)
            self._n_fb = len(fb)
            self._q_part = torch.zeros(nb * self.MAX_OPEN, dtype=torch.float64, device=self.dev)

    def _fill_desc(self, d):
        d.n_open = self.n_open
        d.n_flux = len(self.f_idx)
        d.flux_idx = self.f_idx.data_ptr() if len(self.f_idx) else None
        d.flux_w = self.f_w.data_ptr() if len(self.f_idx) else None
        d.flux_slot = self.f_slot.data_ptr() if len(self.f_idx) else None
        d.flux_block = self._flux_block.data_ptr()
        d.q_part, d.fb_list, d.n_fb = self._q_part.data_ptr(), self._fb_list.data_ptr(), self._n_fb
        d.q_last, d.r_out = self._qlast.data_ptr(), self._r.data_ptr()
        d.pref, d.alpha = self.pref, self.alpha
        d.beat_acc = self._beat_acc.data_ptr()

    def checkpoint(self):
        """lbm.Solver.checkpoint plus the coupling's state: last flows, FP64 outlet pressures, beat sums."""
        st = super().checkpoint()
        st.update({"q_last": self._qlast.cpu().clone(), "beat_acc": self._beat_acc.cpu().clone()})
        return st

    def restore(self, st):
        super().restore(st)
        with torch.cuda.device(self.dev), torch.cuda.stream(self.stream):
            self._qlast.copy_(st["q_last"].to(self.dev))
            self._beat_acc.copy_(st["beat_acc"].to(self.dev))
        self.stream.synchronize()

    def beat_means(self, reset=True):
        """Means of the open ends' pressures p_out (lattice units) and flows Qlast over the steps since the last
        reset, accumulated on the device in FP64 by every step's k_bc -> (p (n_open,), Q (n_open,), steps). The
        reference averages its 1 ms samples of the same series over the beat (simulate.py:325-333)."""
        self.stream.synchronize()
        acc = self._beat_acc.cpu().numpy()
        n = self.n_open
        steps = int(round(acc[2 * n]))
        if reset:
            with torch.cuda.device(self.dev), torch.cuda.stream(self.stream):
                self._beat_acc.zero_()
        k = max(steps, 1)
        return acc[:n] / k, acc[n:2 * n] / k, steps


# ---------------------------------------------------------------------------------------------------------------
# heartbeat loop: probes, coarse-map frames, result files, lumped circuit
# ---------------------------------------------------------------------------------------------------------------

def _segments(idx, seg, n_seg, n_cells, inv=None):
    """Cell lists grouped by segment (stable), as device-ready (cells, start) arrays; lattice ids mapped through inv
    (the solver's internal numbering) when given."""
    idx = np.asarray(idx, np.int64).reshape(-1)
    seg = np.asarray(seg, np.int64).reshape(-1)
    if len(idx) != len(seg):
        raise ValueError("cell and segment lists differ in length")
    if len(idx) and (idx.min() < 0 or idx.max() >= n_cells or seg.min() < 0 or seg.max() >= n_seg):
        raise ValueError("cell index or segment out of range")
    if inv is not None and len(idx):
        idx = inv[idx]
    order = np.argsort(seg, kind="stable")
    start = np.concatenate([[0], np.cumsum(np.bincount(seg, minlength=n_seg))]).astype(np.int32)
    return idx[order].astype(np.int32), start


class Probes:
    """Pressure probes (simulate.k_gather, simulate.py:85-90): cells idx[j] (lattice ids) belonging to probe
    slot[j]. `sample()` -> (mean pressure per probe in lattice units, NaN for a probe without cells; largest speed
    over all probe cells), reduced on the device in FP64."""

    def __init__(self, s, idx, slot, n_probes):
        self.s = s
        self.n = int(n_probes)
        inv = s.inv.cpu().numpy() if getattr(s, "inv", None) is not None else None
        cells, start = _segments(idx, slot, self.n, s.N, inv)
        self.count = np.diff(start)
        with torch.cuda.device(s.dev):
            self.cells = torch.as_tensor(cells if len(cells) else np.zeros(1, np.int32)).to(s.dev)
            self.start = torch.as_tensor(start).to(s.dev)
            self.psum = torch.zeros(max(1, self.n), dtype=torch.float64, device=s.dev)
            self.umax = torch.zeros(max(1, self.n), dtype=torch.float32, device=s.dev)

    def sample(self):
        s = self.s
        with torch.cuda.device(s.dev), torch.cuda.stream(s.stream):
            check(_lib.load().cs_probe_gather(ctypes_void(s.rho.data_ptr()), ctypes_void(s.vel[s.cur].data_ptr()),
                                              s.N, ctypes_void(self.cells.data_ptr()),
                                              ctypes_void(self.start.data_ptr()), self.n,
                                              ctypes_void(self.psum.data_ptr()), ctypes_void(self.umax.data_ptr()),
                                              ctypes_void(s.stream.cuda_stream)))
        s.stream.synchronize()
        psum = self.psum.cpu().numpy()[:self.n]
        p = np.where(self.count > 0, psum / np.maximum(self.count, 1), np.nan)
        return p, float(self.umax.cpu().numpy()[:self.n].max()) if self.n else 0.0


def coarse_bins(lat, dx_mm, target_mm=0.1):
    """simulate.coarse_map (simulate.py:236-242): cells -> bins of `target_mm` (identity at that spacing, 2x2x2
    averages at half of it) -> (bin coordinates int16, bin of each cell, cells per bin, factor)."""
    f = max(1, int(round(target_mm / dx_mm)))
    key = np.asarray(lat["coords"]) // f
    uk, inv = np.unique(key, axis=0, return_inverse=True)
    inv = inv.ravel()
    return uk.astype(np.int16), inv, np.bincount(inv), f


class CoarseMap:
    """Frames of the stored fields on the coarse bins, averaged on the device: `frame()` -> (p (bins,), u (bins, 3))
    in lattice units."""

    def __init__(self, s, lat, dx_mm, target_mm=0.1):
        self.s = s
        self.uk, self.inv, self.cnt, self.f = coarse_bins(lat, dx_mm, target_mm)
        self.n_bins = len(self.uk)
        inv_int = s.inv.cpu().numpy() if getattr(s, "inv", None) is not None else None
        cells, start = _segments(np.arange(s.N), self.inv, self.n_bins, s.N, inv_int)
        with torch.cuda.device(s.dev):
            self.cells = torch.as_tensor(cells).to(s.dev)
            self.start = torch.as_tensor(start).to(s.dev)
            self.p = torch.empty(self.n_bins, dtype=torch.float32, device=s.dev)
            self.u = torch.empty((self.n_bins, 3), dtype=torch.float32, device=s.dev)

    def frame(self):
        s = self.s
        with torch.cuda.device(s.dev), torch.cuda.stream(s.stream):
            check(_lib.load().cs_bin_fields(ctypes_void(s.rho.data_ptr()), ctypes_void(s.vel[s.cur].data_ptr()), s.N,
                                            ctypes_void(self.cells.data_ptr()), ctypes_void(self.start.data_ptr()),
                                            self.n_bins, ctypes_void(self.p.data_ptr()), ctypes_void(self.u.data_ptr()),
                                            ctypes_void(s.stream.cuda_stream)))
        s.stream.synchronize()
        return self.p.cpu().numpy(), self.u.cpu().numpy()


def run_beats(s, steps_per_beat, beats, every, probes=None, cmap=None, frames=40, on_beat=None):
    """The measurement loop of simulate.run (simulate.py:300-360) on the device: `every` steps at a time (CUDA
    graphs), then a sample — time step, flows Qlast and open-end pressures p_out (an ArterySolver), probe pressures
    and the largest probe speed; `frames` snapshots of the coarse fields evenly over the last beat; `on_beat(s, beat,
    series)` after each beat (where the reference calibrates its inlet). Lattice units throughout."""
    if steps_per_beat % every:
        raise ValueError(f"{steps_per_beat} steps per beat is not a multiple of {every}")
    frame_every = steps_per_beat // max(1, frames)
    if frames and frame_every % every:
        raise ValueError(f"{frame_every} steps per frame is not a multiple of {every}")
    series = {"step": [], "Q": [], "p_open": [], "p_probe": [], "umax": []}
    out = {"t_step": [], "p": [], "u": []}
    total = beats * steps_per_beat
    coupled = hasattr(s, "Qlast")
    while s.steps < total:
        s.run(every, chunk=every)
        series["step"].append(s.steps)
        if coupled:
            series["Q"].append(s.Qlast.numpy().copy())
            series["p_open"].append(s.p_out.cpu().numpy()[:s.n_open].astype(float))
        if probes is not None:
            p, um = probes.sample()
            series["p_probe"].append(p)
            series["umax"].append(um)
        if s.steps % steps_per_beat == 0:
            if not s.ok():
                raise RuntimeError(f"solver diverged at step {s.steps}")
            if on_beat is not None:
                on_beat(s, s.steps // steps_per_beat, series)
        last = s.steps - (beats - 1) * steps_per_beat
        if cmap is not None and frames and last > 0 and last % frame_every == 0:
            p, u = cmap.frame()
            out["t_step"].append(last)
            out["p"].append(p)
            out["u"].append(u)
    return {k: np.array(v) for k, v in series.items()}, {k: np.array(v) for k, v in out.items()}


def fourier(y, nh=10):
    """simulate.fourier (simulate.py:123-130): samples over one period -> [a0, a1, b1, a2, b2, ...] of
    a0 + sum a_k cos(2 pi k t) + b_k sin(2 pi k t)."""
    F = np.fft.rfft(np.asarray(y, float)) / len(y)
    c = [F[0].real]
    for k in range(1, nh + 1):
        c += [2 * F[k].real, -2 * F[k].imag]
    return np.array(c)


def from_fourier(c, t):
    """simulate.from_fourier (simulate.py:133-137): the series at times t (in periods)."""
    y = np.full_like(np.asarray(t, float), c[0], dtype=float)
    for k in range(1, (len(c) - 1) // 2 + 1):
        y += c[2 * k - 1] * np.cos(2 * np.pi * k * t) + c[2 * k] * np.sin(2 * np.pi * k * t)
    return y


MMHG = 133.322


def circuit(R_seg, shape, q_in_ml_min, q_target_ml_min, p_out_mmhg, nh=10):
    """simulate.circuit (simulate.py:138-148), SI: the outlets' resistances that split the mean inflow q_in as
    (q_target, rest) at the mean outlet pressure p_out, and the Fourier coefficients (Pa, absolute) of the inlet
    pressure that draws the inflow waveform q_in * shape (one period of samples, mean 1) through the segment
    resistance R_seg plus the outlets in parallel."""
    q_in = q_in_ml_min * 1e-6 / 60
    q_t = q_target_ml_min * 1e-6 / 60
    p_out = p_out_mmhg * MMHG
    R_t, R_o = p_out / q_t, p_out / (q_in - q_t)
    R_eq = p_out / q_in
    coef = fourier((R_eq + R_seg) * q_in * np.asarray(shape, float), nh)
    return {"R_out": [0.0, R_t, R_o], "R_seg": float(R_seg), "P_in_coef": coef.tolist(), "R_eq": R_eq}


def recalibrate(cal, p_in_mean_pa, q_in_mean_ml_min, shape, q_in_ml_min, q_target_ml_min, p_out_mmhg):
    """The calibrate branch of simulate.run (simulate.py:330-337): the segment resistance implied by a beat's mean
    inlet pressure and inflow, and the circuit rebuilt with it."""
    R_tot = p_in_mean_pa / (q_in_mean_ml_min * 1e-6 / 60)
    return circuit(max(R_tot - cal["R_eq"], 0.0), shape, q_in_ml_min, q_target_ml_min, p_out_mmhg)


def flux_slabs(lat, ends, dx_mm, slab_mm=(2.5, 3.5), reach=1.3):
    """simulate.py:181-192: the cells of each open end's flow slab — depth slab_mm inside the end (mm along the
    inward normal), within `reach` radii of its axis — with weight sign * normal / thickness (inflow positive at end
    0, outflow positive at the others) -> the ArterySolver's flux dict."""
    P = np.asarray(lat["origin"], float) + np.asarray(lat["coords"], float) * dx_mm
    thick = (slab_mm[1] - slab_mm[0]) / dx_mm
    idx, w, slot = [], [], []
    for k, e in enumerate(ends):
        c, nrm = np.asarray(e["centre"], float), np.asarray(e["normal"], float)
        rel = P - c
        depth = -(rel @ nrm)
        side = np.linalg.norm(rel + depth[:, None] * nrm, axis=1) < reach * e["radius"]
        m = np.flatnonzero(side & (depth >= slab_mm[0]) & (depth < slab_mm[1]))
        sign = -1.0 if k == 0 else 1.0
        idx.append(m)
        slot.append(np.full(len(m), k))
        w.append(np.tile(sign * nrm / thick, (len(m), 1)))
    return {"idx": np.concatenate(idx).astype(np.int32), "w": np.vstack(w).astype(np.float32),
            "slot": np.concatenate(slot).astype(np.int32)}


class Calibration:
    """The inlet-pressure calibration of simulate.run (simulate.py:265-289, 325-337) over an ArterySolver whose open
    end 0 is a pressure inlet (p_out[0] follows the drive) and whose other ends drain through resistances.

    The lumped circuit (`circuit`) gives the outlet resistances and the inlet pressure waveform that draws the mean
    inflow q_in (with the waveform `shape`, one period of samples with mean 1) through the segment resistance R_seg
    plus the outlets. After each beat `on_beat` takes the beat's mean inlet pressure and inflow (the solver's
    device-side beat means), finds the segment resistance they imply, rebuilds the circuit and sets the new drive,
    which applies from the next beat's first step. SI units inside the circuit; the solver's lattice units through
    `units` (lbm.Units) as q_si = dx^3 / dt and p_si = rho c^2."""

    def __init__(self, units, shape, q_in_ml_min, q_target_ml_min, p_out_mmhg, steps_per_beat, ramp=0, flow=1.0,
                 R_seg=0.0, nh=10):
        self.un = units
        self.shape = np.asarray(shape, float)
        self.q_in, self.q_target, self.p_out_mmhg = float(q_in_ml_min), float(q_target_ml_min), float(p_out_mmhg)
        self.spb, self.ramp, self.flow, self.nh = int(steps_per_beat), int(ramp), float(flow), int(nh)
        self.q_si = units.dx ** 3 / units.dt
        self.p_si = units.rho * units.c ** 2
        self.pref_lu = self.p_out_mmhg * MMHG / self.p_si
        self.cal = circuit(R_seg, self.shape, self.q_in, self.q_target, self.p_out_mmhg, nh)
        self.history = []
        self.s = None

    def R_lu(self, n_open):
        """Resistance per open end in lattice units (end 0, the inlet, has none)."""
        return [r * self.q_si / self.p_si for r in self.cal["R_out"][:n_open]]

    def attach(self, s):
        """Set the solver's outlet pressures to the reference (gauge 0 at the inlet, -pref elsewhere) and its
        drive from the current circuit."""
        self.s = s
        s.set_outlet_pressure([0.0] + [-self.pref_lu] * (s.n_open - 1))
        self.drive()
        s.beat_means(reset=True)
        return s

    def drive(self):
        """simulate.py:284-289: the circuit's inlet pressure in lattice units, gauge, scaled by `flow`."""
        c = np.array(self.cal["P_in_coef"]) / self.p_si * self.flow
        c[0] -= self.pref_lu
        self.s.set_drive(c, period=self.spb, ramp=self.ramp)

    def on_beat(self, beat):
        """simulate.py:325-337: the beat's mean inlet pressure (Pa, absolute) and inflow (mL/min) -> recalibrated
        circuit -> the next beat's drive."""
        p, q, steps = self.s.beat_means(reset=True)
        p_in = float(self.un.p(p[0])) + self.p_out_mmhg * MMHG
        q_in = float(q[0]) * self.q_si * 6e7
        self.cal = recalibrate(self.cal, p_in, q_in, self.shape, self.q_in, self.q_target, self.p_out_mmhg)
        self.history.append({"beat": int(beat), "steps": steps, "p_in_pa": p_in, "q_in_ml_min": q_in,
                             "R_seg": self.cal["R_seg"]})
        self.drive()


def save(d, meta, series, frames, cmap=None, lat=None, wall_mm=None, dx_mm=None):
    """The result files of simulate.save (simulate.py:361-380): series.npz (one array per series), meta.json, and,
    with frames ({"t", "p_mmhg", "u_m_s"}: one row per frame of the coarse bins, in the caller's units), fields.npz
    (coarse bin coordinates, origin, dx_mm, wall distance per bin, frame times, p and u as float16)."""
    import json
    import os
    os.makedirs(d, exist_ok=True)
    np.savez_compressed(os.path.join(d, "series.npz"), **{k: np.asarray(v) for k, v in series.items()})
    json.dump(meta, open(os.path.join(d, "meta.json"), "w"), indent=1, default=float)
    if frames is not None and len(frames.get("p_mmhg", [])) and cmap is not None:
        wall = (np.bincount(cmap.inv, weights=np.asarray(wall_mm, float), minlength=cmap.n_bins) / cmap.cnt
                if wall_mm is not None else np.zeros(cmap.n_bins))
        np.savez_compressed(os.path.join(d, "fields.npz"), coords=cmap.uk, origin=np.asarray(lat["origin"]),
                            dx_mm=0.1 if cmap.f > 1 else (dx_mm if dx_mm is not None else lat["dx"]),
                            wall_mm=wall.astype(np.float32), t=np.asarray(frames["t"]),
                            p_mmhg=np.asarray(frames["p_mmhg"], np.float16), u_m_s=np.asarray(frames["u_m_s"], np.float16))
