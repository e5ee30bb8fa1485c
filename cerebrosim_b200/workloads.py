"""Synthetic stenosed arteries and the workloads built on them: single vessels, a batched sweep and a request stream.

The reference's own vessel (vessel.build) is one patient's carotid traced from a figure; sweeps over clot size and
pressure need many vessels of controlled size, so this module generates them in the same geometry format
({"branches": {name: {"C", "R0", "R", "caps"}}}) and voxelises them with the same signed distance
(vessel.py:178-245, `cerebrosim_b200.vessel`):

- the parent: a natural cubic spline through `n_ctrl` control points spaced evenly along x over `length` mm, each
  displaced sideways (y, z) by a seeded uniform jitter of +-`jitter` mm, radius `radius` mm; a velocity inlet at
  its start and a pressure outlet at its end;
- a cosine stenosis of area reduction `stenosis` (0 .. 1) and length `sten_len` mm centred mid-parent: the radius
  is R (1 - delta (1 + cos(2 pi (s - s0) / sten_len)) / 2) within sten_len / 2 of the centre, (1 - delta)^2 =
  1 - stenosis; a complete occlusion (stenosis 1) is a solid clot `sten_len` long: the parent is split into a
  proximal and a distal branch with flat closed faces at the clot;
- a straight side branch of radius `branch_radius` leaving the parent at `branch_at` of its length (downstream of
  the stenosis) at `branch_angle` degrees to the parent's tangent, towards a seeded azimuth, `branch_len` mm long.
  Its far end is a pressure outlet, or, for an occluded parent, the velocity inlet: the occluded vessel is fed
  only by the branch, and the parent's start becomes a pressure outlet.

`fourier_drive` makes the seeded periodic inflow (mean and peak/mean given); `sweep` and `request_stream` derive
the batched and served workloads (16 vessels of 0.3-3 M nodes; Poisson arrivals).
"""
import math

import numpy as np
from scipy.interpolate import CubicSpline

from . import lbm, vessel

MMHG_REF = 95.0          # mmHg at which a vessel gets the nominal mean inflow


def _resample(P, h):
    """Points along the polyline P at arc spacing ~h (both ends kept), and their arc lengths."""
    seg = np.linalg.norm(np.diff(P, axis=0), axis=1)
    s = np.concatenate([[0.0], np.cumsum(seg)])
    n = max(2, int(math.ceil(s[-1] / h)) + 1)
    t = np.linspace(0.0, s[-1], n)
    return np.column_stack([np.interp(t, s, P[:, a]) for a in range(3)]), t


def _unit(v):
    return v / np.linalg.norm(v)


def stenosed_vessel(seed=3, length=20.0, jitter=2.0, n_ctrl=5, radius=1.5, branch_radius=1.0, branch_angle=40.0,
                    branch_len=15.0, branch_at=0.7, stenosis=0.7, sten_len=3.0, spacing=0.1):
    """A seeded parent artery with a cosine stenosis and one side branch, in the reference's geometry format.
    Lengths in mm; `spacing` is the centreline sample spacing."""
    if not 0.0 <= stenosis <= 1.0:
        raise ValueError(f"stenosis {stenosis}: an area fraction in [0, 1]")
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, length, n_ctrl)
    lat = rng.uniform(-jitter, jitter, size=(n_ctrl, 2))
    spl = CubicSpline(xs, lat, bc_type="natural")
    fine = np.linspace(0.0, length, 40 * int(math.ceil(length / spacing)) + 1)
    C, s = _resample(np.column_stack([fine, spl(fine)]), spacing)
    # cosine stenosis, centred mid-parent
    s0 = 0.5 * s[-1]
    w = np.where(np.abs(s - s0) < 0.5 * sten_len, 0.5 * (1 + np.cos(2 * np.pi * (s - s0) / sten_len)), 0.0)
    delta = 1.0 - math.sqrt(max(0.0, 1.0 - stenosis))
    R0 = np.full(len(C), float(radius))
    R = R0 * (1.0 - delta * w)
    t0, t1 = _unit(C[1] - C[0]), _unit(C[-1] - C[-2])
    branches = {}
    if stenosis >= 1.0:
        # occlusion: a solid clot sten_len long. A union of round cones cannot close a lumen over a bump shorter
        # than its diameter, so the parent is split at the clot's faces, each face a flat closed cut
        a_, b_ = np.searchsorted(s, s0 - 0.5 * sten_len), np.searchsorted(s, s0 + 0.5 * sten_len)
        Cp, Cd = C[:a_], C[b_:]
        tp, td = _unit(Cp[-1] - Cp[-2]), _unit(Cd[1] - Cd[0])
        branches["trunk"] = {"C": Cp, "R0": R0[:a_], "R": R0[:a_].copy(),
                             "caps": {"start": (Cp[0].copy(), -t0), "end": (Cp[-1].copy(), tp, "closed")}}
        branches["trunk_distal"] = {"C": Cd, "R0": R0[b_:], "R": R0[b_:].copy(),
                                    "caps": {"start": (Cd[0].copy(), -td, "closed"), "end": (Cd[-1].copy(), t1)}}
    else:
        branches["trunk"] = {"C": C, "R0": R0, "R": R,
                             "caps": {"start": (C[0].copy(), -t0), "end": (C[-1].copy(), t1)}}
    # side branch from the parent's centreline at branch_at of its length
    k = int(np.argmin(np.abs(s - branch_at * s[-1])))
    tk = _unit(C[min(k + 1, len(C) - 1)] - C[max(k - 1, 0)])
    a = rng.uniform(0.0, 2 * np.pi)
    e1 = _unit(np.cross(tk, [0.0, 0.0, 1.0] if abs(tk[2]) < 0.9 else [0.0, 1.0, 0.0]))
    e2 = np.cross(tk, e1)
    th = math.radians(branch_angle)
    d = math.cos(th) * tk + math.sin(th) * (math.cos(a) * e1 + math.sin(a) * e2)
    Cb, _ = _resample(np.vstack([C[k], C[k] + branch_len * d]), spacing)
    Rb = np.full(len(Cb), float(branch_radius))
    branches["branch"] = {"C": Cb, "R0": Rb.copy(), "R": Rb, "caps": {"start": None, "end": (Cb[-1].copy(), d.copy())}}
    return {"branches": branches, "stenosis": float(stenosis), "seed": int(seed), "occluded": bool(stenosis >= 1.0)}


def openings(g):
    """Inlet at the parent's start; outlets at the parent's end and the branch's end. An occluded parent is fed
    only by its branch: the branch end is the inlet and the parent's start a pressure outlet (a closed pocket
    behind the plug). Inlets first (the order build_lattice numbers them in)."""
    ops = vessel.openings_of(g)
    if g.get("occluded"):
        for o in ops:
            if o["branch"] == "branch":
                o["kind"] = "inlet"
            elif o["kind"] == "inlet":
                o["kind"] = "outlet"
    ops.sort(key=lambda o: o["kind"] != "inlet")
    return ops


def lattice(g, dx, device=None):
    """The vessel's lattice at dx mm, voxelised and built on the GPU; its host tables are copied from the device
    only when read (a solver uses the device copies)."""
    return vessel.artery_lattice(g, dx, openings=openings(g), device=device, host=False)


def fourier_drive(seed, mean=0.03, peak_over_mean=1.8, harmonics=4, floor=0.2):
    """Seeded periodic inflow a0 + sum_k a_k cos(k phi) + b_k sin(k phi) (the coefficient order of lbm.k_clock,
    lbm.py:90-102) with mean `mean` and max / mean = `peak_over_mean`; redrawn until min / mean >= floor."""
    rng = np.random.default_rng(seed)
    phi = np.linspace(0.0, 2 * np.pi, 4096, endpoint=False)
    for _ in range(1000):
        amp = rng.normal(size=(harmonics, 2)) / np.arange(1, harmonics + 1)[:, None]
        wave = sum(amp[k, 0] * np.cos((k + 1) * phi) + amp[k, 1] * np.sin((k + 1) * phi) for k in range(harmonics))
        scale = (peak_over_mean - 1.0) / wave.max()
        if 1.0 + scale * wave.min() >= floor:
            break
    else:  # pragma: no cover - the draw above succeeds for any sensible target
        raise RuntimeError("no admissible waveform")
    coef = [mean]
    for k in range(harmonics):
        coef += [mean * scale * amp[k, 0], mean * scale * amp[k, 1]]
    return coef


def inflow_scale(pressure_mmhg, stenosis, peak_over_mean=1.8, u_mean=0.03, u_throat_max=0.1):
    """Mean inlet velocity (lattice units) for a vessel at mean pressure p: proportional to p / 95 mmHg, capped so
    that the mean throat velocity at peak flow stays within u_throat_max (the stability limit of the scheme at
    tau 0.52). An occluded parent (stenosis 1) is fed by its branch and has no throat."""
    u = u_mean * pressure_mmhg / MMHG_REF
    if stenosis < 1.0:
        u = min(u, u_throat_max * (1.0 - stenosis) / peak_over_mean)
    return u


def dx_for_nodes(target, nodes_at_ref, dx_ref):
    """Spacing that gives about `target` fluid nodes, for a vessel with nodes_at_ref nodes at dx_ref."""
    return dx_ref * (nodes_at_ref / float(target)) ** (1.0 / 3.0)


def estimated_nodes(g, dx):
    """Lumen volume / dx^3 from the centrelines (round cones summed; the junction overlap is ignored)."""
    vol = 0.0
    for b in g["branches"].values():
        C, R = np.asarray(b["C"]), np.clip(np.asarray(b["R"]), 0.0, None)
        seg = np.linalg.norm(np.diff(C, axis=0), axis=1)
        vol += float((np.pi / 3.0 * seg * (R[:-1] ** 2 + R[:-1] * R[1:] + R[1:] ** 2)).sum())
    return vol / dx ** 3


SWEEP_STENOSIS = [0.0, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9, 0.95, 1.0, 0.3, 0.5, 0.7, 0.9]


def sweep(n=16, seed0=100, nodes_lo=0.3e6, nodes_hi=3.0e6, p_lo=70.0, p_hi=145.0):
    """The batched sweep: n vessels (seeds seed0 ..), stenosis 0, 10, ..., 90, 95, 100 % then repeats at other
    pressures, mean pressures evenly over [p_lo, p_hi] mmHg, sizes log-spaced over [nodes_lo, nodes_hi] in a seeded
    order. Returns a list of specs {seed, stenosis, pressure, nodes}."""
    rng = np.random.default_rng(seed0)
    sizes = nodes_lo * (nodes_hi / nodes_lo) ** (np.arange(n) / max(1, n - 1))
    order = rng.permutation(n)
    return [{"seed": seed0 + i, "stenosis": SWEEP_STENOSIS[i % len(SWEEP_STENOSIS)],
             "pressure": p_lo + (p_hi - p_lo) * i / max(1, n - 1), "nodes": float(sizes[order[i]])}
            for i in range(n)]


def request_stream(n, seed=5, rate=2.0, nodes_lo=0.2e6, nodes_hi=4.0e6, p_lo=70.0, p_hi=145.0, beats=(1, 4)):
    """Poisson arrivals at `rate` per second: each request draws a clot (area fraction U[0, 1]), a mean pressure
    U[p_lo, p_hi] mmHg, a whole number of beats U{beats} and a vessel size log-uniform over [nodes_lo, nodes_hi]."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    out = []
    for k in range(n):
        out.append({"id": k, "arrival": float(t[k]), "seed": int(1000 + k), "stenosis": float(rng.uniform(0, 1)),
                    "pressure": float(rng.uniform(p_lo, p_hi)), "beats": int(rng.integers(beats[0], beats[1] + 1)),
                    "nodes": float(math.exp(rng.uniform(math.log(nodes_lo), math.log(nodes_hi))))})
    return out


def spec_lattice(spec, device=None):
    """Vessel and lattice of a sweep / request spec: the spec's seed and stenosis, dx chosen for its node count."""
    g = stenosed_vessel(seed=spec["seed"], stenosis=spec["stenosis"])
    dx = spec.get("dx") or dx_for_nodes(spec["nodes"], estimated_nodes(g, 0.05), 0.05)
    return g, lattice(g, dx, device=device), dx


def configure(s, spec, lat, period=8000, ramp=1000, sponge=(8, 0.6)):
    """A spec's boundary conditions on a solver (the package's or any with the reference's Solver interface): a
    Fourier drive of period `period` steps scaled by the spec's pressure, pressure outlets at 0, a sponge over
    `sponge[0]` cells at the openings."""
    s.set_sponge(sponge[0], sponge[1])
    s.set_outlet_pressure([0.0] * lat["n_outlets"])
    u = inflow_scale(spec["pressure"], spec["stenosis"])
    s.set_drive([c * u / 0.03 for c in fourier_drive(spec["seed"])], period=period, ramp=ramp)
    return s


def make_solver(spec, lat, tau=0.52, period=8000, ramp=1000, storage="f32", block=None, sponge=(8, 0.6),
                device=None, order="c"):
    """Solver for a spec on its lattice (tau, regularised collision), configured by `configure`."""
    s = lbm.Solver(lat, (tau - 0.5) / 3.0, model="regularised", storage=storage, block=block, device=device,
                   order=order)
    return configure(s, spec, lat, period, ramp, sponge)


def build_spec(spec, storage="f32", block=None, device=None, **kw):
    """Vessel, lattice and solver of a spec -> (solver, geometry, lattice, dx)."""
    g, lat, dx = spec_lattice(spec, device=device)
    return make_solver(spec, lat, storage=storage, block=block, device=device, **kw), g, lat, dx


RHO = 1060.0             # kg/m^3, blood (the reference's vessel.py constants)
NU = 3.5e-3 / RHO        # m^2/s


def pressure_ends(g):
    """The vessel's open ends as pressure boundaries (all of build_lattice's "outlet" kind), the feeding end first:
    end 0 takes the drive as its pressure, the others drain through resistances (simulate.py's ends)."""
    return [dict(o, kind="outlet") for o in openings(g)]


def calibrated_solver(spec, dx_mm=None, storage="f32", block=None, device=None, order="c", steps_per_beat=8000,
                      tau=0.52, pref_lu=0.002, target_share=135.0 / 240.0, relax_steps=100, sponge=(8, 0.6)):
    """A generated vessel run as simulate.run runs the reference's arteries (simulate.py:253-337): pressure inlet
    driven by the lumped circuit's inlet pressure, resistance outlets relaxed towards R Q - pref, flow measured on
    slabs inside each end, and the inlet pressure recalibrated after every beat from the beat's mean inlet pressure
    and inflow (`simulate.Calibration`, attached as `.calibration`).

    Units: dx from the spec (its node count) unless given; dt such that tau holds for blood's viscosity. The target
    mean inflow is the vessel's nominal mean inlet velocity (inflow_scale) through the inlet's area, target_share of
    it for the parent's outlet (the reference's MCA share, 135 of 240 mL/min); the outlets' mean pressure pref_lu
    (lattice units) sets the pressure scale; the inflow waveform is the vessel's seeded Fourier drive, normalised
    to mean 1. The spec's vessel must not be occluded (the parent must carry the flow from end 0)."""
    from . import simulate as S
    g = stenosed_vessel(seed=spec["seed"], stenosis=spec["stenosis"])
    if g["occluded"]:
        raise ValueError("a calibrated vessel needs an open parent")
    dx_mm = dx_mm or spec.get("dx") or dx_for_nodes(spec["nodes"], estimated_nodes(g, 0.05), 0.05)
    ends = pressure_ends(g)
    lat = vessel.artery_lattice(g, dx_mm, openings=ends, device=device)
    nu_lu = (tau - 0.5) / 3.0
    dx = dx_mm * 1e-3
    un = lbm.Units(dx, nu_lu * dx * dx / NU, RHO, NU)
    u_lu = inflow_scale(spec["pressure"], spec["stenosis"])
    q_in = u_lu * un.c * math.pi * (ends[0]["radius"] * 1e-3) ** 2 * 6e7          # mL/min
    coef = fourier_drive(spec["seed"])
    t = np.arange(400) / 400.0
    wave = coef[0] + sum(coef[2 * k - 1] * np.cos(2 * np.pi * k * t) + coef[2 * k] * np.sin(2 * np.pi * k * t)
                         for k in range(1, (len(coef) - 1) // 2 + 1))
    p_out_mmhg = pref_lu * RHO * un.c ** 2 / S.MMHG
    cal = S.Calibration(un, wave / wave.mean(), q_in, target_share * q_in, p_out_mmhg, steps_per_beat,
                        ramp=min(1000, steps_per_beat // 8))
    flux = S.flux_slabs(lat, ends, dx_mm)
    s = S.ArterySolver(lat, nu_lu, flux, cal.R_lu(len(ends)), cal.pref_lu, 1.0 / relax_steps, model="regularised",
                       storage=storage, block=block, device=device, order=order)
    s.set_sponge(sponge[0], sponge[1], kinds=("outlet",))
    cal.attach(s)
    s.calibration = cal
    return s


def calibrated_builder(spec, storage, block, device, steps_per_beat, order="c"):
    """serve.Server builder of calibrated requests (pair with serve.recalibrate_on_beat)."""
    s = calibrated_solver(spec, storage=storage, block=block, device=device, order=order,
                          steps_per_beat=steps_per_beat)
    for k in ("nbr", "q", "_dev"):
        s.lat.pop(k, None)
    return s

