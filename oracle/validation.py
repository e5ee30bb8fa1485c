"""CerebroSim's solver validation (validate.py) restated over any solver with the `lbm.Solver` interface.

The checks, their geometry and their analytic answers follow validate.py: Poiseuille (validate.py:69-83),
Womersley (validate.py:86-117), open pipe with velocity inlet / pressure outlet (validate.py:125-215) and the 70 %
stenosis against Young-Tsai (validate.py:218-286). Each function takes `build` (a build_lattice) and `make`
(a Solver constructor), so the same harness drives the B200 solver and any other implementation. The published
results of the reference (reports/step3_report.md:20-50, geometry/solver.json:20-175) are in PUBLISHED.
"""
import math
import time

import numpy as np

from cerebrosim_b200 import cases

RHO = 1060.0                     # kg/m^3 (vessel.py:49)
MU = 3.5e-3                      # Pa s (vessel.py:50)
NU = MU / RHO
OPERATING = {"healthy": (1.0e-4, 5.0e-6), "narrow70": (1.0e-4, 2.0e-6), "narrow70_fine": (5.0e-5, 1.0e-6)}
SOLVER = {"model": "regularised"}
SPONGE_TAU = 0.55

# reference results (geometry/solver.json:20-175): Poiseuille L2 / flow error, Womersley L2, open pipe errors,
# stenosis pressure drop and MLUPS on an RTX 3090
PUBLISHED = {
    "poiseuille": {(10, True): (0.13532128869870114, -0.14670134092831366),
                   (20, True): (0.03429092846606971, -0.03803448455849523),
                   (40, True): (0.009187449059085594, -0.010294269016544288),
                   (20, False): (0.20496644204979705, -0.22679752766633754)},
    "womersley": {1.4: (194172, 0.03370675662345126), 2.8: (48540, 0.03302506896494258),
                  5.6: (12132, 0.060357378395948014)},
    "open_pipe": {"straight": {"grad_err": 0.08768536633211488, "flow_vs_inlet": -0.001167730051564786,
                               "profile_l2": 0.01247263825422971, "steps": 60000},
                  "tilted": {"grad_err": 0.058565768905948445, "flow_vs_inlet": -0.002742054870268462,
                             "profile_l2": 0.02435777993182073, "steps": 60000}},
    "stenosis": {("narrow70", 100): {"dp_Pa": 3556.4159733738034, "steps": 289600, "mlups": 546.1889225975641},
                 ("narrow70", 200): {"dp_Pa": 12536.677903972353, "steps": 270000, "mlups": 527.5871867922236},
                 ("narrow70_fine", 200): {"dp_Pa": 8247.892698620224, "steps": 289600, "mlups": 658.9443148454122}},
}


class _Units:
    def __init__(self, dx, dt):
        self.dx, self.dt = dx, dt
        self.nu_lu = NU * dt / dx ** 2
        self.tau = 3.0 * self.nu_lu + 0.5
        self.c = dx / dt

    def u_lu(self, u):
        return u / self.c

    def p(self, p_lu):
        return np.asarray(p_lu) * RHO * self.c ** 2


def units(key):
    return _Units(*OPERATING[key])


def l2(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def poiseuille(build, make, D, bouzidi, nu=None):
    """Steady pipe flow driven by a body force: L2 error against the parabola and the flow error."""
    nu = units("healthy").nu_lu if nu is None else nu
    c = cases.case(f"periodic_pipe_D{D}")
    lat = build(**cases.lattice_args(c))
    R = c["meta"]["R"]
    r = c["meta"]["r_grid"][tuple(lat["coords"].T)]
    s = make(lat, nu, bouzidi=bouzidi, **SOLVER)
    F = 4 * nu * 0.02 / R ** 2
    s.set_force([0, 0, F])
    steps = int(14 * R * R / (5.78 * nu))
    s.run(steps)
    _, u = s.fields()
    ua = F / (4 * nu) * (R ** 2 - r ** 2)
    return {"D": D, "bouzidi": bouzidi, "steps": steps, "l2": l2(u[:, 2], ua),
            "flow_err": float(u[:, 2].sum() / ua.sum() - 1), "ok": s.ok()}


def womersley_exact(r, R, Wo, F0, w, t):
    from scipy.special import jv
    k = (1j ** 1.5) * Wo
    U = F0 / (1j * w) * (1 - jv(0, k * r / R) / jv(0, k))
    return np.real(U * np.exp(1j * w * t))


def womersley_flow(r, R, Wo, U_hat, w, t):
    """Oscillatory pipe flow of prescribed cross-section mean velocity Re{U_hat e^(i w t)} (the textbook Womersley
    solution written for a flow rate instead of a pressure gradient): Re{U_hat (1 - J0(k r / R) / J0(k)) /
    (1 - 2 J1(k) / (k J0(k))) e^(i w t)}, k = i^(3/2) Wo. The pressure-driven form above has the same shape."""
    from scipy.special import jv
    k = (1j ** 1.5) * Wo
    shape = (1 - jv(0, k * r / R) / jv(0, k)) / (1 - 2 * jv(1, k) / (k * jv(0, k)))
    return np.real(U_hat * shape * np.exp(1j * w * t))


def womersley(build, make, Wo, D=20, phases=12, nu=None):
    """Pulsatile pipe flow: L2 error over 12 phases of the third period against the Bessel solution."""
    nu = units("healthy").nu_lu if nu is None else nu
    c = cases.case(f"periodic_pipe_D{D}")
    lat = build(**cases.lattice_args(c))
    R = c["meta"]["R"]
    r = c["meta"]["r_grid"][tuple(lat["coords"].T)]
    T = int(round(2 * math.pi * R * R / (Wo * Wo * nu) / phases)) * phases
    w = 2 * math.pi / T
    Wo = R * math.sqrt(w / nu)
    rr = np.linspace(0, R, 50)
    peak = max(np.abs(womersley_exact(rr, R, Wo, 1.0, w, t)).max() for t in np.linspace(0, T, 24))
    F0 = 0.02 / peak
    s = make(lat, nu, **SOLVER)
    s.set_force([0, 0, F0])
    s.set_drive([0.0, 1.0, 0.0], period=T)
    s.run(2 * T)
    num = den = 0.0
    for _ in range(phases):
        s.run(T // phases)
        _, u = s.fields()
        ua = womersley_exact(r, R, Wo, F0, w, s.steps - 0.5)
        num += ((u[:, 2] - ua) ** 2).sum()
        den += (ua ** 2).sum()
    return {"Wo": Wo, "period_steps": T, "l2": float(math.sqrt(num / den)), "ok": s.ok()}


def section_profile(sc, values, L, nb=None):
    nb = nb or int(L)
    edges = np.linspace(0, L, nb + 1)
    k = np.clip(np.digitize(sc, edges) - 1, 0, nb - 1)
    cnt = np.bincount(k, minlength=nb)
    m = np.bincount(k, weights=values, minlength=nb) / np.maximum(cnt, 1)
    return 0.5 * (edges[1:] + edges[:-1]), m


def flow_rate(sc, u_axial, s0, s1):
    m = (sc >= s0) & (sc < s1)
    return float(u_axial[m].sum() / (s1 - s0))


def run_steady(s, measure, chunk, min_chunks=4, max_chunks=40, tol=2e-4):
    hist = []
    for it in range(max_chunks):
        s.run(chunk)
        if not s.ok():
            return hist, False
        hist.append(measure())
        if it + 1 >= min_chunks and abs(hist[-1][0] - hist[-2][0]) <= tol * abs(hist[-1][0]):
            break
    return hist, True


def open_pipe(build, make, name, D=20, length_d=12, U_phys=0.6):
    """Velocity inlet + pressure outlet pipe: pressure gradient vs Hagen-Poiseuille, profile, flow."""
    un = units("healthy")
    U = float(un.u_lu(U_phys))
    c = cases.case(f"open_pipe_{name}_D{D}")
    lat = build(**cases.lattice_args(c))
    R, L = D / 2, length_d * D
    sc, rc = cases.G.axial_radial(lat["coords"], c["meta"]["start"], c["meta"]["axis"])
    ax = c["meta"]["axis"]
    s = make(lat, un.nu_lu, **SOLVER)
    s.set_sponge(D, SPONGE_TAU)
    s.set_drive([U], ramp=4000)
    s.set_outlet_pressure([0.0])
    a, b = 3 * D, (length_d - 3) * D

    def measure():
        p, u = s.fields()
        ua = u @ ax
        Qf = flow_rate(sc, ua, a, b)
        sm, pm = section_profile(sc, p, L)
        m = (sm > a) & (sm < b)
        slope = np.polyfit(sm[m], pm[m], 1)[0]
        return -slope, Qf, ua

    hist, ok = run_steady(s, measure, chunk=10000, min_chunks=6)
    G, Qf, ua = hist[-1]
    G_exact = 8 * un.nu_lu * Qf / (math.pi * R ** 4)
    mid = (sc > a) & (sc < b)
    Um = Qf / (math.pi * R * R)
    return {"name": name, "cells": lat["nbr"].shape[1], "steps": s.steps, "ok": ok, "grad_err": G / G_exact - 1,
            "flow_vs_inlet": Qf / (U * math.pi * R * R) - 1,
            "profile_l2": l2(ua[mid], 2 * Um * (1 - (rc[mid] / R) ** 2)), "counts": lat["counts"]}


def young_tsai(U0, D0, D1, Ls):
    ar = (D0 / D1) ** 2
    Kv = 32 * (0.83 * Ls + 1.64 * D1) / D0 * ar ** 2
    return Kv * MU * U0 / D0 + 1.52 / 2 * RHO * (ar - 1) ** 2 * U0 ** 2


def stenosis(build, make, u_key, Re0, sev=0.7, D0_mm=2.0, Ls_mm=4.0, sync=None):
    """70 % cosine narrowing: steady pressure drop vs Young-Tsai, and the solver's MLUPS over the run."""
    un = units(u_key)
    D = D0_mm * 1e-3 / un.dx
    c = cases.case(f"stenosis70_D{int(round(D))}")
    lat = build(**cases.lattice_args(c))
    s0, Ls, L = c["meta"]["s0"], c["meta"]["Ls"], c["meta"]["L"]
    sc, rc = cases.G.axial_radial(lat["coords"], c["meta"]["start"], c["meta"]["axis"])
    U0_phys = Re0 * NU / (D0_mm * 1e-3)
    U = float(un.u_lu(U0_phys))
    s = make(lat, un.nu_lu, **SOLVER)
    s.set_sponge(D, SPONGE_TAU)
    s.set_drive([U], ramp=int(0.3 * L / U))
    s.set_outlet_pressure([0.0])
    sc_mid = s0 + Ls / 2

    def measure():
        p, _ = s.fields()
        sm, pm = section_profile(sc, p, L)
        up = (sm > 1 * D) & (sm < s0 - 0.5 * D)
        dn = (sm > L - 6 * D) & (sm < L - D)
        fu = np.polyfit(sm[up], pm[up], 1)
        fd = np.polyfit(sm[dn], pm[dn], 1)
        return (np.polyval(fu, sc_mid) - np.polyval(fd, sc_mid),)

    flow_through = L / U
    t0 = time.perf_counter()
    hist, ok = run_steady(s, measure, chunk=int(0.25 * flow_through) // 200 * 200, min_chunks=8, max_chunks=24,
                          tol=2e-3)
    if sync:
        sync()
    secs = time.perf_counter() - t0
    dp_lu = hist[-1][0]
    if len(hist) >= 4:
        dp_lu = float(np.mean([h[0] for h in hist[-4:]]))
    dp = float(un.p(dp_lu))
    yt = young_tsai(U0_phys, D0_mm * 1e-3, D0_mm * 1e-3 * (1 - sev), Ls_mm * 1e-3)
    return {"key": u_key, "Re0": Re0, "cells": lat["nbr"].shape[1], "steps": s.steps, "ok": ok, "dp_Pa": dp,
            "young_tsai_Pa": yt, "vs_young_tsai": dp / yt - 1, "secs": secs,
            "mlups": lat["nbr"].shape[1] * s.steps / secs / 1e6}
