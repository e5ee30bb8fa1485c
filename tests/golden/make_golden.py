"""Generate the golden fixtures for the lattice tables from the reference implementation itself.

Run in a container that has the reference checkout (pure Python + NumPy; its GPU dialect is not needed for the
table builder):

    python tests/golden/make_golden.py /path/to/CerebroSim

The reference modules `lbm.py` and `validate.py` import the `warp` package at module top. Only their NumPy parts
are exercised here (`lbm.build_lattice`, `lbm.Units`, `lbm.Solver.set_sponge`, `validate.periodic_pipe`,
`validate.open_pipe`), so a permissive stand-in module is registered as `warp` before the import: decorators are
identity functions and every other attribute is an inert callable. No reference kernel runs.

Outputs (in this folder):
  tables_small.npz   full tables (phi, nbr, q, uin, coords, counts, openings) for small lattices;
  tables_hash.json   sha256 of phi / nbr / q / uin / coords plus link counts for full-size lattices
                     (validate.py's pipes and stenosis, the 24x24x64 periodic pipe, the R=24 open pipe);
  sponge.npz         tau per cell from `Solver.set_sponge` on a small open pipe;
  units.json         `Units` conversions at the reference's operating points;
  circuit.json       the lumped circuit (simulate.circuit) and its calibration arithmetic (--circuit-only writes
                     just this file).
"""
import hashlib
import json
import math
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class _Inert:
    """Callable, subscriptable, attribute-rich placeholder standing in for any warp object at import time."""

    def __init__(self, *a, **k):
        pass

    def __call__(self, *a, **k):
        if len(a) == 1 and callable(a[0]) and not k:
            return a[0]                       # used as a decorator
        return _Inert()

    def __getattr__(self, name):
        return _Inert()

    def __getitem__(self, key):
        return _Inert()

    def __mul__(self, other):
        return _Inert()

    __rmul__ = __add__ = __radd__ = __sub__ = __rsub__ = __truediv__ = __mul__


def _install_warp_stub():
    wp = types.ModuleType("warp")
    wp.__getattr__ = lambda name: _Inert()
    wp.kernel = lambda f=None, **k: f if f is not None else (lambda g: g)
    wp.func = lambda f=None, **k: f if f is not None else (lambda g: g)
    wp.constant = lambda x: x
    wp.set_module_options = lambda *a, **k: None
    wp.pi = math.pi
    wp.types = types.SimpleNamespace(vector=lambda length, dtype: _Inert)
    sys.modules["warp"] = wp


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def capture_build(lbm):
    """Wrap lbm.build_lattice so every call records its inputs next to its result."""
    calls = []
    orig = lbm.build_lattice

    def wrapped(phi, origin, dx, openings=(), periodic=(), opening_slack=1.0):
        lat = orig(phi, origin, dx, openings=openings, periodic=periodic, opening_slack=opening_slack)
        calls.append({"phi": np.asarray(phi, np.float32).copy(), "origin": np.asarray(origin, float).tolist(),
                      "dx": float(dx), "periodic": list(periodic), "slack": float(opening_slack),
                      "openings": [{"kind": o["kind"], "centre": np.asarray(o["centre"], float).tolist(),
                                    "normal": np.asarray(o["normal"], float).tolist(), "radius": float(o["radius"])}
                                   for o in openings], "lat": lat})
        return lat

    lbm.build_lattice = wrapped
    return calls, orig


def summary(rec):
    lat = rec["lat"]
    return {"shape": list(np.asarray(rec["phi"]).shape), "origin": rec["origin"], "dx": rec["dx"],
            "periodic": rec["periodic"], "slack": rec["slack"], "openings": rec["openings"],
            "N": int(lat["nbr"].shape[1]), "counts": lat["counts"], "phi": sha(rec["phi"]), "nbr": sha(lat["nbr"]),
            "q": sha(lat["q"]), "uin": sha(lat["uin"]), "coords": sha(lat["coords"])}


def main(ref):
    _install_warp_stub()
    sys.path.insert(0, ref)
    import lbm
    import validate
    calls, build = capture_build(lbm)

    small, hashes = {}, {}

    def keep_small(name, rec):
        lat = rec["lat"]
        small[name + "/phi"] = rec["phi"]
        small[name + "/nbr"] = lat["nbr"]
        small[name + "/q"] = lat["q"]
        small[name + "/uin"] = lat["uin"]
        small[name + "/coords"] = lat["coords"]
        small[name + "/meta"] = np.array(json.dumps(summary(rec)))

    # --- validate.py's periodic pipes (Poiseuille / Womersley lattices)
    for D in (10, 20, 40):
        calls.clear()
        validate.periodic_pipe(D)
        hashes[f"periodic_pipe_D{D}"] = summary(calls[-1])
        if D == 10:
            keep_small("periodic_pipe_D10", calls[-1])

    # --- validate.py's open pipes: straight and tilted, D = 20, 12 diameters (test_open_pipe)
    for name, axis in (("straight", (0, 0, 1)), ("tilted", (1, 2, 2))):
        calls.clear()
        validate.open_pipe(axis, 240, lambda s: np.full_like(s, 10.0, dtype=float))
        hashes[f"open_pipe_{name}_D20"] = summary(calls[-1])
        calls.clear()
        validate.open_pipe(axis, 24, lambda s: np.full_like(s, 4.0, dtype=float))
        keep_small(f"open_pipe_{name}_R4", calls[-1])

    # --- validate.py's 70 % stenosis at 0.1 mm (D0 = 20 cells, Ls = 40, s0 = 80, L = 480)
    def sten_radius(D, sev=0.7):
        R0, Ls, s0 = D / 2, 2 * D, 4 * D

        def radius(s):
            s = np.asarray(s, float)
            x = np.clip((s - s0) / Ls, 0, 1)
            return R0 * (1 - sev * 0.5 * (1 - np.cos(2 * math.pi * x)))
        return radius, (4 + 18) * D + Ls

    rad, L = sten_radius(20)
    calls.clear()
    validate.open_pipe((0, 0, 1), L, rad)
    hashes["stenosis70_D20"] = summary(calls[-1])
    rad, L = sten_radius(8)
    calls.clear()
    validate.open_pipe((0, 0, 1), L, rad)
    keep_small("stenosis70_D8", calls[-1])

    # --- Poiseuille cylinder, R = 10 on 24 x 24 x 64, axis at (11.5, 11.5) + validate.OFFSET, periodic along z
    n, nz, R = 24, 64, 10.0
    c0 = np.array([n / 2 - 0.5, n / 2 - 0.5]) + validate.OFFSET[:2]
    I, J, _ = np.meshgrid(np.arange(n), np.arange(n), np.arange(nz), indexing="ij")
    calls.clear()
    lbm.build_lattice(np.hypot(I - c0[0], J - c0[1]) - R, [0, 0, 0], 1.0, periodic=(2,))
    hashes["poiseuille_R10_L64"] = summary(calls[-1])

    # --- open pipe R = 24, length 192 along z (the pulsatile pipe)
    calls.clear()
    validate.open_pipe((0, 0, 1), 192, lambda s: np.full_like(s, 24.0, dtype=float))
    hashes["open_pipe_R24_L192"] = summary(calls[-1])

    # --- synthetic edge cases: NaN / inf in phi, periodic on all axes, several openings, empty and tiny lattices
    rng = np.random.default_rng(7)
    phi = rng.normal(size=(9, 8, 7)).astype(np.float32) - 0.3
    phi[0, 0, 0] = np.nan
    phi[1, 2, 3] = np.inf
    phi[2, 2, 2] = -np.inf
    phi[3, 3, 3] = 0.0
    phi[4, 4, 4] = -0.0
    calls.clear()
    lbm.build_lattice(phi, [0, 0, 0], 1.0)
    keep_small("noise_nan_inf", calls[-1])
    calls.clear()
    lbm.build_lattice(phi, [0.5, -1.0, 2.0], 0.25, periodic=(0, 1, 2))
    keep_small("noise_periodic_xyz", calls[-1])
    calls.clear()
    lbm.build_lattice(phi, [0, 0, 0], 1.0, periodic=(1,))
    keep_small("noise_periodic_y", calls[-1])

    # a box with two inlets and three outlets on its faces (the last inlet sets every inlet cell's profile)
    g = np.stack(np.meshgrid(np.arange(14), np.arange(12), np.arange(16), indexing="ij"), -1).astype(float)
    box = np.max(np.abs(g - np.array([6.6, 5.4, 7.7])) - np.array([5.2, 4.1, 6.3]), axis=-1).astype(np.float32)
    openings = [{"kind": "outlet", "centre": [6.6, 5.4, 14.0], "normal": [0, 0, 1], "radius": 3.0},
                {"kind": "inlet", "centre": [6.6, 5.4, 1.4], "normal": [0, 0, -1], "radius": 3.5},
                {"kind": "outlet", "centre": [11.8, 5.4, 7.7], "normal": [1, 0, 0], "radius": 2.5},
                {"kind": "inlet", "centre": [1.4, 5.4, 7.7], "normal": [-1, 0, 0], "radius": 2.0},
                {"kind": "outlet", "centre": [6.6, 9.5, 7.7], "normal": [0, 1, 0], "radius": 2.0}]
    for slack in (1.0, 0.0, 2.5):
        calls.clear()
        lbm.build_lattice(box, [0, 0, 0], 1.0, openings=openings, opening_slack=slack)
        keep_small(f"box_openings_slack{slack:g}", calls[-1])
    calls.clear()
    lbm.build_lattice(box * 0.1, [10.0, 20.0, 30.0], 0.1,
                      openings=[dict(o, centre=(np.asarray(o["centre"]) * 0.1 + [10, 20, 30]).tolist(),
                                     radius=o["radius"] * 0.1) for o in openings])
    keep_small("box_openings_scaled", calls[-1])

    calls.clear()
    lbm.build_lattice(np.ones((4, 5, 6), np.float32), [0, 0, 0], 1.0)
    keep_small("empty", calls[-1])
    calls.clear()
    one = np.ones((3, 3, 3), np.float32)
    one[1, 1, 1] = -0.5
    lbm.build_lattice(one, [0, 0, 0], 1.0)
    keep_small("single_node", calls[-1])
    calls.clear()
    lbm.build_lattice(np.full((1, 1, 1), -1.0, np.float32), [0, 0, 0], 1.0, periodic=(0, 1, 2))
    keep_small("one_cell_periodic", calls[-1])

    np.savez_compressed(os.path.join(HERE, "tables_small.npz"), **small)
    with open(os.path.join(HERE, "tables_hash.json"), "w") as f:
        json.dump(hashes, f, indent=1)

    # --- sponge: lbm.Solver.set_sponge on the small open pipe (its NumPy part only, on a minimal stand-in self)
    lbm.build_lattice = build
    lat = build(small["open_pipe_tilted_R4/phi"], [0, 0, 0], 1.0,
                openings=json.loads(str(small["open_pipe_tilted_R4/meta"]))["openings"])
    sp = {}
    for tag, tau, length, tau_max, kinds in (("a", 0.50495, 20.0, 0.55, ("inlet", "outlet")),
                                             ("b", 0.55, 6.0, 0.9, ("outlet",)),
                                             ("c", 0.8, 3.5, 0.6, ("inlet",))):
        holder = {}
        fake = types.SimpleNamespace(lat=lat, N=lat["nbr"].shape[1], tau=tau,
                                     om=types.SimpleNamespace(assign=lambda a, h=holder: h.setdefault("om", a)))
        lbm.Solver.set_sponge(fake, length, tau_max, kinds)
        sp[f"{tag}/tau_cell"] = fake.tau_cell
        sp[f"{tag}/om"] = holder["om"]
        sp[f"{tag}/args"] = np.array(json.dumps({"tau": tau, "length": length, "tau_max": tau_max,
                                                 "kinds": list(kinds)}))
    np.savez_compressed(os.path.join(HERE, "sponge.npz"), **sp)

    # --- units at validate.py's operating points
    units = {}
    for key, (dx, dt) in validate.OPERATING.items():
        u = lbm.Units(dx, dt, 1060.0, 3.5e-3 / 1060.0)
        units[key] = {"dx": dx, "dt": dt, "nu_lu": u.nu_lu, "tau": u.tau, "c": u.c,
                      "u_of_0.02": float(u.u(0.02)), "p_of_1e-4": float(u.p(1e-4)),
                      "u_lu_of_0.6": float(u.u_lu(0.6)), "p_lu_of_1000": float(u.p_lu(1000.0))}
    units["constants"] = {"C": lbm.C.tolist(), "W": lbm.W.tolist(), "OPP": lbm.OPP.tolist(),
                          "WALL": lbm.WALL, "INLET": lbm.INLET, "OUTLET0": lbm.OUTLET0}
    with open(os.path.join(HERE, "units.json"), "w") as f:
        json.dump(units, f, indent=1)
    # --- the reference's vessels (vessel.build is NumPy): centrelines, radii and caps as vessel.sdf_grid packs them
    # (vessel.py:210-227), their bounds (vessel.py:224-227) and validate.artery_lattice's openings (validate.py:294-308)
    import vessel as V
    art = {}
    for case in ("healthy", "narrow70", "occluded"):
        g = V.build(case)
        names, pts, rad, start, count, cp, cn, cr = V._packed(g)
        lo, hi = V.bounds(g)
        openings = []
        for name, b in g["branches"].items():
            for key, kind in (("start", "inlet"), ("end", "outlet")):
                cap = b["caps"][key]
                if cap is not None:
                    r = b["R"][0] if key == "start" else b["R"][-1]
                    openings.append({"kind": kind, "centre": np.asarray(cap[0], float).tolist(),
                                     "normal": np.asarray(cap[1], float).tolist(), "radius": float(r)})
        openings.sort(key=lambda o: o["kind"] != "inlet")
        art[f"{case}/pts"] = pts
        art[f"{case}/rad"] = rad
        art[f"{case}/start"] = np.asarray(start, np.int32)
        art[f"{case}/count"] = np.asarray(count, np.int32)
        art[f"{case}/cap_p"] = cp
        art[f"{case}/cap_n"] = cn
        art[f"{case}/cap_r"] = cr
        art[f"{case}/lo"] = np.asarray(lo, float)
        art[f"{case}/hi"] = np.asarray(hi, float)
        art[f"{case}/meta"] = np.array(json.dumps({"names": names, "blend": V.JUNCTION_BLEND, "openings": openings}))
    np.savez_compressed(os.path.join(HERE, "vessels.npz"), **art)
    print("wrote", sorted(os.listdir(HERE)))
    for k, v in hashes.items():
        print(f"  {k}: N={v['N']} counts={v['counts']}")


def circuit(ref):
    """circuit.json: the reference's lumped circuit (simulate.circuit, simulate.py:138-148) at three segment
    resistances, and the calibrate branch's arithmetic (simulate.py:330-337) on two beat means, with the inputs
    they read (vessel.py's flow targets and inflow waveform, simulate.py's outlet pressure)."""
    _install_warp_stub()
    sys.path.insert(0, ref)
    import simulate
    import vessel as V
    _, shape = V.inflow_waveform(400)
    out = {"inputs": {"q_in_ml_min": V.Q_INLET_MEAN, "q_target_ml_min": V.Q_MCA_TARGET,
                      "p_out_mmhg": simulate.P_OUT_MMHG, "harmonics": simulate.HARMONICS,
                      "shape": np.asarray(shape, float).tolist()},
           "circuit": [], "recalibrate": []}
    for R_seg in (0.0, 1.0e8, 3.0e9):
        c = simulate.circuit(R_seg)
        out["circuit"].append({"R_seg": R_seg, "R_out": [float(x) for x in c["R_out"]],
                               "P_in_coef": [float(x) for x in c["P_in_coef"]], "R_eq": float(c["R_eq"])})
    cal = simulate.circuit(0.0)
    for p_in_mmhg, q_ml_min in ((92.0, 231.0), (101.5, 244.0)):
        # the calibrate branch: R_tot from the beat's mean inlet pressure and inflow, then circuit(R_tot - R_eq)
        p_in = p_in_mmhg * simulate.MMHG
        R_tot = p_in / (q_ml_min * 1e-6 / 60)
        c = simulate.circuit(float(max(R_tot - cal["R_eq"], 0.0)))
        out["recalibrate"].append({"p_in_pa": p_in, "q_in_ml_min": q_ml_min, "R_seg": float(c["R_seg"]),
                                   "P_in_coef": [float(x) for x in c["P_in_coef"]]})
    with open(os.path.join(HERE, "circuit.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote circuit.json")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    ref_dir = args[0] if args else os.environ.get("CEREBROSIM_REF", ".")
    if "--circuit-only" not in sys.argv:
        main(ref_dir)
    circuit(ref_dir)
