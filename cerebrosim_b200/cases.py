"""Named lattices of the validation suite and the benchmark workloads (inputs to `build_lattice`).

`case(name)` returns {"phi", "origin", "dx", "openings", "periodic"} ready for `build_lattice(**case(name))`, plus
"meta" (geometry facts the checks need: pipe start / axis / radius). Names:
  periodic_pipe_D{10,20,40}   validate.py:59-66 (Poiseuille / Womersley pipes, 2 cells long, periodic)
  poiseuille_R10_L64          circular cylinder R = 10, 24 x 24 x 64, periodic along z (~20 k nodes)
  open_pipe_straight_D20      validate.py:179-186, axis (0, 0, 1), 12 diameters
  open_pipe_tilted_D20        the same pipe along (1, 2, 2)
  stenosis70_D{8,20,40}       validate.py:226-239, 70 % cosine narrowing, D0 cells across
  open_pipe_R24_L192          R = 24, 192 long, velocity inlet + pressure outlet (the pulsatile pipe, ~347 k nodes)
  open_pipe_R{r}_L{l}         any other radius / length along z
"""
import re

import numpy as np

from . import geometry as G


def _open(axis, L, radius_fn, meta):
    phi, openings, start, ax = G.open_pipe(axis, L, radius_fn)
    meta = dict(meta, start=start, axis=ax, L=L)
    return {"phi": phi, "origin": [0, 0, 0], "dx": 1.0, "openings": openings, "periodic": (), "meta": meta}


def case(name):
    m = re.fullmatch(r"periodic_pipe_D(\d+)", name)
    if m:
        D = int(m.group(1))
        phi, r, R = G.periodic_pipe(D)
        return {"phi": phi, "origin": [0, 0, 0], "dx": 1.0, "openings": [], "periodic": (2,),
                "meta": {"D": D, "R": R, "r_grid": r}}
    if name == "poiseuille_R10_L64":
        phi, r = G.poiseuille_cylinder()
        return {"phi": phi, "origin": [0, 0, 0], "dx": 1.0, "openings": [], "periodic": (2,),
                "meta": {"R": 10.0, "r_grid": r}}
    m = re.fullmatch(r"open_pipe_(straight|tilted)_D(\d+)", name)
    if m:
        D = int(m.group(2))
        axis = (0, 0, 1) if m.group(1) == "straight" else (1, 2, 2)
        R = D / 2
        return _open(axis, 12 * D, lambda s: np.full_like(s, R, dtype=float), {"D": D, "R": R})
    m = re.fullmatch(r"stenosis70_D(\d+)", name)
    if m:
        D = int(m.group(1))
        radius, L, s0, Ls = G.stenosis_radius(D)
        return _open((0, 0, 1), L, radius, {"D": D, "R": D / 2, "s0": s0, "Ls": Ls})
    m = re.fullmatch(r"open_pipe_R(\d+)_L(\d+)", name)
    if m:
        R, L = float(m.group(1)), int(m.group(2))
        return _open((0, 0, 1), L, lambda s: np.full_like(s, R, dtype=float), {"R": R})
    raise KeyError(f"unknown case {name!r}")


def lattice_args(c):
    """The keyword arguments of build_lattice from a case dict."""
    return {k: c[k] for k in ("phi", "origin", "dx", "openings", "periodic")}


def plug_inlet(lat):
    """Replace the builder's parabolic inlet profile by a plug of unit speed along the inward normal of the last
    inlet (the pulsatile pipe's inflow: the drive then scales it to u0 (1 + 0.5 sin(2 pi t / T)))."""
    inlet = [o for o in lat["openings"] if o["kind"] == "inlet"][-1]
    cells = (np.asarray(lat["nbr"]) == -2).any(0)
    uin = np.zeros_like(np.asarray(lat["uin"]))
    uin[cells] = (-np.asarray(inlet["normal"], float)).astype(np.float32)
    lat["uin"] = uin
    if "_dev" in lat:
        import torch
        lat["_dev"]["uin"] = torch.as_tensor(uin).to(lat["_dev"]["nbr"].device)
    return lat
