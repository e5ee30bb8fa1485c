"""Run a named lattice for a number of steps and print throughput (a small command-line front end).

    python -m cerebrosim_b200.run_case --case open_pipe_R24_L192 --steps 200 [--storage f16] [--block 128]
    python -m cerebrosim_b200.run_case --artery 3 --steps 200 [--dx 0.05]    # a generated stenosed artery

The open pipes get the pulsatile plug inlet used by bench.py (u0 (1 + 0.5 sin(2 pi t / 4000)), u0 = 0.02, tau 0.55,
pressure outlet); periodic pipes get a body force. --artery SEED runs the stenosed-artery generator's vessel of that
seed (70 % stenosis, side branch, Fourier inflow, tau 0.52; about 1.57 M nodes at dx 0.05 mm for seed 3). Steps run
as CUDA graphs of 100 steps plus single launches.
"""
import argparse
import json
import time

import numpy as np
import torch

from . import cases, lbm


def plug_inlet(lat):
    inlet = [o for o in lat["openings"] if o["kind"] == "inlet"][-1]
    cells = (lat["nbr"] == lbm.INLET).any(0)
    uin = np.zeros_like(lat["uin"])
    uin[cells] = (-np.asarray(inlet["normal"], float)).astype(np.float32)
    lat["uin"] = uin
    if "_dev" in lat:
        lat["_dev"]["uin"] = torch.as_tensor(uin).to(lat["_dev"]["nbr"].device)
    return lat


def make_solver(name, storage="f32", block=None, tau=0.55, device=None):
    c = cases.case(name)
    lat = lbm.build_lattice(**cases.lattice_args(c), device=device)
    nu = (tau - 0.5) / 3.0
    if lat["n_outlets"] or any(o["kind"] == "inlet" for o in lat["openings"]):
        lat = plug_inlet(lat)
        s = lbm.Solver(lat, nu, model="regularised", storage=storage, block=block, device=device)
        s.set_drive([0.02, 0.0, 0.01], period=4000)
        s.set_outlet_pressure([0.0] * max(1, lat["n_outlets"]))
    else:
        s = lbm.Solver(lat, nu, model="regularised", storage=storage, block=block, device=device)
        s.set_force([0.0, 0.0, 1e-6])
    return s


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="open_pipe_R24_L192")
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"])
    ap.add_argument("--block", type=int, default=None)
    ap.add_argument("--artery", type=int, default=None, help="seed of a generated stenosed artery")
    ap.add_argument("--dx", type=float, default=0.05, help="voxel size of --artery, mm")
    a = ap.parse_args()
    if a.artery is not None:
        from . import workloads
        spec = {"seed": a.artery, "stenosis": 0.7, "pressure": 95.0}
        lat = workloads.lattice(workloads.stenosed_vessel(a.artery), a.dx)
        s = workloads.make_solver(spec, lat, storage=a.storage, block=a.block)
        a.case = f"artery_seed{a.artery}_dx{a.dx}"
    else:
        s = make_solver(a.case, a.storage, a.block)
    s.run(10)
    s.synchronize()
    t = time.perf_counter()
    s.run(a.steps, chunk=100)
    s.synchronize()
    secs = time.perf_counter() - t
    print(json.dumps({"case": a.case, "nodes": s.N, "steps": a.steps, "storage": a.storage, "block": s.block,
                      "mlups": s.N * a.steps / secs / 1e6, "ok": s.ok()}))


if __name__ == "__main__":
    main()
