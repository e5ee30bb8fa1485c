"""Autotuner of the step's launch shape and node ordering, by measurement on the GPU.

For a lattice (or a representative of a batch) each candidate — threads per bulk block x internal node order
(lbm.node_order: the lattice's C order, C order along the vessel's longest axis, a Morton curve) — is built, warmed
up and timed with CUDA events over a short run on the solver's stream; the fastest wins. A batch shares one block
size; the node order is per instance but is chosen once for a family of similar vessels. `tune_schedule` chooses
a batch's schedule (batch.SCHEDULES: fused launches or instance after instance) the same way, on the batch itself.
"""
import torch

from . import lbm

BLOCKS = (64, 128, 192, 256)


def time_steps(s, steps, warmup):
    """Seconds per step of solver s over `steps` steps after `warmup` (CUDA graphs of 100 steps)."""
    s.run(warmup, chunk=100)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.device(s.dev):
        e0.record(s.stream)
        s.run(steps, chunk=100)
        e1.record(s.stream)
    s.synchronize()
    return e0.elapsed_time(e1) * 1e-3 / steps


def tune(lat, nu_lu, configure=None, storage="f32", blocks=BLOCKS, orders=lbm.ORDERS, steps=300, warmup=100,
         device=None, **solver_kw):
    """Time every (block, order) candidate on `lat` and return (best, table): best = {"block", "order",
    "us_per_step", "mlups"}; table = one such dict per candidate. `configure(solver)` sets the drive, outlets and
    sponge before timing (the boundary work is part of the step)."""
    table = []
    n = lbm.n_nodes(lat)
    seen = set()
    for order in orders:
        perm = lbm.node_order(lat, order)
        key_order = "c" if perm is None else order      # an order that equals C order is not timed twice
        for block in blocks:
            if (key_order, block) in seen:
                continue
            seen.add((key_order, block))
            s = lbm.Solver(lat, nu_lu, storage=storage, block=block, order=order, device=device, **solver_kw)
            if configure is not None:
                configure(s)
            sec = time_steps(s, steps, warmup)
            table.append({"block": block, "order": order, "us_per_step": sec * 1e6, "mlups": n / sec / 1e6})
            del s
    best = min(table, key=lambda r: r["us_per_step"])
    return dict(best), table


def tune_schedule(batch, steps=400, chunk=200, warmup=200):
    """Time each batch schedule on `batch` (its members advance `warmup + steps` steps per candidate) and leave the
    fastest set -> (best, table): best = {"schedule", "us_per_step"}; table = one such dict per schedule. The
    schedules give the same results, so timing them advances the members as ordinary steps would."""
    from .batch import SCHEDULES
    table = []
    for sch in SCHEDULES:
        batch.schedule = sch
        batch.run(warmup, chunk=chunk)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.device(batch.dev):
            e0.record(batch.stream)
            batch.run(steps, chunk=chunk)
            e1.record(batch.stream)
        batch.synchronize()
        table.append({"schedule": sch, "us_per_step": e0.elapsed_time(e1) * 1e3 / steps})
    best = min(table, key=lambda r: r["us_per_step"])
    batch.schedule = best["schedule"]
    return dict(best), table
