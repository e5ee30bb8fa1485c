"""Serving loop: simulation requests (clot size, mean pressure, beats) solved as they arrive, with continuous batching.

The reference runs each simulation as its own one-GPU job (simulate.py, submitted as a Slurm job array); a request
waits for a whole GPU. Here one process serves a stream of requests on one GPU:

- requests queue in arrival order; the head of the queue is admitted when the active set has a free slot and its
  estimated device memory fits the HBM budget (its lattice is then built on the GPU and its populations stay
  resident until its last beat);
- every active request advances in the same batched launches (`BatchSolver`), chunk after chunk; a request joins
  or leaves between chunks with its own buffer parity, so requests that arrive while others run overlap on the
  device instead of waiting for them;
- the host keeps `ahead` chunks enqueued and learns of their completion through CUDA events, so admissions, lattice
  builds and result read-back overlap the GPU's work; beat ends are timed on the device timeline.

Each request's result is the same as when it runs alone: the batched kernels apply each instance's own arithmetic
to its own buffers, whatever else is in the launch.
"""
import collections
import time

import numpy as np
import torch

from . import workloads
from .batch import BatchSolver

# resident device bytes per fluid node, populations + velocity + tables (estimate used for admission; the
# measured figure replaces it once the request is built)
BYTES_PER_NODE = {"f32": 380.0, "f16": 270.0, "bf16": 270.0}


class Request:
    """One solve: `spec` as workloads.request_stream makes it ({id, arrival, seed, stenosis, pressure, beats,
    nodes}). Filled in by the server: admit / done (seconds since the stream started), beat_end (device timeline,
    seconds), queue_wait, N, bytes, ok, fields."""

    def __init__(self, spec):
        self.spec = dict(spec)
        self.id = spec.get("id")
        self.arrival = float(spec.get("arrival", 0.0))
        self.beats = int(spec["beats"])
        self.admit = None
        self.done = None
        self.beat_end = []
        self.N = 0
        self.bytes = 0
        self.ok = None
        self.fields = None
        self.solver = None
        self.steps_total = 0
        self.steps_enq = 0
        self.evicted = None          # beat after which the request was evicted for diverging
        self.beat_flags = []         # device flags of non-finite densities, one per enqueued beat end

    @property
    def queue_wait(self):
        return None if self.admit is None else self.admit - self.arrival

    def beat_latencies(self):
        """Wall time of each beat: from admission (first beat) or the previous beat's end to this beat's end."""
        ends = [self.admit] + list(self.beat_end)
        return [b - a for a, b in zip(ends[:-1], ends[1:])]


def default_builder(spec, storage, block, device, steps_per_beat, order="c"):
    """Solver for a request: the workloads generator's vessel at the request's size, clot and pressure."""
    g, lat, dx = workloads.spec_lattice(spec, device=device)
    s = workloads.make_solver(spec, lat, storage=storage, block=block, period=steps_per_beat,
                              ramp=min(1000, steps_per_beat // 8), device=device, order=order)
    lat.pop("_dev", None)          # the full tables: the solver keeps its compressed form
    for k in ("nbr", "q"):
        lat.pop(k, None)
    return s


class Server:
    """Continuous-batching server on one GPU.

    storage: population format of every request's solver; FP16 by default, the 16-bit form that holds velocity and
    wall shear stress within 1 % of an FP64 run on the 1.57 M-node artery (BF16 does not: about 11 % and 12 %).
    budget_bytes: device memory the resident requests may hold (admission control); max_active: largest batch;
    chunk: steps per scheduling round (a divisor of steps_per_beat); graph_chunk: steps per captured graph;
    ahead: chunks kept enqueued; keep_fields: read each result's (p, u) back to the host; block and order: the
    launch shape and node order of every request's solver (autotune.tune picks them); schedule: the batch's schedule
    (batch.SCHEDULES; autotune.tune_schedule picks it); on_beat(request, beat): called
    when a request completes a beat (not its last), with its solver's state final for that beat — what it changes
    (a recalibrated drive: recalibrate_on_beat) applies from the next beat's first step.

    Divergence: at every beat end (before on_beat) a request's densities are checked for non-finite values
    (simulate.py:321-322 raises there) by a reduction enqueued on the batch stream right after the beat's last
    step; a request that has diverged is evicted at once — its steps stop, its slot and
    budget are released, and it ends with ok = False and `evicted` = the beat — while the others go on unchanged.

    log(record): called at every beat end with a JSON-ready dict — request id, beat, device time (s), the beat's
    latency (s), nodes and the request's update rate over the beat (MLUPS) — for a per-beat metrics stream."""

    def __init__(self, budget_bytes=150e9, storage="f16", steps_per_beat=8000, chunk=1000, graph_chunk=200,
                 max_active=64, block=128, ahead=2, keep_fields=True, device=None, builder=default_builder,
                 order="c", on_beat=None, schedule="fused", log=None):
        if steps_per_beat % chunk or chunk % 2 or graph_chunk % 2:
            raise ValueError("chunk must divide steps_per_beat; chunk and graph_chunk must be even")
        self.budget = float(budget_bytes)
        self.storage = storage
        self.steps_per_beat = int(steps_per_beat)
        self.chunk = int(chunk)
        self.graph_chunk = int(min(graph_chunk, chunk))
        self.max_active = int(max_active)
        self.block = int(block)
        self.ahead = max(1, int(ahead))
        self.keep_fields = bool(keep_fields)
        self.device = device
        self.builder = builder
        self.order = order
        self.on_beat = on_beat
        self.log = log
        self.schedule = schedule
        self.trace = []         # (seconds, active requests, reserved bytes) after each admission

    def estimate(self, spec):
        return BYTES_PER_NODE[self.storage] * float(spec["nodes"])

    def _admit(self, r, batch, t0):
        # built on the side stream, which never waits for the batch: the enqueued chunks keep running meanwhile
        before = torch.cuda.memory_allocated(self.device)
        with torch.cuda.stream(self._side):
            s = self.builder(r.spec, self.storage, self.block, self.device, self.steps_per_beat, self.order)
        self._side.synchronize()
        s.synchronize()
        r.bytes = max(0, torch.cuda.memory_allocated(self.device) - before)
        r.solver, r.N = s, s.N
        r.steps_total = r.beats * self.steps_per_beat
        r.steps_enq = 0
        batch.add(s)
        r.admit = time.perf_counter() - t0

    def _finish(self, r, t_done):
        # the chunk that ended the request has completed: its buffers are final; read them on the side stream
        s = r.solver
        r.done = t_done
        with torch.cuda.stream(self._side):
            r.ok = s.ok()
            if self.keep_fields:
                r.fields = s.fields()
        r.solver = None

    def _flag_beat(self, batch, r):
        """Enqueue, on the batch stream right after the chunk that ends one of r's beats, a device flag of whether
        any of r's densities is non-finite (read once that chunk has completed)."""
        with torch.cuda.stream(batch.stream):
            r.beat_flags.append(torch.isfinite(r.solver.rho).logical_not().any())

    def _finite(self, r):
        """Densities all finite at the beat end just completed (the oldest flag `_flag_beat` enqueued)."""
        return not (r.beat_flags and bool(r.beat_flags.pop(0).item()))

    def _evict(self, r, beat, t):
        """Stop a diverged request: leave the batch once the chunks already enqueued for it have run, release its
        slot and budget."""
        s = r.solver
        if s in self._batch.members:
            self._batch.remove(s, sync=True)
        if r in self._active:
            self._active.remove(r)
        r.evicted, r.ok, r.done, r.solver = int(beat), False, t, None
        return r.bytes_reserved

    def _complete(self, item, base, start):
        """A chunk has completed: record beat ends, check for divergence, call on_beat, finish the requests it
        ended; returns the bytes those requests release."""
        ev, snap = item
        ev.synchronize()
        t = base + start.elapsed_time(ev) / 1e3
        freed = 0.0
        for r, steps in snap:
            if r.evicted is not None:
                continue
            if steps % self.steps_per_beat == 0:
                r.beat_end.append(t)
                torch.cuda.nvtx.mark(f"request {r.id} beat {steps // self.steps_per_beat} done")
                if self.log is not None:
                    lat = r.beat_latencies()[-1]
                    self.log({"request": r.id, "beat": steps // self.steps_per_beat, "t_s": t, "latency_s": lat,
                              "nodes": r.N, "mlups": r.N * self.steps_per_beat / max(lat, 1e-12) / 1e6})
                if steps < r.steps_total:
                    beat = steps // self.steps_per_beat
                    if not self._finite(r):
                        freed += self._evict(r, beat, t)
                        continue
                    if self.on_beat is not None:
                        self.on_beat(r, beat)
            if steps >= r.steps_total:
                self._finish(r, t)
                freed += r.bytes_reserved
        return freed

    def _drain(self, inflight, base, start, active):
        while inflight:
            self._used -= self._complete(inflight.popleft(), base, start)

    def serve(self, specs, realtime=True):
        """Serve the requests (arrival times in seconds from now when realtime, else all queued at once, in
        arrival order) -> list of `Request` in arrival order, with timings and results."""
        reqs = sorted((Request(s) for s in specs), key=lambda r: r.arrival)
        if not realtime:
            for r in reqs:
                r.arrival = 0.0
        self.trace = []
        pending = collections.deque(reqs)
        queue = collections.deque()
        active = []
        inflight = collections.deque()     # (event, [(request, steps enqueued after this chunk)])
        self._used = 0.0
        batch = None
        self._batch, self._active = None, active
        self._side = torch.cuda.Stream(self.device)
        t0 = time.perf_counter()
        start = None
        while pending or queue or active or inflight:
            now = time.perf_counter() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                queue.append(pending.popleft())
            # admission: FIFO, while a slot is free and the estimate fits the budget
            while queue and len(active) < self.max_active:
                r = queue[0]
                need = self.estimate(r.spec)
                if self._used + need > self.budget:
                    if not active and not inflight:
                        raise RuntimeError(f"request {r.id} needs ~{need / 1e9:.1f} GB, over the "
                                           f"{self.budget / 1e9:.1f} GB budget")
                    break
                queue.popleft()
                if batch is None:
                    batch = self._batch = BatchSolver(block=self.block, schedule=self.schedule)
                self._admit(r, batch, t0)
                if start is None:
                    start = torch.cuda.Event(enable_timing=True)
                    start.record(batch.stream)
                    base = time.perf_counter() - t0
                self._used += max(need, r.bytes)
                r.bytes_reserved = max(need, r.bytes)
                active.append(r)
                self.trace.append((r.admit, len(active), self._used))
            if active and self.on_beat is not None and inflight and any(
                    0 < r.steps_enq < r.steps_total and r.steps_enq % self.steps_per_beat == 0 for r in active):
                # a member has just been given its beat's last chunk: let it finish, so that on_beat sees the beat's
                # final state and what it changes applies from the next beat's first step (simulate.py:330-337)
                self._drain(inflight, base, start, active)
            if active and batch.members:
                # an NVTX range per scheduling round (members, steps) for a timeline profiler
                with torch.cuda.nvtx.range(f"serve chunk: {len(active)} requests x {self.chunk} steps"):
                    batch.run(self.chunk, chunk=self.graph_chunk)
                snap = []
                for r in active:
                    r.steps_enq += self.chunk
                    snap.append((r, r.steps_enq))
                    if r.steps_enq % self.steps_per_beat == 0 and r.steps_enq < r.steps_total:
                        self._flag_beat(batch, r)
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(batch.stream)
                inflight.append((ev, snap))
                for r in [r for r in active if r.steps_enq >= r.steps_total]:
                    batch.remove(r.solver, sync=False)
                    active.remove(r)
            # completed chunks: beat ends, finished requests (their buffers are final once the event has passed)
            while inflight and (len(inflight) > self.ahead or not active or inflight[0][0].query()):
                self._used -= self._complete(inflight.popleft(), base, start)
                if not active:
                    break
            if not active and not inflight and not queue and pending and realtime:
                time.sleep(max(0.0, min(0.05, pending[0].arrival - (time.perf_counter() - t0))))
        del batch
        self._batch = self._active = None
        return reqs


def recalibrate_on_beat(r, beat):
    """Server on_beat hook for requests built by workloads.calibrated_builder: the lumped circuit recalibrated from
    the beat's mean inlet pressure and inflow, its new inlet pressure driving the next beat (simulate.py:330-337)."""
    r.solver.calibration.on_beat(beat)


def summary(reqs, steps_per_beat):
    """p50 / p99 of the per-beat latency and of the queue wait, and aggregate MLUPS over the whole stream."""
    lat = np.array([x for r in reqs for x in r.beat_latencies()])
    evicted = [r.id for r in reqs if r.evicted is not None]
    wait = np.array([r.queue_wait for r in reqs])
    lu = sum(r.N * (r.beats if r.evicted is None else r.evicted) * steps_per_beat for r in reqs)
    t_first = min(r.arrival for r in reqs)
    t_last = max(r.done for r in reqs)
    return {"requests": len(reqs), "beats": int(lat.size), "lattice_updates": float(lu),
            "beat_latency_p50_s": float(np.percentile(lat, 50)), "beat_latency_p99_s": float(np.percentile(lat, 99)),
            "queue_wait_p50_s": float(np.percentile(wait, 50)), "queue_wait_p99_s": float(np.percentile(wait, 99)),
            "makespan_s": float(t_last - t_first), "mlups": float(lu / max(t_last - t_first, 1e-9) / 1e6),
            "all_ok": bool(all(r.ok for r in reqs)), "evicted": evicted}


def one_by_one(specs, storage="f32", steps_per_beat=8000, graph_chunk=200, block=None, device=None,
               builder=default_builder, order="c"):
    """The same requests run one after another, each on its own dedicated solver (plain form): total seconds,
    lattice updates and MLUPS, builds included as in the served stream."""
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    lu = 0.0
    ok = True
    for sp in sorted(specs, key=lambda s: s.get("arrival", 0.0)):
        s = builder(sp, storage, block, device, steps_per_beat, order)
        steps = int(sp["beats"]) * steps_per_beat
        s.run(steps, chunk=graph_chunk)
        ok &= s.ok()
        s.fields()
        lu += s.N * steps
        del s
    torch.cuda.synchronize(device)
    dt = time.perf_counter() - t0
    return {"seconds": dt, "lattice_updates": lu, "mlups": lu / dt / 1e6, "all_ok": bool(ok)}
