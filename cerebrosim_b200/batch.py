"""Many vessels in one launch: `BatchSolver` advances several `lbm.Solver` / `ArterySolver` instances together.

The reference runs one simulation per GPU process and scales out with a Slurm job array of one-GPU jobs
(slurm/submit_all.sh:21,36-38, slurm/config.sh:20); small vessels then leave most of a B200 idle. Here the
instances' node lists are concatenated into one work list and one persistent launch per kernel and step covers up
to 64 of them (csrc/step.cu, `cs_batch_step`): each block takes work items — a bulk block or a boundary block of
some instance — and reads that instance's descriptor (buffers, clock, drive, outlet pressures, coupling) from the
kernel's parameters. The arithmetic of every instance is the single-lattice kernels' own, so an instance evolves
exactly as it would alone.

Instances may join and leave between runs (continuous batching): each keeps its own buffer parity, and the batch
descriptor table is rebuilt when the membership or an instance's parameters change.

Two schedules advance the members, with the same results (each instance's steps are the same arithmetic on its own
buffers either way):
- "fused": every step is one batched launch per kernel over all members (above);
- "by-instance": each member advances a whole `run` with its own single-lattice kernels and graphs, one member after
  the other on the batch stream. A member whose working set fits in the L2 then keeps it there from step to step,
  where the fused launches stream every member's populations through the L2 at every step;
- "concurrent:K": the members split into K groups of about equal node counts, each group by instance on a stream of
  its own, the K streams at once: a small member's kernels (a grid of a wave or two) then share the GPU with another
  group's instead of leaving SMs idle at every step's tail.
`autotune.tune_schedule` chooses among them by measurement.
"""
import ctypes

import torch

from . import _lib
from ._lib import check
from .lbm import ctypes_void

MAX_GROUPS = 64          # launch groups of CS_BATCH_GROUP instances: up to 4096 instances per batch
# steps per CUDA graph of the fused schedule at most: each of its launches carries its group's 22 KB descriptor
# table as kernel parameters, so a graph holds ~66 KB of parameters per step and group
FUSED_GRAPH_MAX = 400
SCHEDULES = ("fused", "by-instance", "concurrent:2", "concurrent:4", "concurrent:8")


class BatchSolver:
    """Advance `solvers` (same device, storage format, collision model and Galilean setting) together.

    block: threads per bulk block for every member (their flux partitions are rebuilt to match).
    persistent: size the grids to the GPU (SMs x resident blocks) and loop over work items, instead of one block
    per work item. schedule: "fused" or "by-instance" (module docstring)."""

    def __init__(self, solvers=(), block=128, persistent=True, device=None, schedule="fused"):
        if schedule not in SCHEDULES and not schedule.startswith("concurrent:"):
            raise ValueError(f"schedule {schedule!r}: one of {SCHEDULES}")
        self.members = []
        self.block = int(block)
        self.persistent = bool(persistent)
        self.schedule = schedule
        self.dev = None
        self.cur = 0
        self.steps = 0
        self.graphs = {}
        self._parity = []
        self._key = None
        self.stream = None
        for s in solvers:
            self.add(s)

    # --- membership
    def add(self, s):
        """Join an instance; it continues from its own state and step count."""
        if self.dev is None:
            self.dev = s.dev
            self.stream = torch.cuda.Stream(self.dev)
        if s.dev != self.dev:
            raise ValueError("all instances of a batch must be on one device")
        if self.members:
            m0 = self.members[0]
            if (s.storage, s.model, s.gal) != (m0.storage, m0.model, m0.gal):
                raise ValueError("instances of a batch share the storage format, collision model and Galilean setting")
        if s.block != self.block:
            s.block = self.block
            if hasattr(s, "_set_flux_blocks"):
                s._set_flux_blocks()
            s._drop_graphs()
        self.members.append(s)
        self._parity.append(s.cur ^ self.cur)
        self._key = None

    def remove(self, s, sync=True):
        """Leave the batch; the instance keeps its state and can run alone or join another batch.
        sync=False returns at once: steps already enqueued still update the instance, so its buffers must stay
        alive, and its fields are final only after the batch stream has passed them (a serving loop tracks that
        with events)."""
        k = self.members.index(s)
        if sync:
            self.stream.synchronize()
        del self.members[k]
        del self._parity[k]
        self._key = None

    # --- descriptor table
    def _drop_graphs(self):
        lib = _lib.load()
        for g in self.graphs.values():
            lib.cs_graph_destroy(g)
        self.graphs = {}

    def _refresh(self):
        """(Re)build the batch descriptor when members or their parameters changed. The instances' descriptors
        are host arrays the library copies into the kernels' parameters at every launch or capture."""
        descs = [m._desc() for m in self.members]
        raw = b"".join(bytes(d) for d in descs)
        key = (raw, tuple(self._parity))
        if key == self._key:
            return
        self._drop_graphs()
        n = len(self.members)
        self._descs = (_lib.StepDesc * n)(*descs)
        self._par = (ctypes.c_int32 * n)(*self._parity)
        if n > MAX_GROUPS * _lib.BATCH_GROUP:
            raise ValueError(f"{n} instances: at most {MAX_GROUPS * _lib.BATCH_GROUP} per batch")
        if getattr(self, "_counter", None) is None:
            # allocated once: graphs still in flight after a membership change keep using it
            with torch.cuda.device(self.dev):
                self._counter = torch.zeros(MAX_GROUPS, dtype=torch.int32, device=self.dev)
        m0 = self.members[0]
        b = _lib.BatchDesc()
        b.n_inst = n
        b.storage, b.model, b.gal = _lib.STORE[m0.storage], m0.model, m0.gal
        b.force = int(any(any(x != 0.0 for x in m.force) for m in self.members))
        b.any_open = int(any(getattr(m, "n_open", 0) > 0 for m in self.members))
        b.block = self.block
        sms = torch.cuda.get_device_properties(self.dev).multi_processor_count
        # the bulk kernel keeps 1024 threads resident per SM (64 registers each): 4 blocks of 256, 8 of 128
        b.grid_bulk = sms * max(1, 1024 // self.block) if self.persistent else 0
        b.grid_bnd = sms * 16 if self.persistent else 0          # 16 boundary blocks per SM (2 waves of 8)
        b.descs = ctypes.addressof(self._descs)
        b.parity = ctypes.addressof(self._par)
        b.counter = self._counter.data_ptr()
        self.desc = b
        self._key = key

    # --- stepping
    def _sync_in(self):
        self.stream.wait_stream(torch.cuda.current_stream(self.dev))
        for m in self.members:
            self.stream.wait_stream(m.stream)

    def _sync_out(self):
        torch.cuda.current_stream(self.dev).wait_stream(self.stream)
        for m in self.members:
            m.stream.wait_stream(self.stream)

    def prepare(self, chunk):
        """Capture the CUDA graphs a later `run(k * chunk, chunk=chunk)` replays (a whole heartbeat per graph, for
        instance), so that the capture happens before a timed region rather than inside it."""
        chunk += chunk % 2
        if not self.members:
            return
        if self.schedule == "fused":
            chunk = min(chunk, FUSED_GRAPH_MAX)
            self._refresh()
            key = (self.cur, chunk)
            if key not in self.graphs:
                lib = _lib.load()
                g = ctypes.c_void_p()
                self._sync_in()
                with torch.cuda.device(self.dev), torch.cuda.stream(self.stream):
                    check(lib.cs_batch_graph_capture(ctypes.byref(self.desc), self.cur, chunk,
                                                     ctypes_void(self.stream.cuda_stream), ctypes.byref(g)))
                self.graphs[key] = g
        else:
            for m in self.members:
                m.prepare(chunk)

    def run(self, steps, chunk=200):
        """Advance every member `steps` steps (CUDA graphs of `chunk` batched steps; chunk even)."""
        if not self.members:
            return
        if self.schedule == "by-instance":
            return self._run_by_instance(steps, chunk)
        if self.schedule.startswith("concurrent"):
            return self._run_concurrent(steps, chunk, int(self.schedule.split(":")[1]))
        self._refresh()
        lib = _lib.load()
        chunk += chunk % 2
        chunk = min(chunk, FUSED_GRAPH_MAX)
        full, rest = divmod(int(steps), chunk)
        self._sync_in()
        sp = ctypes_void(self.stream.cuda_stream)
        with torch.cuda.device(self.dev), torch.cuda.stream(self.stream):
            if full:
                key = (self.cur, chunk)
                if key not in self.graphs:
                    g = ctypes.c_void_p()
                    check(lib.cs_batch_graph_capture(ctypes.byref(self.desc), self.cur, chunk, sp, ctypes.byref(g)))
                    self.graphs[key] = g
                for _ in range(full):
                    check(lib.cs_graph_launch(self.graphs[key], sp))
            if rest:
                check(lib.cs_batch_step(ctypes.byref(self.desc), self.cur, rest, sp))
                if rest % 2:
                    self.cur = 1 - self.cur
        self._sync_out()
        self.steps += int(steps)
        for m, p in zip(self.members, self._parity):
            m.cur = self.cur ^ p
            m.steps += int(steps)

    def _run_by_instance(self, steps, chunk):
        """Each member's `run` in turn with the batch stream current: `Solver.run` makes its own stream wait for
        the current one and the current one for its own, so the members run one after the other, in order."""
        self._sync_in()
        with torch.cuda.device(self.dev), torch.cuda.stream(self.stream):
            for m in self.members:
                m.run(steps, chunk=chunk)          # advances m.cur and m.steps itself
        self._sync_out()
        self.steps += int(steps)
        if int(steps) % 2:
            self.cur = 1 - self.cur

    def _run_concurrent(self, steps, chunk, k):
        """Groups of members of about equal node counts (largest first into the lightest group), each group by
        instance on its own stream, the streams concurrently; the batch stream then waits for all of them."""
        k = max(1, min(k, len(self.members)))
        if len(getattr(self, "_streams", [])) < k:
            self._streams = [torch.cuda.Stream(self.dev) for _ in range(k)]
        groups, load = [[] for _ in range(k)], [0] * k
        for m in sorted(self.members, key=lambda m: -m.N):
            j = load.index(min(load))
            groups[j].append(m)
            load[j] += m.N
        self._sync_in()
        with torch.cuda.device(self.dev):
            for st, grp in zip(self._streams, groups):
                st.wait_stream(self.stream)
                with torch.cuda.stream(st):
                    for m in grp:
                        m.run(steps, chunk=chunk)
            for st in self._streams[:k]:
                self.stream.wait_stream(st)
        self._sync_out()
        self.steps += int(steps)
        if int(steps) % 2:
            self.cur = 1 - self.cur

    def synchronize(self):
        self.stream.synchronize()

    @property
    def nodes(self):
        return sum(m.N for m in self.members)

    def __del__(self):
        try:
            self._drop_graphs()
        except Exception:
            pass
