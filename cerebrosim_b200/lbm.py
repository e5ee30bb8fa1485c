"""Drop-in replacement for CerebroSim's `lbm` module (lbm.py), running on a B200 through libcerebrosim_b200.so.

Same public surface as the reference: `LATTICE, C, W, Q, OPP, WALL, INLET, OUTLET0` (lbm.py:33-58), `Units`
(lbm.py:63-82), `build_lattice` (lbm.py:264-330), `scatter` (lbm.py:333-338) and `Solver` (lbm.py:346-455) with
`set_drive`, `set_force`, `set_sponge`, `set_outlet_pressure`, `run`, `fields`, `ok` and the `_launch(a)` hook.
State lives in PyTorch CUDA tensors; every step is one hand-written sm_100a kernel (csrc/step.cu) and runs of steps
are CUDA graphs, as in the reference. There is no CPU path: without a CUDA device or the library, construction
raises.

Differences a caller can see:
  - only D3Q27 (the reference's default; ARTERY_LBM_LATTICE=D3Q19 raises ValueError);
  - `Solver(..., storage="f32" | "f16" | "bf16", block=None, order="c")`: population storage format, threads per
    block and the internal node order (fields are returned in the lattice's order whatever it is);
  - `vels[k]` is an (N, 3) view of a (3, N) structure-of-arrays buffer; `fields()` returns NumPy copies as before.
"""
import ctypes
import os

import numpy as np
import torch

from . import _lib
from ._lib import check

LATTICE = os.environ.get("ARTERY_LBM_LATTICE", "D3Q27")
if LATTICE != "D3Q27":
    raise ValueError(f"ARTERY_LBM_LATTICE={LATTICE}: this package implements D3Q27 only")

# lbm.py:34-47
C = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
              [1, 1, 0], [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1], [1, 0, -1], [-1, 0, 1],
              [0, 1, 1], [0, -1, -1], [0, 1, -1], [0, -1, 1],
              [1, 1, 1], [-1, -1, -1], [1, 1, -1], [-1, -1, 1], [1, -1, 1], [-1, 1, -1], [-1, 1, 1], [1, -1, -1]],
             np.int32)
W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
Q = len(C)
OPP = np.array([int(np.flatnonzero((C == -c).all(1))[0]) for c in C], np.int32)
WALL, INLET, OUTLET0 = -1, -2, -3
SEG_STRIDE = 28          # words per row of the compressed connectivity's segment table (CS_SEG_STRIDE)


class Units:
    """Physical <-> lattice units for spacing dx (m), step dt (s), density rho (kg/m^3), viscosity nu (m^2/s)."""

    def __init__(self, dx, dt, rho, nu):
        self.dx, self.dt, self.rho, self.nu = dx, dt, rho, nu
        self.nu_lu = nu * dt / dx ** 2
        self.tau = 3.0 * self.nu_lu + 0.5
        self.c = dx / dt

    def u(self, u_lu):
        return np.asarray(u_lu) * self.c

    def u_lu(self, u):
        return np.asarray(u) / self.c

    def p(self, p_lu):
        return np.asarray(p_lu) * self.rho * self.c ** 2

    def p_lu(self, p):
        return np.asarray(p) / (self.rho * self.c ** 2)


def _device(device=None):
    if not torch.cuda.is_available():
        raise RuntimeError("cerebrosim_b200 needs a CUDA device (there is no CPU fallback)")
    if device is None:
        return torch.device("cuda", torch.cuda.current_device())
    d = torch.device(device)
    if d.type != "cuda":
        raise ValueError(f"device {device!r}: cerebrosim_b200 runs on CUDA devices only")
    return torch.device("cuda", d.index if d.index is not None else torch.cuda.current_device())


def ctypes_void(x):
    return ctypes.c_void_p(int(x))


class Lattice(dict):
    """build_lattice's result: the reference's dict. When built with host=False its host tables (nbr, q, uin,
    coords) are copied from the device copies in "_dev" the first time they are read, so a caller that only hands
    the lattice to a Solver (which uses the device copies) never moves them."""

    _LAZY = ("nbr", "q", "uin", "coords")

    def __missing__(self, key):
        dev = dict.get(self, "_dev")
        if key in self._LAZY and isinstance(dev, dict) and key in dev:
            v = dev[key].cpu().numpy()
            self[key] = v
            return v
        raise KeyError(key)


def n_nodes(lat):
    """Fluid node count of a lattice, without reading its host tables."""
    dev = lat.get("_dev") if isinstance(lat.get("_dev"), dict) else None
    return int((dev if dev is not None else lat)["nbr"].shape[1])


def build_lattice(phi, origin, dx, openings=(), periodic=(), opening_slack=1.0, device=None, host=True):
    """Sparse lattice from a signed distance on grid nodes (negative = fluid), built on the GPU (lbm.py:264-330).

    Returns the reference's dict of NumPy arrays (nbr (Q, N) int32, q (Q, N) float32, uin (N, 3) float32,
    coords (N, 3) int32, origin, dx, shape, n_outlets, counts, openings), bit-identical to lbm.build_lattice, plus
    "_dev": the same tables as CUDA tensors, which `Solver` reuses instead of uploading them again. host=False: the
    four host tables are copied from "_dev" only when first read (`Lattice`)."""
    lib = _lib.load()
    if isinstance(phi, torch.Tensor) and phi.is_cuda:   # a field already on the device (vessel.sdf_grid)
        dev = _device(phi.device if device is None else device)
        phi_h = None
        shape = tuple(int(s) for s in phi.shape)
    else:
        dev = _device(device)
        phi_h = np.ascontiguousarray(np.asarray(phi, np.float32))
        shape = phi_h.shape
    if len(shape) != 3:
        raise ValueError(f"phi must be 3-D, got shape {shape}")
    nx, ny, nz = shape
    origin_a = np.asarray(origin, float)
    mask = 0
    for a in periodic:
        if a not in (0, 1, 2):
            raise ValueError(f"periodic axis {a}")
        mask |= 1 << int(a)
    ops = list(openings)
    carr = (_lib.Opening * max(1, len(ops)))()
    for k, o in enumerate(ops):
        if o["kind"] not in ("inlet", "outlet"):
            raise ValueError(f"opening kind {o['kind']!r}")
        carr[k].kind = 0 if o["kind"] == "inlet" else 1
        c, nrm = np.asarray(o["centre"], float), np.asarray(o["normal"], float)
        for a in range(3):
            carr[k].centre[a] = float(c[a])
            carr[k].normal[a] = float(nrm[a])
        carr[k].radius = float(o["radius"])
    inlets = [o for o in ops if o["kind"] == "inlet"]
    outlets = [o for o in ops if o["kind"] == "outlet"]
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev)
        sp = ctypes.c_void_p(stream.cuda_stream)
        phi_d = (torch.from_numpy(phi_h).to(dev) if phi_h is not None
                 else phi.to(dev, torch.float32).contiguous())
        scratch = torch.empty(max(1, int(lib.cs_lattice_scratch_bytes(nx, ny, nz))), dtype=torch.uint8, device=dev)
        n_fluid = ctypes.c_int64(0)
        check(lib.cs_lattice_count(ctypes.c_void_p(phi_d.data_ptr()), nx, ny, nz,
                                   ctypes.c_void_p(scratch.data_ptr()), ctypes.byref(n_fluid), sp))
        N = n_fluid.value
        nbr = torch.empty((Q, N), dtype=torch.int32, device=dev)
        q = torch.empty((Q, N), dtype=torch.float32, device=dev)
        uin = torch.empty((N, 3), dtype=torch.float32, device=dev)
        coords = torch.empty((N, 3), dtype=torch.int32, device=dev)
        counts = torch.empty(2 + len(outlets), dtype=torch.int64, device=dev)
        org = (ctypes.c_double * 3)(*origin_a.reshape(3).tolist())

        def ptr(t):
            return ctypes.c_void_p(t.data_ptr() if t.numel() else 0)
        check(lib.cs_lattice_fill(ctypes.c_void_p(phi_d.data_ptr()), nx, ny, nz, org, float(dx), carr, len(ops),
                                  mask, float(opening_slack), ctypes.c_void_p(scratch.data_ptr()), N, ptr(nbr),
                                  ptr(q), ptr(uin), ptr(coords), ptr(counts), sp))
        stream.synchronize()
        del scratch, phi_d
    cnt = counts.cpu().numpy()
    lat = Lattice(origin=origin_a, dx=dx, shape=shape, n_outlets=len(outlets),
                  counts={"wall": int(cnt[0]), "inlet": int(cnt[1]), "outlet": [int(x) for x in cnt[2:]]},
                  openings=inlets + outlets, _dev={"nbr": nbr, "q": q, "uin": uin, "coords": coords})
    if host:
        for k in Lattice._LAZY:
            lat[k]
    return lat


def scatter(lat, values, fill=np.nan):
    """Per-cell values -> dense grid (`fill` outside the fluid), lbm.py:333-338."""
    values = np.asarray(values)
    out = np.full(tuple(lat["shape"]) + values.shape[1:], fill, values.dtype if values.dtype.kind == "f" else float)
    out[tuple(lat["coords"].T)] = values
    return out


def sponge_tau(lat, tau, length, tau_max, kinds=("inlet", "outlet")):
    """Per-cell tau raised smoothly towards the openings of the given kinds (lbm.py:398-416): tau_max at the
    opening plane, back to tau at `length` cells inside, within 1.5 radii of the opening's axis."""
    pos = lat["origin"] + lat["coords"] * lat["dx"]
    out = np.full(len(lat["coords"]), tau)
    for o in lat["openings"]:
        if o["kind"] not in kinds:
            continue
        c, nrm = np.asarray(o["centre"], float), np.asarray(o["normal"], float)
        rel = pos - c
        along = rel @ nrm
        depth = -along / lat["dx"]
        near = np.linalg.norm(rel - along[:, None] * nrm, axis=1) < 1.5 * o["radius"]
        w = np.clip(1.0 - depth / length, 0.0, 1.0)
        w = w * w * (3.0 - 2.0 * w)
        out = np.maximum(out, np.where(near, tau + (tau_max - tau) * w, tau))
    return out


def _upload(x, dtype, dev):
    """Host table -> device: torch tensors (e.g. pinned) are copied asynchronously, NumPy arrays as they are."""
    if isinstance(x, torch.Tensor):
        return x.to(dev, dtype=dtype, non_blocking=True).contiguous()
    np_dtype = {torch.int32: np.int32, torch.float32: np.float32}[dtype]
    return torch.as_tensor(np.ascontiguousarray(x, np_dtype)).to(dev)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else None


class Solver:
    """Sparse D3Q27 lattice Boltzmann on one GPU (lbm.py:346-455). tau from the lattice viscosity; model "trt"
    (magic = Lambda) or "regularised"; sigma < 1 blends the regularised stress with the finite-difference one.

    storage: "f32" (the reference's FP32 populations), "f16" or "bf16" (16-bit shifted populations, FP32
    arithmetic). FP16 keeps velocity and wall shear stress within 1 % of an FP64 run over two beats of the 1.57 M-node
    artery; BF16's 8-bit mantissa does not (about 11 % and 12 %, and the pressure drop is lost) and suits small or
    short runs only. block: threads per block (None: the tuned default). order: internal node numbering (see
    node_order); fields() always return the lattice's order, while the state tensors (rho, vel, f) are in the
    internal one."""

    def __init__(self, lat, nu_lu, magic=3.0 / 16.0, bouzidi=True, model="trt", sigma=1.0, galilean=None,
                 device=None, storage="f32", block=None, order="c"):
        lib = _lib.load()
        self.dev = _device(device)
        self.lat = lat
        self.N = N = n_nodes(lat)
        # the axis and split orders are found on the device once the tables are there (a host pass over the 27 x N
        # table, or a host sort of the coordinates, would cost more than the rest of the construction)
        on_device = order in _DEVICE_ORDERS
        perm = None if on_device else node_order(lat, order)
        self.order = order
        self.tau = 3.0 * nu_lu + 0.5
        self.magic = float(magic)
        self.bouzidi = int(bool(bouzidi))
        self.model = {"trt": 0, "regularised": 1}[model]
        self.sigma = float(sigma)
        self.gal = int(LATTICE == "D3Q27" if galilean is None else bool(galilean))
        if storage not in _lib.STORE:
            raise ValueError(f"storage {storage!r}: use one of {sorted(_lib.STORE)}")
        self.storage = storage
        self.block = int(block) if block else default_block(N)
        if self.block < 32 or self.block > 256 or self.block % 32:
            raise ValueError(f"block {self.block}: a multiple of 32 in 32..256")
        pop_dtype = {"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16}[storage]
        with torch.cuda.device(self.dev):
            # set-up (uploads, table kernels, allocations) runs on the caller's stream, so that the caching
            # allocator serves a Solver built after another one freed its tensors from the same pool; the steps
            # run on a private stream, ordered after the set-up, and every tensor the steps use is recorded on it
            self.stream = torch.cuda.Stream(self.dev)
            setup = torch.cuda.current_stream(self.dev)
            sp = ctypes_void(setup.cuda_stream)
            dev = self.dev
            tabs = lat.get("_dev") if isinstance(lat.get("_dev"), dict) else None
            side = None
            if tabs is not None and tabs["nbr"].device == dev:
                nbr, q, uin = tabs["nbr"], tabs["q"], tabs["uin"]
            elif all(isinstance(lat[k], torch.Tensor) for k in ("nbr", "q", "uin")):
                # host tensors (pinned: asynchronous copies): q and uin cross PCIe on a side stream while the work
                # that needs only nbr (renumbering, the ghost count) runs; the set-up waits for them before use
                nbr = _upload(lat["nbr"], torch.int32, dev)
                q = torch.empty(tuple(lat["q"].shape), dtype=torch.float32, device=dev)
                uin = torch.empty(tuple(lat["uin"].shape), dtype=torch.float32, device=dev)
                side = torch.cuda.Stream(dev)
                side.wait_stream(setup)
                with torch.cuda.stream(side):
                    q.copy_(lat["q"], non_blocking=True)
                    uin.copy_(lat["uin"], non_blocking=True)
            else:
                nbr = _upload(lat["nbr"], torch.int32, dev)
                q = _upload(lat["q"], torch.float32, dev)
                uin = _upload(lat["uin"], torch.float32, dev)
            self.perm = self.inv = None
            if on_device and N:
                perm = _device_order(lat, nbr, order, dev)
            if perm is not None:
                # internal node k is the lattice's node perm[k]; sources renumbered through inv
                self.perm = perm if isinstance(perm, torch.Tensor) else torch.as_tensor(perm.astype(np.int64)).to(dev)
                self.inv = torch.empty_like(self.perm)
                self.inv[self.perm] = torch.arange(N, device=dev)
                src = nbr[:, self.perm]
                nbr = torch.where(src >= 0, self.inv[src.clamp(min=0)].to(torch.int32), src).contiguous()
            self.inl = (nbr == INLET).any(0).to(torch.int32) if N else torch.zeros(0, dtype=torch.int32, device=dev)
            n_out = max(1, int(lat["n_outlets"]))
            # step link tables: fluid pull sources, and a ghost slot per boundary link (csrc/links.cu)
            scratch = torch.empty(max(1, int(lib.cs_links_scratch_bytes(N))), dtype=torch.uint8, device=dev)
            ghosts = (ctypes.c_int64 * Q)()
            check(lib.cs_links_count(_ptr(nbr), N, _ptr(scratch), ghosts, sp))
            if side is not None:
                setup.wait_stream(side)
            if self.perm is not None:
                q = q[:, self.perm].contiguous()
                uin = uin[self.perm]
            self.uin = uin.contiguous()
            self.ghosts = [int(x) for x in ghosts]
            self.gmax = max(self.ghosts) if N else 0
            self.npad = N + self.gmax
            gcols = max(1, self.gmax)
            self.links = torch.empty((Q, N), dtype=torch.int32, device=dev)
            self.gnode = torch.full((Q, gcols), -1, dtype=torch.int32, device=dev)
            self.ginfo = torch.full((Q, gcols), WALL, dtype=torch.int32, device=dev)
            self.gq = torch.full((Q, gcols), -1.0, dtype=torch.float32, device=dev)
            status = torch.empty(2, dtype=torch.int64, device=dev)
            check(lib.cs_links_fill(_ptr(nbr), _ptr(q), N, n_out, self.gmax, _ptr(scratch), _ptr(self.links),
                                    _ptr(self.gnode), _ptr(self.ginfo), _ptr(self.gq), _ptr(status), sp))
            del scratch
            # compressed connectivity (csrc/compress.cu): 4 bytes per regular node instead of 108
            scratch = torch.empty(max(1, int(lib.cs_compress_scratch_bytes(N))), dtype=torch.uint8, device=dev)
            n_seg, n_irr = ctypes.c_int64(0), ctypes.c_int64(0)
            check(lib.cs_compress_count(_ptr(self.links), N, _ptr(scratch), ctypes.byref(n_seg),
                                        ctypes.byref(n_irr), sp))
            self.n_seg, self.n_irr = int(n_seg.value), int(n_irr.value)
            self.lcode = torch.empty(max(1, N), dtype=torch.int32, device=dev)
            self.segdelta = torch.empty((max(1, self.n_seg), SEG_STRIDE), dtype=torch.int32, device=dev)
            self.irr = torch.empty((Q, max(1, self.n_irr)), dtype=torch.int32, device=dev)
            assert self.segdelta.numel() >= self.n_seg * SEG_STRIDE and self.irr.numel() >= self.n_irr * Q
            assert self.segdelta.data_ptr() % 16 == 0   # rows are read with 128-bit loads
            check(lib.cs_compress_fill(_ptr(self.links), N, self.n_seg, self.n_irr, _ptr(scratch),
                                       _ptr(self.lcode), _ptr(self.segdelta), _ptr(self.irr), sp))
            setup.synchronize()
            del scratch
            self.links = None                          # the full 27 x N table is not needed by the step
            self.f = [torch.zeros((Q, self.npad), dtype=pop_dtype, device=dev) for _ in range(2)]
            self.vel = [torch.zeros((3, N), dtype=torch.float32, device=dev) for _ in range(2)]
            self.vels = [v.T for v in self.vel]
            self.rho = torch.zeros(N, dtype=torch.float32, device=dev)
            self.p_out = torch.zeros(n_out, dtype=torch.float32, device=dev)
            self.p_out64 = torch.zeros(n_out, dtype=torch.float64, device=dev)
            # 1 / tau per node, negated on cells with an inlet link (the kernel's inlet-cell flag)
            self._om_sign = 1.0 - 2.0 * self.inl.to(torch.float32)
            self.om = torch.full((N,), 1.0 / self.tau, dtype=torch.float32, device=dev) * self._om_sign
            self.tick = torch.zeros(2, dtype=torch.int32, device=dev)
            self.drv = torch.zeros(1, dtype=torch.float32, device=dev)
            for t in (self.perm, self.inv, self.uin, self.inl, self.gnode, self.ginfo, self.gq, self.lcode,
                      self.segdelta, self.irr, *self.f, *self.vel, self.rho, self.p_out, self.p_out64,
                      self._om_sign, self.om, self.tick, self.drv):
                if t is not None:
                    t.record_stream(self.stream)
            self.stream.wait_stream(setup)
        self.force = (0.0, 0.0, 0.0)
        self.graphs = {}
        self.set_drive([1.0])
        self.cur = 0
        self.steps = 0

    # --- inputs
    def set_drive(self, coef, period=1, ramp=0):
        """drive(t) = coef[0] + sum_k coef[2k-1] cos(2 pi k t / period) + coef[2k] sin(...), times a smooth start
        over `ramp` steps; scales the inlet profile and the body force (lbm.py:384-392)."""
        coef = np.asarray(coef, np.float32)
        if len(coef) % 2 == 0:
            coef = np.append(coef, 0.0).astype(np.float32)
        if int(period) < 1:
            raise ValueError(f"period {period}: at least 1 step")
        with torch.cuda.device(self.dev), torch.cuda.stream(self.stream):
            self.coef = torch.as_tensor(coef).to(self.dev)
        self.nh, self.period, self.ramp = (len(coef) - 1) // 2, int(period), int(ramp)
        self._drop_graphs()

    def set_force(self, F):
        self.force = tuple(float(np.float32(x)) for x in F)
        self._drop_graphs()

    def set_sponge(self, length, tau_max, kinds=("inlet", "outlet")):
        """Raise the viscosity smoothly towards the openings of the given kinds (lbm.py:398-416). Computed on the
        device (csrc/lattice_build.cu k_sponge) with the reference's float64 operations: the same per-cell tau as
        `sponge_tau`, which restates it on the host."""
        mask = (1 if "inlet" in kinds else 0) | (2 if "outlet" in kinds else 0)
        ops = list(self.lat["openings"])
        carr = (_lib.Opening * max(1, len(ops)))()
        for j, o in enumerate(ops):
            carr[j].kind = 0 if o["kind"] == "inlet" else 1
            c, nrm = np.asarray(o["centre"], float), np.asarray(o["normal"], float)
            for a in range(3):
                carr[j].centre[a] = float(c[a])
                carr[j].normal[a] = float(nrm[a])
            carr[j].radius = float(o["radius"])
        self._sponge = (carr, len(ops), mask, float(length), float(tau_max))
        with torch.cuda.device(self.dev):
            # on the caller's stream (temporaries from its pool), after the steps already enqueued
            cur = torch.cuda.current_stream(self.dev)
            cur.wait_stream(self.stream)
            om = self._sponge_eval(cur)
            if self.perm is not None:
                om = om[self.perm]
            self.om.copy_(om * self._om_sign)
            self.stream.wait_stream(cur)

    def _sponge_eval(self, stream, tau_out=None):
        """om = float32(1 / tau_cell) per cell (lattice order) of the last set_sponge, on `stream`."""
        carr, n_ops, mask, length, tau_max = self._sponge
        org = (ctypes.c_double * 3)(*np.asarray(self.lat["origin"], float).reshape(3).tolist())
        tabs = self.lat.get("_dev") if isinstance(self.lat.get("_dev"), dict) else {}
        coords = tabs.get("coords")
        if coords is None or coords.device != self.dev:
            coords = torch.as_tensor(np.ascontiguousarray(self.lat["coords"], np.int32)).to(self.dev)
        om = torch.empty(self.N, dtype=torch.float32, device=self.dev)
        check(_lib.load().cs_sponge_om(_ptr(coords), self.N, org, float(self.lat["dx"]), carr, n_ops, mask,
                                       float(self.tau), length, tau_max, _ptr(om), _ptr(tau_out),
                                       ctypes_void(stream.cuda_stream)))
        return om

    @property
    def tau_cell(self):
        """Relaxation time per cell (lattice order, float64 NumPy; lbm.py:366, 415), evaluated on request."""
        if getattr(self, "_sponge", None) is None:
            return np.full(self.N, self.tau)
        with torch.cuda.device(self.dev):
            cur = torch.cuda.current_stream(self.dev)
            tau = torch.empty(self.N, dtype=torch.float64, device=self.dev)
            self._sponge_eval(cur, tau)
            return tau.cpu().numpy()

    def set_outlet_pressure(self, p_lu):
        p = np.asarray(p_lu, np.float32).reshape(-1)
        with torch.cuda.device(self.dev), torch.cuda.stream(self.stream):
            self.p_out[:len(p)].copy_(torch.as_tensor(p).to(self.dev))
            self.p_out64[:len(p)].copy_(torch.as_tensor(p.astype(np.float64)).to(self.dev))

    # --- stepping
    def _desc(self):
        d = _lib.StepDesc()
        d.n, d.npad, d.gmax = self.N, self.npad, self.gmax
        run = 0
        for i in range(Q):                       # the boundary-link grid without padding blocks
            d.gblock[i] = run
            run += -(-self.ghosts[i] // 256)
        d.gblock[Q] = run
        d.gnode, d.ginfo, d.gq = self.gnode.data_ptr(), self.ginfo.data_ptr(), self.gq.data_ptr()
        d.storage = _lib.STORE[self.storage]
        d.model, d.bouzidi, d.gal = self.model, self.bouzidi, self.gal
        d.sigma, d.magic = self.sigma, self.magic
        for k in range(3):
            d.force[k] = self.force[k]
        d.block = self.block
        d.f[0], d.f[1] = self.f[0].data_ptr(), self.f[1].data_ptr()
        d.vel[0], d.vel[1] = self.vel[0].data_ptr(), self.vel[1].data_ptr()
        d.rho, d.uin, d.om = self.rho.data_ptr(), self.uin.data_ptr(), self.om.data_ptr()
        d.lcode, d.segdelta, d.irr, d.n_irr = (self.lcode.data_ptr(), self.segdelta.data_ptr(), self.irr.data_ptr(),
                                               max(1, self.n_irr))
        d.p_out, d.n_out = self.p_out.data_ptr(), len(self.p_out)
        d.tick, d.drive, d.coef = self.tick.data_ptr(), self.drv.data_ptr(), self.coef.data_ptr()
        d.nh, d.period, d.ramp = self.nh, self.period, self.ramp
        d.p_out64 = self.p_out64.data_ptr()
        self._fill_desc(d)
        return d

    def _fill_desc(self, d):
        """Hook for subclasses that add the outlet-resistance coupling."""
        d.n_open = 0

    def _launch(self, a):
        """One step reading buffer a and writing 1 - a (lbm.py:422-428)."""
        check(_lib.load().cs_step(ctypes.byref(self._desc()), int(a), 1, ctypes_void(self.stream.cuda_stream)))

    def _drop_graphs(self):
        lib = _lib.load()
        for g in getattr(self, "graphs", {}).values():
            if isinstance(g, torch.cuda.CUDAGraph):
                continue
            lib.cs_graph_destroy(g)
        self.graphs = {}

    def _capture(self, a, chunk):
        if type(self)._launch is Solver._launch:
            g = ctypes.c_void_p()
            check(_lib.load().cs_graph_capture(ctypes.byref(self._desc()), int(a), int(chunk),
                                               ctypes_void(self.stream.cuda_stream), ctypes.byref(g)))
            return g
        # a subclass extended _launch: capture its Python-level launches with torch's graph API
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=self.stream):
            for _ in range(chunk):
                self._launch(a)
                a = 1 - a
        return graph

    def _replay(self, g):
        if isinstance(g, torch.cuda.CUDAGraph):
            g.replay()
        else:
            check(_lib.load().cs_graph_launch(g, ctypes_void(self.stream.cuda_stream)))

    def prepare(self, chunk):
        """Capture the CUDA graph of `chunk` steps that the next `run(k * chunk, chunk=chunk)` replays (for a graph
        of a whole heartbeat, captured before a timed run); nothing is launched."""
        chunk += chunk % 2
        key = (self.cur, chunk)
        if key not in self.graphs:
            self.stream.wait_stream(torch.cuda.current_stream(self.dev))
            with torch.cuda.device(self.dev), torch.cuda.stream(self.stream):
                self.graphs[key] = self._capture(self.cur, chunk)

    def run(self, steps, chunk=200):
        """Advance `steps` steps (CUDA graphs of `chunk` steps; chunk even), lbm.py:430-448."""
        chunk += chunk % 2
        full, rest = divmod(int(steps), chunk)
        cur_stream = torch.cuda.current_stream(self.dev)
        self.stream.wait_stream(cur_stream)
        with torch.cuda.nvtx.range(f"Solver.run {steps} steps, {self.N} nodes"), torch.cuda.device(self.dev), \
                torch.cuda.stream(self.stream):
            if full:
                key = (self.cur, chunk)
                if key not in self.graphs:
                    self.graphs[key] = self._capture(self.cur, chunk)
                for _ in range(full):
                    self._replay(self.graphs[key])
            if rest and type(self)._launch is Solver._launch:
                # the leftover steps in one library call (the same launches, without a descriptor per step)
                check(_lib.load().cs_step(ctypes.byref(self._desc()), int(self.cur), int(rest),
                                          ctypes_void(self.stream.cuda_stream)))
                self.cur ^= rest & 1
            else:
                for _ in range(rest):
                    self._launch(self.cur)
                    self.cur = 1 - self.cur
        cur_stream.wait_stream(self.stream)
        self.steps += int(steps)

    def synchronize(self):
        self.stream.synchronize()

    def link_table(self):
        """The step's 27 x N pull-source table (nodes < N, ghost slots >= N), expanded from its compressed form."""
        links = torch.empty((Q, self.N), dtype=torch.int32, device=self.dev)
        with torch.cuda.device(self.dev), torch.cuda.stream(self.stream):
            check(_lib.load().cs_compress_expand(_ptr(self.lcode), _ptr(self.segdelta), _ptr(self.irr), self.N,
                                                 max(1, self.n_irr), _ptr(links),
                                                 ctypes_void(self.stream.cuda_stream)))
        self.stream.synchronize()
        return links

    def tick_value(self):
        """The device step counter (k_clock's tick): steps taken since construction."""
        self.stream.synchronize()
        return int(self.tick[self.cur].item())

    def fields(self):
        """(pressure, velocity) per cell of the lattice (its node order, whatever the internal one), lattice units,
        as NumPy (lbm.py:450-452)."""
        self.stream.synchronize()
        # on the caller's stream (the steps are done): its pool holds the construction's freed blocks
        with torch.cuda.device(self.dev):
            rho, vel = self.rho, self.vel[self.cur]
            if self.inv is not None:
                rho, vel = rho[self.inv], vel[:, self.inv]
            # the (3, N) buffer transposed on the device: the read-back is one contiguous copy, not a strided one on
            # the host; p = rho / 3 stays a host division, as the reference's
            u = vel.t().contiguous().cpu().numpy()
            p = rho.cpu().numpy()
        return p / 3.0, u

    # --- checkpoint / resume (the reference saves outputs only and restarts whole runs, README.md:144)
    _STATE = ("rho", "p_out", "p_out64", "tick", "drv", "coef", "om")

    def checkpoint(self):
        """The solver's evolving state as host tensors: the current populations (in their storage format, ghost
        slots included), the current velocity, density, clock, drive coefficients, outlet pressures and relaxation
        rates, and the step count. `restore` on a solver built from the same lattice and settings continues the run
        bit for bit."""
        self.stream.synchronize()
        st = {k: getattr(self, k).detach().cpu().clone() for k in self._STATE}
        # the two-slot clock: the restored solver reads buffer 0, so both slots carry the count of the next step
        st["tick"] = self.tick[self.cur].detach().cpu().repeat(2)
        st.update({"f": self.f[self.cur].detach().cpu().clone(), "vel": self.vel[self.cur].detach().cpu().clone(),
                   "steps": int(self.steps), "N": int(self.N), "storage": self.storage, "order": self.order,
                   "drive": (int(self.nh), int(self.period), int(self.ramp)), "force": tuple(self.force)})
        return st

    def restore(self, st):
        """Load a `checkpoint` taken on a solver of the same lattice, storage format and node order."""
        if (st["N"], st["storage"], st["order"]) != (self.N, self.storage, self.order):
            raise ValueError(f"checkpoint of {st['N']} nodes, {st['storage']}, order {st['order']}: this solver has "
                             f"{self.N}, {self.storage}, order {self.order}")
        if tuple(st["f"].shape) != tuple(self.f[0].shape):
            raise ValueError("checkpoint populations have another shape (different ghost slots)")
        with torch.cuda.device(self.dev), torch.cuda.stream(self.stream):
            self.cur = 0
            self.f[0].copy_(st["f"].to(self.dev))
            self.vel[0].copy_(st["vel"].to(self.dev))
            for k in self._STATE:
                if k == "coef":
                    self.coef = st["coef"].to(self.dev)
                else:
                    getattr(self, k).copy_(st[k].to(self.dev))
        self.nh, self.period, self.ramp = st["drive"]
        self.force = tuple(st["force"])
        self.steps = int(st["steps"])
        self._drop_graphs()
        self.stream.synchronize()

    def save(self, path):
        """Write a checkpoint to `path` (torch.save)."""
        torch.save(self.checkpoint(), path)

    def load(self, path):
        """Restore the checkpoint written by `save`."""
        self.restore(torch.load(path, weights_only=False))

    def ok(self):
        """All densities finite (lbm.py:454-455)."""
        self.stream.synchronize()
        return bool(torch.isfinite(self.rho).all().item())

    def __del__(self):
        try:
            self._drop_graphs()
        except Exception:
            pass


ORDERS = ("c", "axis", "morton", "split", "axis-split", "boundary-first", "axis-boundary-first")
# orders that separate the nodes with a boundary link from the others, and on which base order
_SPLITS = {"split": ("c", False), "axis-split": ("axis", False), "boundary-first": ("c", True),
           "axis-boundary-first": ("axis", True)}


_DEVICE_ORDERS = ("axis", "split", "axis-split", "boundary-first", "axis-boundary-first")


def _device_order(lat, nbr, order, dev):
    """node_order(lat, order) computed on the device from the (Q, N) table `nbr` already there (and the coordinates,
    uploaded if the lattice has no device copy): a CUDA int64 tensor, or None for the C order. The same permutation
    as the host's: the axis order's lexicographic key is one integer per node (coordinates are unique, so the sort
    has no ties), and the split orders are stable partitions."""
    N = int(nbr.shape[1])
    base = None
    if order.startswith("axis"):
        tabs = lat.get("_dev") if isinstance(lat.get("_dev"), dict) else {}
        c = tabs.get("coords")
        if c is None or c.device != dev:
            c = torch.as_tensor(np.ascontiguousarray(lat["coords"], np.int32)).to(dev)
        c = c.to(torch.int64)
        lo = c.min(0).values
        ext = c.max(0).values - lo
        fast = int(torch.argmax(ext).item())              # the first largest extent, as np.argmax
        s0, s1 = [a for a in (0, 1, 2) if a != fast]
        span = ext + 1
        key = ((c[:, s0] - lo[s0]) * span[s1] + (c[:, s1] - lo[s1])) * span[fast] + (c[:, fast] - lo[fast])
        base = torch.argsort(key)
    if order == "axis":
        perm = base
    else:
        bnd = (nbr < 0).any(0)
        if base is not None:
            bnd = bnd[base]
        parts = [torch.nonzero(~bnd).flatten(), torch.nonzero(bnd).flatten()]
        idx = torch.cat(parts[::-1] if _SPLITS[order][1] else parts)
        perm = idx if base is None else base[idx]
    if bool((perm == torch.arange(N, device=dev)).all()):
        return None
    return perm


def node_order(lat, order="c"):
    """Internal numbering of a lattice's nodes (internal node k = lattice node perm[k]); None for the lattice's own
    C order. "axis": C order with the axis of largest extent varying fastest (long runs along a vessel); "morton":
    Z-order curve of the grid coordinates; "split" / "axis-split": C / axis order with the nodes that have a
    boundary link moved after all others (so the boundary-link kernel reads consecutive nodes and the bulk
    kernel's warps are all plain or all boundary); "boundary-first" / "axis-boundary-first": the same with those
    nodes first, so that the bulk grid's slowest blocks (irregular connectivity, inlet cells) start first and the
    plain blocks fill its last wave."""
    if order not in ORDERS:
        raise ValueError(f"order {order!r}: one of {ORDERS}")
    if order == "c" or lat["nbr"].shape[1] == 0:
        return None
    c = np.asarray(lat["coords"], np.int64)
    if order in _SPLITS:
        base_order, first = _SPLITS[order]
        base = node_order(lat, base_order) if base_order != "c" else None
        base = np.arange(len(c)) if base is None else base
        bnd = (np.asarray(lat["nbr"]) < 0).any(0)[base]
        perm = np.concatenate([base[bnd], base[~bnd]] if first else [base[~bnd], base[bnd]])
        return None if np.array_equal(perm, np.arange(len(perm))) else perm
    if order == "axis":
        ext = c.max(0) - c.min(0)
        fast = int(np.argmax(ext))
        slow = [a for a in (0, 1, 2) if a != fast]
        perm = np.lexsort((c[:, fast], c[:, slow[1]], c[:, slow[0]]))
    else:
        code = np.zeros(len(c), np.int64)
        for b in range(21):
            for a in range(3):
                code |= ((c[:, a] >> b) & 1) << (3 * b + (2 - a))
        perm = np.argsort(code, kind="stable")
    if np.array_equal(perm, np.arange(len(perm))):
        return None
    return perm


def default_block(n):
    """Threads per block of the step kernel: 128, what the autotuner settles on for the pipes and arteries measured
    (8 blocks of 128 per SM finish more evenly than 4 of 256)."""
    return 128


__all__ = ["LATTICE", "C", "W", "Q", "OPP", "WALL", "INLET", "OUTLET0", "Units", "build_lattice", "scatter",
           "Solver", "sponge_tau"]
