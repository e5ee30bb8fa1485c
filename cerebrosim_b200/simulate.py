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
