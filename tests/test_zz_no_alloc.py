"""cs_links_build_noalloc: the link-table build for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc: a plugin whose host application owns all device memory and hands it only its
input and output buffers, or a process whose fixed device-memory budget is already committed. This entry point
keeps its scratch in a static array inside the library, so such a caller passes only inputs and outputs. The test
checks it against the regular two-call build (cs_links_count + cs_links_fill with a caller-provided scratch
buffer) on several calls in a row — the shared static scratch must not carry anything over from one call to the
next — and that sizes beyond its stated limit are refused.

This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from cerebrosim_b200 import _lib, cases, lbm  # noqa: E402

LIMIT = 1 << 24


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def reference_tables(nbr, q, n, n_out, stream):
    """The regular build: count, then fill, with scratch allocated here."""
    lib = _lib.load()
    scratch = torch.empty(int(lib.cs_links_scratch_bytes(n)), dtype=torch.uint8, device=nbr.device)
    ghosts = (ctypes.c_int64 * 27)()
    _lib.check(lib.cs_links_count(ptr(nbr), n, ptr(scratch), ghosts, stream))
    gmax = max(ghosts)
    out = new_outputs(n, gmax, nbr.device)
    status = torch.empty(2, dtype=torch.int64, device=nbr.device)
    _lib.check(lib.cs_links_fill(ptr(nbr), ptr(q), n, n_out, gmax, ptr(scratch), *[ptr(t) for t in out], ptr(status),
                                 stream))
    return list(ghosts), gmax, out


def new_outputs(n, gmax, dev):
    cols = max(1, gmax)
    return [torch.empty((27, n), dtype=torch.int32, device=dev),
            torch.full((27, cols), -1, dtype=torch.int32, device=dev),
            torch.full((27, cols), -1, dtype=torch.int32, device=dev),
            torch.full((27, cols), -1.0, dtype=torch.float32, device=dev)]


def noalloc_tables(nbr, q, n, n_out, gmax_cap, stream):
    lib = _lib.load()
    out = new_outputs(n, gmax_cap, nbr.device)
    ghosts = (ctypes.c_int64 * 27)()
    rc = lib.cs_links_build_noalloc(ptr(nbr), ptr(q), n, n_out, gmax_cap, *[ptr(t) for t in out], ghosts, stream)
    return rc, list(ghosts), out


@pytest.mark.parametrize("order", [("stenosis70_D20", "open_pipe_tilted_D20", "stenosis70_D20")])
def test_noalloc_build_matches_regular_build(order):
    torch.cuda.set_device(0)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for name in order:                              # successive calls share the library's static scratch
        lat = lbm.build_lattice(**cases.lattice_args(cases.case(name)))
        nbr, q = lat["_dev"]["nbr"], lat["_dev"]["q"]
        n, n_out = int(lat["nbr"].shape[1]), max(1, lat["n_outlets"])
        ghosts_ref, gmax, ref = reference_tables(nbr, q, n, n_out, stream)
        rc, ghosts, got = noalloc_tables(nbr, q, n, n_out, gmax, stream)
        _lib.check(rc)
        torch.cuda.synchronize()
        assert ghosts == ghosts_ref
        for a, b in zip(got, ref):
            assert torch.equal(a.view(torch.int32) if a.dtype == torch.float32 else a,
                               b.view(torch.int32) if b.dtype == torch.float32 else b), name


def test_noalloc_refuses_what_it_cannot_hold():
    lib = _lib.load()
    torch.cuda.set_device(0)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ghosts = (ctypes.c_int64 * 27)()
    rc = lib.cs_links_build_noalloc(None, None, LIMIT + 1, 1, 0, None, None, None, None, ghosts, stream)
    assert rc == _lib.CS_ERR_SIZE and "static scratch limit" in _lib.last_error()
    # a ghost capacity below what the lattice needs: refused, with the counts reported
    lat = lbm.build_lattice(**cases.lattice_args(cases.case("open_pipe_straight_D20")))
    nbr, q = lat["_dev"]["nbr"], lat["_dev"]["q"]
    n = int(lat["nbr"].shape[1])
    rc, counts, _ = noalloc_tables(nbr, q, n, 1, 10, stream)
    assert rc == _lib.CS_ERR_SIZE and "gmax_cap" in _lib.last_error()
    assert counts == [int((lat["nbr"][i] < 0).sum()) for i in range(27)]
    # the step runs on tables from the no-allocation build exactly as on the regular ones
    s = lbm.Solver(lat, 0.02, model="regularised")
    assert np.array_equal(s.link_table().cpu().numpy()[lat["nbr"] >= 0], lat["nbr"][lat["nbr"] >= 0])
