"""cs_links_build_noalloc: the link-table build for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc: a plugin whose host application owns all device memory and hands it only its
input and output buffers, or a process whose fixed device-memory budget is already committed. This entry point
keeps its scratch in a static array inside the library, so such a caller passes only inputs and outputs. The test
checks it against the regular two-call build (cs_links_count + cs_links_fill with a caller-provided scratch
buffer) on several calls in a row — the shared static scratch must not carry anything over from one call to the
next — with exactly sized and with oversized ghost tables, runs the step on its tables against the regular ones, and
checks that sizes beyond its stated limit are refused.

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


@pytest.mark.parametrize("extra", [0, 300])
def test_noalloc_build_matches_regular_build(extra):
    """Three lattices in a row (the static scratch must carry nothing over); ghost tables sized exactly (extra 0)
    or with 300 spare slots per direction, whose entries must stay as the caller pre-filled them."""
    torch.cuda.set_device(0)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for name in ("stenosis70_D20", "open_pipe_tilted_D20", "stenosis70_D20"):
        lat = lbm.build_lattice(**cases.lattice_args(cases.case(name)))
        nbr, q = lat["_dev"]["nbr"], lat["_dev"]["q"]
        n, n_out = int(lat["nbr"].shape[1]), max(1, lat["n_outlets"])
        ghosts_ref, gmax, ref = reference_tables(nbr, q, n, n_out, stream)
        rc, ghosts, got = noalloc_tables(nbr, q, n, n_out, gmax + extra, stream)
        _lib.check(rc)
        torch.cuda.synchronize()
        assert ghosts == ghosts_ref
        assert torch.equal(got[0], ref[0]), name
        for a, b, fill in zip(got[1:], ref[1:], (-1, -1, -1.0)):
            assert torch.equal(a[:, :gmax], b), name
            assert bool((a[:, gmax:] == fill).all()), name


def solver_on_noalloc_tables(lat, extra, stream):
    """A Solver whose step tables come from cs_links_build_noalloc with `extra` spare ghost slots per direction
    (so the ghost stride, and the population padding, differ from the regular build's)."""
    lib = _lib.load()
    s = lbm.Solver(lat, 0.02, model="regularised")
    n, n_out = s.N, len(s.p_out)
    gmax_cap = s.gmax + extra
    rc, ghosts, (links, gnode, ginfo, gq) = noalloc_tables(lat["_dev"]["nbr"], lat["_dev"]["q"], n, n_out, gmax_cap,
                                                           stream)
    _lib.check(rc)
    n_seg, n_irr = ctypes.c_int64(0), ctypes.c_int64(0)
    scratch = torch.empty(max(1, int(lib.cs_compress_scratch_bytes(n))), dtype=torch.uint8, device=links.device)
    _lib.check(lib.cs_compress_count(ptr(links), n, ptr(scratch), ctypes.byref(n_seg), ctypes.byref(n_irr), stream))
    s.n_seg, s.n_irr = int(n_seg.value), int(n_irr.value)
    s.lcode = torch.empty(max(1, n), dtype=torch.int32, device=links.device)
    s.segdelta = torch.empty((max(1, s.n_seg), lbm.SEG_STRIDE), dtype=torch.int32, device=links.device)
    s.irr = torch.empty((27, max(1, s.n_irr)), dtype=torch.int32, device=links.device)
    _lib.check(lib.cs_compress_fill(ptr(links), n, s.n_seg, s.n_irr, ptr(scratch), ptr(s.lcode), ptr(s.segdelta),
                                    ptr(s.irr), stream))
    torch.cuda.synchronize()
    s.ghosts, s.gmax, s.npad = ghosts, gmax_cap, n + gmax_cap
    s.gnode, s.ginfo, s.gq = gnode, ginfo, gq
    s.f = [torch.zeros((27, s.npad), dtype=torch.float32, device=links.device) for _ in range(2)]
    s._drop_graphs()
    return s


@pytest.mark.parametrize("extra", [0, 300])
def test_step_on_noalloc_tables(extra):
    """The step on tables from the no-allocation build ends bit for bit where it ends on the regular tables."""
    torch.cuda.set_device(0)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    lat = lbm.build_lattice(**cases.lattice_args(cases.case("open_pipe_straight_D20")))
    solvers = [lbm.Solver(lat, 0.02, model="regularised"), solver_on_noalloc_tables(lat, extra, stream)]
    for s in solvers:
        s.set_sponge(10, 0.6)
        s.set_drive([0.03, 0.005, 0.0], period=100, ramp=50)
        s.set_outlet_pressure([0.0])
        s.run(120, chunk=40)
    (p0, u0), (p1, u1) = solvers[0].fields(), solvers[1].fields()
    assert solvers[1].ok() and np.abs(u0).max() > 0
    assert np.array_equal(p0, p1) and np.array_equal(u0, u1)


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
