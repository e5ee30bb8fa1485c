"""The C ABI without a GPU: the library loads, exports every symbol include/cerebrosim.h declares, its struct
layouts match the bindings, and argument errors come back as status codes with messages (no CUDA call is made
on these paths)."""
import ctypes
import subprocess

import pytest

from cerebrosim_b200 import _lib


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _lib.header_symbols()
    assert declared, "no declarations parsed"
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.split()}
    for name in declared:
        assert name in exported, f"{name} declared but not exported"
        assert hasattr(lib, name)
        assert name in _lib.SIGNATURES, f"{name} has no binding"


def test_abi_sizes_and_version():
    lib = _lib.load()
    assert lib.cs_abi_sizeof(0) == ctypes.sizeof(_lib.Opening) == 64
    assert lib.cs_abi_sizeof(1) == ctypes.sizeof(_lib.StepDesc)
    assert lib.cs_abi_sizeof(7) == 0
    from cerebrosim_b200 import lbm
    assert lib.cs_abi_sizeof(2) == lbm.SEG_STRIDE
    assert b"sm_100a" in lib.cs_version()


def test_scratch_size_is_host_only():
    lib = _lib.load()
    s = lib.cs_lattice_scratch_bytes(10, 20, 30)
    assert s >= 10 * 20 * 30 * 4
    assert lib.cs_lattice_scratch_bytes(-1, 2, 2) == 0


@pytest.mark.parametrize("call", [
    lambda lib: lib.cs_step(None, 0, 1, None),
    lambda lib: lib.cs_graph_launch(None, None),
    lambda lib: lib.cs_links_fill(None, None, 10, 0, 0, None, None, None, None, None, None, None),
    lambda lib: lib.cs_links_fill(None, None, 10, 1, 80_000_000, None, None, None, None, None, None, None),
    lambda lib: lib.cs_links_count(None, -1, None, (ctypes.c_int64 * 27)(), None),
    lambda lib: lib.cs_links_decode(None, None, None, -1, 0, None, None, None),
    lambda lib: lib.cs_flux_blocks(None, 0, 10, 16, None, None),
    lambda lib: lib.cs_lattice_count(None, -1, 2, 2, None, ctypes.byref(ctypes.c_int64()), None),
])
def test_argument_errors_are_reported(call):
    lib = _lib.load()
    rc = call(lib)
    assert rc in (_lib.CS_ERR_ARG, _lib.CS_ERR_SIZE)
    msg = _lib.last_error()
    assert msg.startswith("cs_")
    with pytest.raises(_lib.CerebroSimError):
        _lib.check(rc)


def test_step_desc_validation_without_gpu():
    lib = _lib.load()
    d = _lib.StepDesc()
    d.n, d.period, d.block = 100, 0, 128
    assert lib.cs_step(ctypes.byref(d), 0, 1, None) == _lib.CS_ERR_SIZE
    assert "npad" in _lib.last_error()
    d.npad = 100
    assert lib.cs_step(ctypes.byref(d), 0, 1, None) == _lib.CS_ERR_ARG
    assert "period" in _lib.last_error()
    d.period, d.block = 1, 100
    assert lib.cs_step(ctypes.byref(d), 0, 1, None) == _lib.CS_ERR_ARG
    assert "block" in _lib.last_error()
    d.block, d.storage = 128, 5
    assert lib.cs_step(ctypes.byref(d), 0, 1, None) == _lib.CS_ERR_ARG
