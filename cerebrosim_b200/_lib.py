"""ctypes binding of libcerebrosim_b200.so (the C ABI declared in include/cerebrosim.h).

Loading fails loudly: there is no CPU fallback. `load()` raises if the library is missing (build it with
`python -m cerebrosim_b200.csrc.build`) and `check(rc)` turns every non-zero status into a `CerebroSimError` carrying
the library's message.
"""
import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
# the in-tree build; CEREBROSIM_B200_LIB may name another build of the same ABI (checked at load)
LIB_PATH = os.environ.get("CEREBROSIM_B200_LIB") or os.path.join(HERE, "libcerebrosim_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "cerebrosim.h")

CS_OK, CS_ERR_ARG, CS_ERR_CUDA, CS_ERR_SIZE, CS_ERR_DEVICE = 0, 1, 2, 3, 4
STORE = {"f32": 0, "f16": 1, "bf16": 2}


class CerebroSimError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__(f"[cs error {code}] {msg}")
        self.code = code


class Opening(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("pad_", ctypes.c_int32), ("centre", ctypes.c_double * 3),
                ("normal", ctypes.c_double * 3), ("radius", ctypes.c_double)]


class StepDesc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("npad", ctypes.c_int64), ("gmax", ctypes.c_int64),
                ("storage", ctypes.c_int32), ("model", ctypes.c_int32),
                ("bouzidi", ctypes.c_int32), ("gal", ctypes.c_int32), ("sigma", ctypes.c_float),
                ("magic", ctypes.c_float), ("force", ctypes.c_float * 3), ("block", ctypes.c_int32),
                ("f", ctypes.c_void_p * 2), ("vel", ctypes.c_void_p * 2), ("rho", ctypes.c_void_p),
                ("lcode", ctypes.c_void_p), ("segdelta", ctypes.c_void_p), ("irr", ctypes.c_void_p),
                ("n_irr", ctypes.c_int64), ("gnode", ctypes.c_void_p), ("ginfo", ctypes.c_void_p),
                ("gq", ctypes.c_void_p), ("uin", ctypes.c_void_p), ("om", ctypes.c_void_p),
                ("p_out", ctypes.c_void_p), ("n_out", ctypes.c_int32), ("tick", ctypes.c_void_p),
                ("drive", ctypes.c_void_p), ("coef", ctypes.c_void_p), ("nh", ctypes.c_int32),
                ("period", ctypes.c_int32), ("ramp", ctypes.c_int32),
                ("n_open", ctypes.c_int32), ("n_flux", ctypes.c_int64), ("flux_idx", ctypes.c_void_p),
                ("flux_w", ctypes.c_void_p), ("flux_slot", ctypes.c_void_p), ("flux_block", ctypes.c_void_p),
                ("q_part", ctypes.c_void_p), ("fb_list", ctypes.c_void_p), ("n_fb", ctypes.c_int32),
                ("q_last", ctypes.c_void_p), ("p_out64", ctypes.c_void_p),
                ("r_out", ctypes.c_void_p), ("pref", ctypes.c_double), ("alpha", ctypes.c_double),
                ("gblock", ctypes.c_int32 * 28), ("beat_acc", ctypes.c_void_p)]


class BatchDesc(ctypes.Structure):
    _fields_ = [("n_inst", ctypes.c_int32), ("storage", ctypes.c_int32), ("model", ctypes.c_int32),
                ("gal", ctypes.c_int32), ("force", ctypes.c_int32), ("any_open", ctypes.c_int32),
                ("block", ctypes.c_int32), ("grid_bulk", ctypes.c_int32), ("grid_bnd", ctypes.c_int32),
                ("pad_", ctypes.c_int32), ("descs", ctypes.c_void_p), ("parity", ctypes.c_void_p),
                ("counter", ctypes.c_void_p)]


BATCH_GROUP = 64   # CS_BATCH_GROUP


_P = ctypes.c_void_p
_I32, _I64, _D, _SZ = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_size_t

# name -> (restype, argtypes); every symbol declared in include/cerebrosim.h
SIGNATURES = {
    "cs_sdf_vessel": (_I32, [_P, _P, _P, _P, _I32, _P, _P, _P, ctypes.c_float, ctypes.POINTER(ctypes.c_float),
                             ctypes.c_float, _I64, _I64, _I64, _P, _P]),
    "cs_lattice_scratch_bytes": (_SZ, [_I64, _I64, _I64]),
    "cs_lattice_count": (_I32, [_P, _I64, _I64, _I64, _P, ctypes.POINTER(_I64), _P]),
    "cs_lattice_fill": (_I32, [_P, _I64, _I64, _I64, ctypes.POINTER(_D), _D, ctypes.POINTER(Opening), _I32, _I32,
                               _D, _P, _I64, _P, _P, _P, _P, _P, _P]),
    "cs_sponge_om": (_I32, [_P, _I64, ctypes.POINTER(_D), _D, ctypes.POINTER(Opening), _I32, _I32, _D, _D, _D, _P, _P,
                            _P]),
    "cs_links_scratch_bytes": (_SZ, [_I64]),
    "cs_links_count": (_I32, [_P, _I64, _P, ctypes.POINTER(_I64), _P]),
    "cs_links_fill": (_I32, [_P, _P, _I64, _I32, _I64, _P, _P, _P, _P, _P, _P, _P]),
    "cs_links_decode": (_I32, [_P, _P, _P, _I64, _I64, _P, _P, _P]),
    "cs_links_build_noalloc": (_I32, [_P, _P, _I64, _I32, _I64, _P, _P, _P, _P, ctypes.POINTER(_I64), _P]),
    "cs_compress_scratch_bytes": (_SZ, [_I64]),
    "cs_compress_count": (_I32, [_P, _I64, _P, ctypes.POINTER(_I64), ctypes.POINTER(_I64), _P]),
    "cs_compress_fill": (_I32, [_P, _I64, _I64, _I64, _P, _P, _P, _P, _P]),
    "cs_compress_expand": (_I32, [_P, _P, _P, _I64, _I64, _P, _P]),
    "cs_flux_blocks": (_I32, [_P, _I64, _I64, _I32, _P, _P]),
    "cs_step": (_I32, [ctypes.POINTER(StepDesc), _I32, _I32, _P]),
    "cs_step_check": (_I32, [ctypes.POINTER(StepDesc)]),
    "cs_batch_step": (_I32, [ctypes.POINTER(BatchDesc), _I32, _I32, _P]),
    "cs_batch_graph_capture": (_I32, [ctypes.POINTER(BatchDesc), _I32, _I32, _P, ctypes.POINTER(_P)]),
    "cs_graph_capture": (_I32, [ctypes.POINTER(StepDesc), _I32, _I32, _P, ctypes.POINTER(_P)]),
    "cs_graph_launch": (_I32, [_P, _P]),
    "cs_graph_destroy": (_I32, [_P]),
    "cs_wss_shear": (_I32, [_P, _I64, _P, _P, _P, _I64, _I32, _D, _P, _P]),
    "cs_probe_gather": (_I32, [_P, _P, _I64, _P, _P, _I32, _P, _P, _P]),
    "cs_bin_fields": (_I32, [_P, _P, _I64, _P, _P, _I64, _P, _P, _P]),
    "cs_last_error": (_I32, [ctypes.c_char_p, _I32]),
    "cs_version": (ctypes.c_char_p, []),
    "cs_abi_sizeof": (_SZ, [_I32]),
}

_lib = None


def header_symbols():
    """Function names declared in include/cerebrosim.h (for the export check)."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cs_[a-z0-9_]+)\s*\(", text)))


def load():
    """Load the library once, bind every signature and check the ABI struct sizes."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cerebrosim_b200.csrc.build` "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if (lib.cs_abi_sizeof(0) != ctypes.sizeof(Opening) or lib.cs_abi_sizeof(1) != ctypes.sizeof(StepDesc)
            or lib.cs_abi_sizeof(3) != ctypes.sizeof(BatchDesc)):
        raise ImportError("libcerebrosim_b200.so ABI mismatch: rebuild the library")
    _lib = lib
    return lib


def last_error():
    buf = ctypes.create_string_buffer(1024)
    load().cs_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc):
    if rc != CS_OK:
        raise CerebroSimError(rc, last_error())
    return rc
