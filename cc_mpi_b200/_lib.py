"""ctypes binding of libccb200.so (the C ABI declared in include/ccgpu.h and
the reference-facing calls in include/cc.h, include/cc_mpi.h, ...).

The library is built in-tree by ``__graft_entry__.build()`` (or ``make -C
cc_mpi_b200/csrc``).  There is no fallback: if the shared object is missing or
does not load, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libccb200.so")
CLI_PATH = os.path.join(_HERE, "bin", "mpi_cc_benchmark")

STATUS = {
    0: "OK", 1: "INVALID", 2: "CUDA", 3: "OOM", 4: "TIMEOUT", 5: "LIMIT",
    6: "NODEVICE", 7: "IO", 8: "FORMAT",
}


class CCGPUError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"ccgpu status {status} ({STATUS.get(status, '?')}): {msg}")
        self.status = status


class CCOpts(C.Structure):
    _fields_ = [("chunk_size", C.c_int), ("sample_rounds", C.c_int),
                ("heavy_degree", C.c_int), ("skip_giant", C.c_int), ("hook_mode", C.c_int)]


class CCStats(C.Structure):
    _fields_ = [("giant_label", C.c_uint32), ("heavy_rows", C.c_uint32),
                ("components", C.c_uint32), ("kernels", C.c_uint32),
                ("finish_rows", C.c_uint64), ("finish_edges", C.c_uint64)]


class CSRGraph(C.Structure):
    """include/graph.h CSRGraph (reference include/graph.h:8-14)."""
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint64),
                ("row_ptr", C.POINTER(C.c_uint64)), ("col_idx", C.POINTER(C.c_uint32))]


class DistCSRGraph(C.Structure):
    """include/graph_dist.h DistCSRGraph (reference include/graph_dist.h:15-28)."""
    _fields_ = [("n_global", C.c_uint32), ("m_global", C.c_uint64),
                ("n_local", C.c_uint32), ("m_local", C.c_uint64),
                ("v_start", C.c_uint32), ("v_end", C.c_uint32),
                ("row_ptr", C.POINTER(C.c_uint64)), ("col_idx", C.POINTER(C.c_uint32)),
                ("part_bounds", C.POINTER(C.c_uint32)),
                ("part_size", C.c_int), ("part_kind", C.c_int)]


_lib = None

_VP = C.c_void_p
_U32 = C.c_uint32
_U64 = C.c_uint64
_INT = C.c_int

# name -> (restype, argtypes)
_SIGS = {
    "ccgpu_last_error": (C.c_char_p, []),
    "ccgpu_clear_error": (None, []),
    "ccgpu_version": (_INT, []),
    "ccgpu_device_check": (_INT, []),
    "ccgpu_ctx_create": (_INT, [C.POINTER(_VP)]),
    "ccgpu_ctx_destroy": (None, [_VP]),
    "ccgpu_ctx_scratch_bytes": (C.c_size_t, [_VP]),
    "ccgpu_ctx_launches": (_U64, [_VP]),
    "ccgpu_prof_enable": (_INT, [_VP, _INT]),
    "ccgpu_prof_collect": (_INT, [_VP, _VP, _VP]),
    "ccgpu_prof_kernels": (_INT, []),
    "ccgpu_prof_name": (C.c_char_p, [_INT]),
    "ccgpu_cc_opts_default": (None, [C.POINTER(CCOpts)]),
    "ccgpu_local_cc": (_INT, [_VP, _VP, _VP, _U32, _U64, _VP, C.POINTER(CCOpts),
                              C.POINTER(CCStats), _VP]),
    "ccgpu_local_cc_host": (_INT, [_VP, _VP, _VP, _U32, _U64, _VP, C.POINTER(CCOpts),
                                   C.POINTER(CCStats)]),
    "ccgpu_count_roots": (_INT, [_VP, _VP, _U32, C.POINTER(_U64), _VP]),
    "ccgpu_local_cc_plan": (_INT, [_VP, _VP, _U32, _U64, _VP, C.POINTER(CCOpts),
                                   C.POINTER(_VP)]),
    "ccgpu_plan_launch": (_INT, [_VP, _VP]),
    "ccgpu_plan_kernels": (_INT, [_VP]),
    "ccgpu_plan_destroy": (None, [_VP]),
    "ccgpu_check_labels": (_INT, [_VP, _VP, _VP, _U32, _U64, _VP, C.POINTER(_U64), _VP]),
}


def lib():
    """Load libccb200.so (once).  Raises if it is missing: no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; "
            f"g.build()'` or `make -C cc_mpi_b200/csrc`")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def declare(name, restype, argtypes):
    """Attach a signature to one more exported function (used by modules
    that bind the reference-facing calls)."""
    f = getattr(lib(), name)
    f.restype = restype
    f.argtypes = argtypes
    return f


def check(status):
    if status != 0:
        msg = lib().ccgpu_last_error()
        raise CCGPUError(status, msg.decode() if msg else "")
    return status


HOOK_FIRST, HOOK_LAZY, HOOK_CADENCE = 1, 2, 4


def opts(chunk_size=4096, sample_rounds=2, heavy_degree=8192, skip_giant=1,
         hook_mode=HOOK_CADENCE | 8):
    return CCOpts(chunk_size, sample_rounds, heavy_degree, skip_giant, hook_mode)
