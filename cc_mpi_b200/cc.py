"""Host-side mirror of include/cc.h and the local-CC part of include/ccgpu.h.

Every function passes pointers straight to libccb200.so; nothing here
computes labels.  Device arrays are torch tensors (plumbing only: memory and
streams); host arrays are numpy arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import CCOpts, CCStats, CSRGraph, check, lib

_cc_bound = False


def _bind():
    global _cc_bound
    if _cc_bound:
        return
    L = lib()
    _lib.declare("compute_connected_components_pthreads", None,
                 [C.POINTER(CSRGraph), C.c_void_p, C.c_int, C.c_int])
    for name in ("compute_connected_components", "compute_connected_components_bfs"):
        _lib.declare(name, None, [C.POINTER(CSRGraph), C.c_void_p])
    for name in ("compute_connected_components_omp", "compute_connected_components_cilk"):
        _lib.declare(name, None, [C.POINTER(CSRGraph), C.c_void_p, C.c_int])
    _lib.declare("count_unique_labels", C.c_uint32, [C.c_void_p, C.c_uint32])
    _lib.declare("ccb200_set_exit_on_error", C.c_int, [C.c_int])
    _cc_bound = True
    return L


def csr_struct(row_ptr: np.ndarray, col_idx: np.ndarray) -> CSRGraph:
    """CSRGraph view of numpy arrays (kept alive by the caller)."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.uint64)
    col_idx = np.ascontiguousarray(col_idx, dtype=np.uint32)
    g = CSRGraph()
    g.n = len(row_ptr) - 1
    g.m = int(row_ptr[-1]) if len(row_ptr) else 0
    g.row_ptr = row_ptr.ctypes.data_as(C.POINTER(C.c_uint64))
    g.col_idx = col_idx.ctypes.data_as(C.POINTER(C.c_uint32))
    return g


def compute_connected_components_pthreads(row_ptr, col_idx, num_threads=0, chunk_size=0,
                                          labels=None):
    """Mirror of the reference's compute_connected_components_pthreads
    (include/cc.h:27-28): host CSR in, host labels (min id per component)
    out.  Calls the C symbol of the same name; a failure raises instead of
    exiting the process."""
    _bind()
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.uint64)
    col_idx = np.ascontiguousarray(col_idx, dtype=np.uint32)
    n = len(row_ptr) - 1
    if labels is None:
        labels = np.empty(n, dtype=np.uint32)
    g = csr_struct(row_ptr, col_idx)
    L = lib()
    prev = L.ccb200_set_exit_on_error(0)
    try:
        L.ccgpu_clear_error()
        L.compute_connected_components_pthreads(C.byref(g), labels.ctypes.data, num_threads,
                                                chunk_size)
        msg = L.ccgpu_last_error()
        if msg:
            raise _lib.CCGPUError(2, msg.decode())
    finally:
        L.ccb200_set_exit_on_error(prev)
    return labels


def count_unique_labels(labels: np.ndarray) -> int:
    _bind()
    labels = np.ascontiguousarray(labels, dtype=np.uint32)
    return int(lib().count_unique_labels(labels.ctypes.data, len(labels)))


def local_cc_host(row_ptr, col_idx, opts: CCOpts | None = None, stats=False, ctx=None):
    """ccgpu_local_cc_host: host buffers in and out, status-checked."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.uint64)
    col_idx = np.ascontiguousarray(col_idx, dtype=np.uint32)
    n = len(row_ptr) - 1
    labels = np.empty(max(n, 0), dtype=np.uint32)
    st = CCStats()
    check(lib().ccgpu_local_cc_host(ctx, row_ptr.ctypes.data, col_idx.ctypes.data, n,
                                    int(row_ptr[-1]) if n >= 0 else 0, labels.ctypes.data,
                                    C.byref(opts) if opts is not None else None,
                                    C.byref(st) if stats else None))
    return (labels, st) if stats else labels


def local_cc_device(d_row_ptr, d_col_idx, n, m, d_labels, opts: CCOpts | None = None,
                    stats=False, stream=None, ctx=None):
    """ccgpu_local_cc on device pointers (ints) or torch tensors."""
    def ptr(x):
        return x if isinstance(x, int) else x.data_ptr()
    st = CCStats()
    if stream is None:
        import torch
        stream = torch.cuda.current_stream().cuda_stream
    check(lib().ccgpu_local_cc(ctx, ptr(d_row_ptr), ptr(d_col_idx), n, m, ptr(d_labels),
                               C.byref(opts) if opts is not None else None,
                               C.byref(st) if stats else None, stream))
    return st if stats else None


def count_roots_device(d_labels, n, stream=None, ctx=None):
    import torch
    out = C.c_uint64(0)
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    check(lib().ccgpu_count_roots(ctx, d_labels.data_ptr(), n, C.byref(out), stream))
    return out.value


def check_labels_device(d_row_ptr, d_col_idx, n, m, d_labels, stream=None, ctx=None):
    import torch
    out = C.c_uint64(0)
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    check(lib().ccgpu_check_labels(ctx, d_row_ptr.data_ptr(), d_col_idx.data_ptr(), n, m,
                                   d_labels.data_ptr(), C.byref(out), stream))
    return out.value
