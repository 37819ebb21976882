"""Host-side mirror of the partitioned path (include/cc_mpi.h,
include/graph_dist.h, include/boundary_sort.h and the ccgpu_dist_* /
ccgpu_boundary_* calls of include/ccgpu.h).  Pointers only: the work is done
by libccb200.so."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib


class DistOpts(C.Structure):
    _fields_ = [("parts", C.c_int), ("use_edge", C.c_int), ("chunk_size", C.c_int),
                ("exchange_interval", C.c_int), ("verbose", C.c_int)]


class DistStats(C.Structure):
    _fields_ = [("rounds", C.c_int), ("exchanges", C.c_int), ("sort_passes", C.c_int),
                ("pad", C.c_int), ("boundary_raw", C.c_uint64), ("pair_count", C.c_uint64),
                ("ghost_count", C.c_uint64), ("rep_count", C.c_uint64), ("roots", C.c_uint64),
                ("sent_pairs", C.c_uint64), ("ms_bounds", C.c_double), ("ms_local", C.c_double),
                ("ms_pairs", C.c_double), ("ms_sort", C.c_double), ("ms_ghosts", C.c_double),
                ("ms_merge", C.c_double), ("ms_total", C.c_double),
                ("sorted_keys", C.c_uint64), ("local_entries", C.c_uint64),
                ("sorted_rows", C.c_int), ("row_runs", C.c_int)]


_bound = False


def _bind():
    global _bound
    if _bound:
        return
    vp, u32, u64, i = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
    _lib.declare("ccgpu_dist_opts_default", None, [C.POINTER(DistOpts)])
    _lib.declare("ccgpu_dist_cc", i, [vp, vp, vp, u32, u64, C.POINTER(DistOpts), vp, vp,
                                      C.POINTER(DistStats), vp])
    _lib.declare("ccgpu_partition_bounds", i, [vp, u32, i, i, vp, vp])
    _lib.declare("ccgpu_boundary_sort", i, [vp, vp, u64, u32, u32, vp])
    _lib.declare("ccgpu_boundary_dedup", i, [vp, vp, u64, C.POINTER(u64), vp])
    _bound = True


def _ptr(x):
    return x if isinstance(x, int) or x is None else x.data_ptr()


def _stream(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return stream


def dist_cc_device(d_row_ptr, d_col, n, m, parts, use_edge=1, chunk_size=2048,
                   exchange_interval=1, d_labels=None, verbose=0, stream=None, ctx=None):
    """ccgpu_dist_cc -> (stats, bounds ndarray[parts+1])."""
    _bind()
    o = DistOpts(parts, use_edge, chunk_size, exchange_interval, verbose)
    st = DistStats()
    bounds = np.zeros(parts + 1, dtype=np.uint32)
    check(lib().ccgpu_dist_cc(ctx, _ptr(d_row_ptr), _ptr(d_col), n, m, C.byref(o),
                              _ptr(d_labels), bounds.ctypes.data, C.byref(st), _stream(stream)))
    return st, bounds


def partition_bounds_device(d_row_ptr, n, parts, use_edge=1, stream=None):
    _bind()
    bounds = np.zeros(parts + 1, dtype=np.uint32)
    check(lib().ccgpu_partition_bounds(_ptr(d_row_ptr), n, parts, use_edge, bounds.ctypes.data,
                                       _stream(stream)))
    return bounds


def boundary_sort_device(d_pairs, count, max_rep=0xFFFFFFFF, max_remote=0xFFFFFFFF,
                         stream=None, ctx=None):
    _bind()
    check(lib().ccgpu_boundary_sort(ctx, _ptr(d_pairs), count, max_rep, max_remote,
                                    _stream(stream)))


def boundary_dedup_device(d_pairs, count, stream=None, ctx=None):
    _bind()
    out = C.c_uint64(0)
    check(lib().ccgpu_boundary_dedup(ctx, _ptr(d_pairs), count, C.byref(out), _stream(stream)))
    return out.value
