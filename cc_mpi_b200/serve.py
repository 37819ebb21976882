"""Host-side mirror of the request server in include/ccgpu.h
(ccgpu_server_*): submit host CSRs, wait for their labels.  The server's
worker thread, pool and batching live in libccb200.so."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib


class ServerOpts(C.Structure):
    _fields_ = [("hbm_bytes", C.c_size_t), ("max_graphs", C.c_uint32),
                ("max_batch", C.c_uint32), ("streams", C.c_int)]


class RequestInfo(C.Structure):
    _fields_ = [("t_submit", C.c_double), ("t_admit", C.c_double), ("t_start", C.c_double),
                ("t_done", C.c_double), ("components", C.c_uint32),
                ("batch_graphs", C.c_uint32), ("status", C.c_int)]

    @property
    def latency(self):
        return self.t_done - self.t_submit


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("batches", C.c_uint64),
                ("in_flight", C.c_uint32), ("max_in_flight", C.c_uint32),
                ("max_batch_seen", C.c_uint32), ("pending", C.c_uint32),
                ("resident", C.c_uint32), ("pool_bytes", C.c_size_t),
                ("pool_used", C.c_size_t), ("pool_peak", C.c_size_t)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_bound = False


def _bind():
    global _bound
    if _bound:
        return lib()
    from .batch import Tuning
    vp = C.c_void_p
    _lib.declare("ccgpu_server_opts_default", None, [C.POINTER(ServerOpts)])
    _lib.declare("ccgpu_server_create", C.c_int, [C.POINTER(ServerOpts), C.POINTER(Tuning),
                                                  C.POINTER(vp)])
    _lib.declare("ccgpu_server_submit", C.c_int, [vp, vp, vp, C.c_uint32, C.c_uint64, vp,
                                                  C.POINTER(C.c_uint64)])
    _lib.declare("ccgpu_server_wait", C.c_int, [vp, C.c_uint64, C.c_double,
                                                C.POINTER(RequestInfo)])
    _lib.declare("ccgpu_server_stats_get", C.c_int, [vp, C.POINTER(ServerStats)])
    _lib.declare("ccgpu_server_now", C.c_double, [vp])
    _lib.declare("ccgpu_server_destroy", None, [vp])
    _bound = True
    return lib()


class Server:
    """One ccgpu_server.  Arrays passed to submit() are kept alive here until
    their wait() returns."""

    def __init__(self, hbm_bytes=0, max_graphs=8192, max_batch=4096, streams=2, tuning=None):
        L = _bind()
        o = ServerOpts(hbm_bytes, max_graphs, max_batch, streams)
        self.s = C.c_void_p()
        check(L.ccgpu_server_create(C.byref(o), C.byref(tuning) if tuning else None,
                                    C.byref(self.s)))
        self._held = {}

    def submit(self, row_ptr, col_idx, labels=None):
        row_ptr = np.ascontiguousarray(row_ptr, dtype=np.uint64)
        col_idx = np.ascontiguousarray(col_idx, dtype=np.uint32)
        n = len(row_ptr) - 1
        if labels is None:
            labels = np.empty(max(n, 0), dtype=np.uint32)
        t = C.c_uint64()
        check(lib().ccgpu_server_submit(self.s, row_ptr.ctypes.data,
                                        col_idx.ctypes.data if len(col_idx) else None, n,
                                        int(row_ptr[-1]) if n >= 0 else 0,
                                        labels.ctypes.data if n else None, C.byref(t)))
        self._held[t.value] = (row_ptr, col_idx, labels)
        return t.value

    def wait(self, ticket, timeout=-1.0):
        info = RequestInfo()
        check(lib().ccgpu_server_wait(self.s, ticket, timeout, C.byref(info)))
        _, _, labels = self._held.pop(ticket)
        return labels, info

    def stats(self) -> ServerStats:
        st = ServerStats()
        check(lib().ccgpu_server_stats_get(self.s, C.byref(st)))
        return st

    def now(self):
        return lib().ccgpu_server_now(self.s)

    def close(self):
        if self.s:
            lib().ccgpu_server_destroy(self.s)
            self.s = C.c_void_p()
            self._held.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
