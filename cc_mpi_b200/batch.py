"""Host-side mirror of the batched-CC part of include/ccgpu.h.

A batch is a packed CSR-of-CSRs: graph g's local row pointers at
``row_ptr[vtx_off[g] + g]`` (n_g + 1 entries, 0-based), its local int32
neighbour ids at ``col[edge_off[g]]`` and its labels at
``labels[vtx_off[g]]``.  Everything here only packs arrays and passes
pointers to libccb200.so; labels are computed by the library.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check, lib

CLASSES = 3


class Batch(C.Structure):
    _fields_ = [("graphs", C.c_uint32), ("h_vtx_off", C.POINTER(C.c_uint64)),
                ("h_edge_off", C.POINTER(C.c_uint64)), ("d_row_ptr", C.c_void_p),
                ("d_col", C.c_void_p), ("d_labels", C.c_void_p)]


class ClassOpts(C.Structure):
    _fields_ = [("sample_rounds", C.c_int), ("cadence", C.c_int), ("tile", C.c_int),
                ("warp_degree", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(C.Structure):
    _fields_ = [("class_bounds", C.c_float * (CLASSES - 1)), ("heavy_degree", C.c_int),
                ("cls", ClassOpts * CLASSES), ("persistent", C.c_int), ("wait_ms", C.c_int),
                ("stall_graph", C.c_int)]

    def as_dict(self):
        return {"class_bounds": list(self.class_bounds), "heavy_degree": self.heavy_degree,
                "classes": [self.cls[c].as_dict() for c in range(CLASSES)],
                "persistent": self.persistent, "wait_ms": self.wait_ms}


_bound = False


def _bind():
    global _bound
    if _bound:
        return lib()
    vp, i = C.c_void_p, C.c_int
    _lib.declare("ccgpu_batch_tuning_default", None, [C.POINTER(Tuning)])
    _lib.declare("ccgpu_batch_plan_create", i, [vp, C.POINTER(Batch), C.POINTER(Tuning),
                                                C.POINTER(vp)])
    _lib.declare("ccgpu_batch_plan_run", i, [vp, vp])
    _lib.declare("ccgpu_batch_plan_launch", i, [vp, vp])
    _lib.declare("ccgpu_batch_plan_kernels", i, [vp])
    _lib.declare("ccgpu_batch_plan_autotune", i, [vp, vp, C.POINTER(Tuning)])
    _lib.declare("ccgpu_batch_plan_tuning", i, [vp, C.POINTER(Tuning)])
    _lib.declare("ccgpu_batch_plan_class_graphs", i, [vp, vp])
    _lib.declare("ccgpu_batch_plan_results", i, [vp, vp, vp, vp])
    _lib.declare("ccgpu_batch_plan_destroy", None, [vp])
    _lib.declare("ccgpu_batch_cc", i, [vp, C.POINTER(Batch), C.POINTER(Tuning), vp, vp])
    _bound = True
    return lib()


def default_tuning() -> Tuning:
    t = Tuning()
    _bind().ccgpu_batch_tuning_default(C.byref(t))
    return t


def pack(graphs):
    """[(row_ptr, col), ...] numpy CSRs -> (vtx_off, edge_off, row_ptr, col)
    numpy arrays of the packed layout."""
    ns = np.array([len(rp) - 1 for rp, _ in graphs], dtype=np.uint64)
    ms = np.array([int(rp[-1]) for rp, _ in graphs], dtype=np.uint64)
    vtx_off = np.zeros(len(graphs) + 1, dtype=np.uint64)
    edge_off = np.zeros(len(graphs) + 1, dtype=np.uint64)
    np.cumsum(ns, out=vtx_off[1:])
    np.cumsum(ms, out=edge_off[1:])
    row_ptr = np.concatenate([np.asarray(rp, dtype=np.uint64) for rp, _ in graphs]) \
        if graphs else np.zeros(0, np.uint64)
    col = np.concatenate([np.asarray(c, dtype=np.uint32) for _, c in graphs]) \
        if graphs else np.zeros(0, np.uint32)
    return vtx_off, edge_off, row_ptr, col


class BatchPlan:
    """ccgpu_batch_plan over device arrays (torch tensors, kept alive here)."""

    def __init__(self, vtx_off, edge_off, d_row_ptr, d_col, d_labels, tuning=None, ctx=None):
        L = _bind()
        self.vtx_off = np.ascontiguousarray(vtx_off, dtype=np.uint64)
        self.edge_off = np.ascontiguousarray(edge_off, dtype=np.uint64)
        self.G = len(self.vtx_off) - 1
        self._keep = (d_row_ptr, d_col, d_labels)
        self.d_labels = d_labels
        b = Batch()
        b.graphs = self.G
        b.h_vtx_off = self.vtx_off.ctypes.data_as(C.POINTER(C.c_uint64))
        b.h_edge_off = self.edge_off.ctypes.data_as(C.POINTER(C.c_uint64))
        b.d_row_ptr = d_row_ptr.data_ptr()
        b.d_col = d_col.data_ptr() if d_col.numel() else None
        b.d_labels = d_labels.data_ptr()
        self._b = b
        self.p = C.c_void_p()
        check(L.ccgpu_batch_plan_create(ctx, C.byref(b), C.byref(tuning) if tuning else None,
                                        C.byref(self.p)))

    @staticmethod
    def _stream(stream):
        if stream is None:
            import torch
            return torch.cuda.current_stream().cuda_stream
        return stream

    def run(self, stream=None):
        check(lib().ccgpu_batch_plan_run(self.p, self._stream(stream)))

    def launch(self, stream=None):
        check(lib().ccgpu_batch_plan_launch(self.p, self._stream(stream)))

    def kernels(self):
        return lib().ccgpu_batch_plan_kernels(self.p)

    def autotune(self, stream=None) -> Tuning:
        t = Tuning()
        check(lib().ccgpu_batch_plan_autotune(self.p, self._stream(stream), C.byref(t)))
        return t

    def tuning(self) -> Tuning:
        t = Tuning()
        check(lib().ccgpu_batch_plan_tuning(self.p, C.byref(t)))
        return t

    def class_graphs(self):
        a = np.zeros(CLASSES, dtype=np.uint32)
        check(lib().ccgpu_batch_plan_class_graphs(self.p, a.ctypes.data))
        return a

    def results(self, stream=None):
        comps = np.zeros(self.G, dtype=np.uint32)
        done = np.zeros(self.G, dtype=np.uint32)
        check(lib().ccgpu_batch_plan_results(self.p, comps.ctypes.data, done.ctypes.data,
                                             self._stream(stream)))
        return comps, done

    def close(self):
        if self.p:
            lib().ccgpu_batch_plan_destroy(self.p)
            self.p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def labels_of(labels: np.ndarray, vtx_off: np.ndarray, g: int) -> np.ndarray:
    return labels[int(vtx_off[g]):int(vtx_off[g + 1])]


# --------------------------------------------------------------- workloads


def mix_spec(graphs=4096, n_min=1_000, n_max=2_000_000, seed=7):
    """The batched workload's mix: vertex counts log-uniform in
    [n_min, n_max], one third each Erdos-Renyi (mean degree 8), R-MAT (edge
    factor 16) and 2-D grids with 10% of edges deleted, kinds assigned in a
    seeded random order.  Returns [(kind, n, seed), ...]."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(n_min), math.log(n_max), graphs)).astype(np.int64)
    kinds = np.array(["er", "rmat", "grid"])[rng.permutation(graphs) % 3]
    seeds = rng.integers(1, 2**31 - 1, graphs)
    return [(str(k), int(n), int(s)) for k, n, s in zip(kinds, ns, seeds)]


def build_one_torch(torch, kind, n, seed, device="cuda"):
    from . import graphs as G
    if kind == "er":
        return G.er_csr_torch(torch, n, 8.0, seed=seed, device=device)
    if kind == "rmat":
        scale = max(1, math.ceil(math.log2(max(n, 2))))
        frac = n / float(1 << scale)
        samples = int(16 * n / (frac * frac))
        return G.rmat_csr_torch(torch, scale, 16, seed=seed, device=device, n=n,
                                samples=samples)
    rows = max(1, int(math.isqrt(n)))
    cols = max(1, n // rows)
    return G.grid_csr_torch(torch, rows, cols, 0.1, seed=seed, device=device)


def build_batch_torch(torch, spec, device="cuda"):
    """Builds every graph of `spec` on the device and packs them.  Returns
    (vtx_off, edge_off host numpy, d_row_ptr int64, d_col int32, kinds).
    Graphs are seeded, so a first pass only measures their sizes and a
    second pass rebuilds each one straight into the packed arrays: peak
    memory is the packed batch plus one graph's temporaries."""
    ns, ms = [], []
    for kind, n, seed in spec:
        rp, col = build_one_torch(torch, kind, n, seed, device)
        ns.append(rp.numel() - 1)
        ms.append(col.numel())
        del rp, col
    vtx_off = np.zeros(len(spec) + 1, dtype=np.uint64)
    edge_off = np.zeros(len(spec) + 1, dtype=np.uint64)
    np.cumsum(np.array(ns, dtype=np.uint64), out=vtx_off[1:])
    np.cumsum(np.array(ms, dtype=np.uint64), out=edge_off[1:])
    d_rp = torch.empty(int(vtx_off[-1]) + len(spec), dtype=torch.int64, device=device)
    d_col = torch.empty(max(int(edge_off[-1]), 1), dtype=torch.int32, device=device)
    for g, (kind, n, seed) in enumerate(spec):
        rp, col = build_one_torch(torch, kind, n, seed, device)
        assert rp.numel() - 1 == ns[g] and col.numel() == ms[g], "graph builder not deterministic"
        a = int(vtx_off[g]) + g
        d_rp[a:a + rp.numel()].copy_(rp)
        if col.numel():
            e = int(edge_off[g])
            d_col[e:e + col.numel()].copy_(col)
        del rp, col
    return vtx_off, edge_off, d_rp, d_col, [k for k, _, _ in spec]
