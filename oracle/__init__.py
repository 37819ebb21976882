"""CPU oracle for the CC hot path - TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline / reference
legs of bench.py may import this package.  It wraps:

* ``liboracle.so`` - the C restatement of the reference's algorithm in
  oracle.c (label propagation, union-find labels, partition bounds, boundary
  sort/dedup, the full distributed merge with its exchange schedule);
* ``_ref/libccref.so`` - the reference's own cc_pthreads.c, boundary_sort.c,
  opt_parser.c and results_writer.c compiled unmodified;
* ``_ref/mpi_cc_benchmark`` - the reference's whole CLI and MPI path
  (cc_mpi.c, exchange_plan.c, graph_dist.c, graph.c, ...) compiled
  unmodified against the fakempi / fakematio shims in this folder; ranks are
  forked processes (``FAKEMPI_NP``).  ``ref_mpi_run`` runs it and parses what
  it prints (per-rank partition sizes and boundary/ghost/plan counts, merge
  rounds, component count, run times).

Both ``_ref`` files are built from the reference sources by
``make -C oracle ref REF=<reference tree>`` (``build(ref_tree=...)``);
prebuilt copies travel with the repository to machines without that tree.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libccref.so")
REF_MPI_BIN = os.path.join(HERE, "_ref", "mpi_cc_benchmark")


class Pair(C.Structure):
    _fields_ = [("rep", C.c_uint32), ("remote", C.c_uint32)]


class DistStats(C.Structure):
    _fields_ = [("rounds", C.c_int), ("exchanges", C.c_int),
                ("boundary_raw", C.c_uint64), ("pair_count", C.c_uint64),
                ("ghost_count", C.c_uint64), ("rep_count", C.c_uint64),
                ("roots", C.c_uint64), ("sent_pairs", C.c_uint64)]


PAIR_DTYPE = np.dtype([("rep", np.uint32), ("remote", np.uint32)])


def build(ref_tree=None):
    """Compile liboracle.so, and the reference-built checkers in _ref/ from
    the reference sources under ``ref_tree`` when that tree is given and
    present (otherwise the prebuilt _ref/ files are used)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref_tree and os.path.isdir(ref_tree):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_tree}"], check=True)


_o = None
_r = None


def olib():
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        vp, u32, u64, i = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
        L.orc_uf_labels.argtypes = [u32, vp, vp, vp]
        L.orc_lp_labels.argtypes = [u32, vp, vp, vp]
        L.orc_lp_labels.restype = i
        L.orc_vertex_range.argtypes = [u32, i, i, C.POINTER(u32), C.POINTER(u32)]
        L.orc_weighted_bounds.argtypes = [vp, u32, i, u32, vp]
        L.orc_owner_of_vertex.argtypes = [u32, u32, i, i, vp]
        L.orc_owner_of_vertex.restype = i
        L.orc_boundary_sort.argtypes = [vp, u64]
        L.orc_boundary_sort.restype = i
        L.orc_boundary_dedup.argtypes = [vp, u64]
        L.orc_boundary_dedup.restype = u64
        L.orc_count_components.argtypes = [vp, u32]
        L.orc_count_components.restype = u32
        L.orc_dist_cc.argtypes = [u32, vp, vp, i, i, i, i, vp, vp, C.POINTER(DistStats)]
        L.orc_dist_cc.restype = i
        L.orc_dist_partition.argtypes = [u32, vp, vp, i, i, i, vp, vp, u64, vp, u64, vp, u64,
                                         vp, vp]
        L.orc_dist_partition.restype = i
        _o = L
    return _o


def rlib():
    """The reference's own code (raises if it was never built)."""
    global _r
    if _r is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} missing; run `make -C oracle ref` where the "
                                    "reference tree is available")
        L = C.CDLL(REF_SO)
        L.boundary_edges_sort.argtypes = [C.c_void_p, C.c_uint64]
        L.boundary_edges_dedup.argtypes = [C.c_void_p, C.c_uint64]
        L.boundary_edges_dedup.restype = C.c_uint64
        _r = L
    return _r


def have_ref():
    return os.path.exists(REF_SO)


def _arr(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def uf_labels(row_ptr, col):
    row_ptr, col = _arr(row_ptr, np.uint64), _arr(col, np.uint32)
    n = len(row_ptr) - 1
    out = np.empty(n, dtype=np.uint32)
    olib().orc_uf_labels(n, row_ptr.ctypes.data, col.ctypes.data, out.ctypes.data)
    return out


def lp_labels(row_ptr, col):
    row_ptr, col = _arr(row_ptr, np.uint64), _arr(col, np.uint32)
    n = len(row_ptr) - 1
    out = np.empty(n, dtype=np.uint32)
    rounds = olib().orc_lp_labels(n, row_ptr.ctypes.data, col.ctypes.data, out.ctypes.data)
    return out, rounds


def weighted_bounds(row_ptr, parts, vertex_weight=1):
    row_ptr = _arr(row_ptr, np.uint64)
    b = np.empty(parts + 1, dtype=np.uint32)
    olib().orc_weighted_bounds(row_ptr.ctypes.data, len(row_ptr) - 1, parts, vertex_weight,
                               b.ctypes.data)
    return b


def vertex_range(n, parts, r):
    s, e = C.c_uint32(), C.c_uint32()
    olib().orc_vertex_range(n, parts, r, C.byref(s), C.byref(e))
    return s.value, e.value


def owner_of_vertex(v, n, parts, kind, bounds=None):
    bp = _arr(bounds, np.uint32).ctypes.data if bounds is not None else None
    return olib().orc_owner_of_vertex(v, n, parts, kind, bp)


def boundary_sort_dedup(pairs):
    """pairs: structured array (rep, remote) -> sorted, deduplicated copy."""
    a = np.array(pairs, dtype=PAIR_DTYPE, copy=True)
    L = olib()
    if L.orc_boundary_sort(a.ctypes.data, len(a)) != 0:
        raise MemoryError("orc_boundary_sort")
    k = L.orc_boundary_dedup(a.ctypes.data, len(a))
    return a[:k]


def ref_boundary_sort_dedup(pairs):
    """The reference's own boundary_edges_sort + boundary_edges_dedup."""
    a = np.array(pairs, dtype=PAIR_DTYPE, copy=True)
    L = rlib()
    L.boundary_edges_sort(a.ctypes.data, len(a))
    k = L.boundary_edges_dedup(a.ctypes.data, len(a))
    return a[:k]


def ref_pthreads_labels(row_ptr, col, threads=4, chunk=4096):
    """The reference's compute_connected_components_pthreads, unmodified."""
    row_ptr, col = _arr(row_ptr, np.uint64), _arr(col, np.uint32)
    n = len(row_ptr) - 1

    class CSR(C.Structure):
        _fields_ = [("n", C.c_uint32), ("m", C.c_uint64), ("row_ptr", C.c_void_p),
                    ("col_idx", C.c_void_p)]

    g = CSR(n, int(row_ptr[-1]), row_ptr.ctypes.data, col.ctypes.data)
    out = np.empty(n, dtype=np.uint32)
    f = rlib().compute_connected_components_pthreads
    f.argtypes = [C.POINTER(CSR), C.c_void_p, C.c_int, C.c_int]
    f.restype = None
    if n:
        f(C.byref(g), out.ctypes.data, threads, chunk)
    return out


def count_components(labels):
    labels = _arr(labels, np.uint32)
    return int(olib().orc_count_components(labels.ctypes.data, len(labels)))


def dist_cc(row_ptr, col, parts, kind=1, interval=1, gauss_seidel=False):
    """Restated distributed CC -> (labels, bounds, stats)."""
    row_ptr, col = _arr(row_ptr, np.uint64), _arr(col, np.uint32)
    n = len(row_ptr) - 1
    labels = np.empty(n, dtype=np.uint32)
    bounds = np.empty(parts + 1, dtype=np.uint32)
    st = DistStats()
    rc = olib().orc_dist_cc(n, row_ptr.ctypes.data, col.ctypes.data if len(col) else None,
                            parts, kind, interval, int(gauss_seidel), labels.ctypes.data,
                            bounds.ctypes.data, C.byref(st))
    if rc != 0:
        raise RuntimeError(f"orc_dist_cc failed ({rc})")
    return labels, bounds, st


def dist_partition(row_ptr, col, parts, kind, p):
    """Per-partition artefacts: dict of comp_of, rep_list, pairs, ghosts, seg."""
    row_ptr, col = _arr(row_ptr, np.uint64), _arr(col, np.uint32)
    n = len(row_ptr) - 1
    m = int(row_ptr[-1])
    comp_of = np.empty(max(n, 1), dtype=np.uint32)
    reps = np.empty(max(n, 1), dtype=np.uint32)
    pairs = np.empty(max(m, 1), dtype=PAIR_DTYPE)
    ghosts = np.empty(max(m, 1), dtype=np.uint32)
    seg = np.empty(parts + 1, dtype=np.uint32)
    sizes = np.zeros(4, dtype=np.uint64)
    rc = olib().orc_dist_partition(n, row_ptr.ctypes.data, col.ctypes.data, parts, kind, p,
                                   comp_of.ctypes.data, reps.ctypes.data, len(reps),
                                   pairs.ctypes.data, len(pairs), ghosts.ctypes.data,
                                   len(ghosts), seg.ctypes.data, sizes.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"orc_dist_partition failed ({rc})")
    b = weighted_bounds(row_ptr, parts) if (kind and parts > 1) else None
    if b is None:
        s, e = vertex_range(n, parts, p)
    else:
        s, e = int(b[p]), int(b[p + 1])
    nl = e - s
    return {"v_start": s, "v_end": e, "comp_of": comp_of[:nl].copy(),
            "rep_list": reps[:int(sizes[0])].copy(), "pairs": pairs[:int(sizes[1])].copy(),
            "ghosts": ghosts[:int(sizes[2])].copy(), "seg": seg.copy(),
            "boundary_raw": int(sizes[3])}


# ------------------------------------------------ the reference's MPI path

def have_ref_mpi():
    return os.path.exists(REF_MPI_BIN)


def write_mat(path, row_ptr, col):
    """A symmetric CSR graph as a MAT level-5 file holding struct Problem
    with sparse logical field A (the layout of the SuiteSparse .mat files
    the reference loads), written by scipy (a writer independent of both
    the product's and the shim's readers)."""
    import scipy.io as sio
    import scipy.sparse as sp
    row_ptr, col = _arr(row_ptr, np.uint64), _arr(col, np.uint32)
    n = len(row_ptr) - 1
    A = sp.csc_matrix((np.ones(len(col), dtype=bool), col.astype(np.int64),
                       row_ptr.astype(np.int64)), shape=(n, n))
    sio.savemat(path, {"Problem": {"A": A}}, do_compression=True)


def write_csrbin(path, row_ptr, col):
    """The CSR binary format (magic CSRB, version 1, n, pad, m, row_ptr
    u64[n+1], col u32[m]); the matio shim serves it as one sparse variable
    when the file is named ``*.mat``, for graphs MAT v5 cannot hold."""
    row_ptr, col = _arr(row_ptr, np.uint64), _arr(col, np.uint32)
    n, m = len(row_ptr) - 1, int(row_ptr[-1])
    with open(path, "wb") as f:
        f.write(b"CSRB")
        f.write(np.array([1, n, 1], dtype=np.uint32).tobytes())
        f.write(np.array([m], dtype=np.uint64).tobytes())
        f.write(memoryview(row_ptr).cast("B"))
        f.write(memoryview(col).cast("B"))


def parse_ref_mpi(text, ranks):
    """What the reference CLI prints (src/mpi_cc_benchmark.c:121-247 and
    src/cc_mpi.c:318-746), per run: per-rank local sizes (n_local gives the
    partition bounds), boundary raw/dedup, ghost and plan counts, rank 0's
    rep count, merge rounds, component count, run time."""
    import re
    runs, cur = [], None
    graph = {}
    for line in text.splitlines():
        mt = re.match(r"Graph loaded \(n=(\d+), m=(\d+)\) in ([0-9.]+) seconds", line)
        if mt:
            graph = {"n": int(mt[1]), "m": int(mt[2]), "load_s": float(mt[3])}
            continue
        mt = re.match(r"\[rank (\d+)\] Local CC done: n_local=(\d+) m_local=(\d+) "
                      r"threads=(\d+)", line)
        if mt:
            if cur is None or int(mt[1]) in cur["n_local"]:
                cur = {"n_local": {}, "m_local": {}, "raw": {}, "dedup": {}, "ghosts": {},
                       "plan": {}, "reps0": None, "rounds": None, "components": None,
                       "seconds": None, "threads": int(mt[4])}
                runs.append(cur)
            cur["n_local"][int(mt[1])] = int(mt[2])
            cur["m_local"][int(mt[1])] = int(mt[3])
            continue
        if cur is None:
            continue
        mt = re.match(r"\[rank 0\] reps=(\d+)", line)
        if mt:
            cur["reps0"] = int(mt[1])
            continue
        mt = re.match(r"\[rank (\d+)\] boundary_edges raw=(\d+) dedup=(\d+)", line)
        if mt:
            cur["raw"][int(mt[1])] = int(mt[2])
            cur["dedup"][int(mt[1])] = int(mt[3])
            continue
        mt = re.match(r"\[rank (\d+)\] ghost_count=(\d+)", line)
        if mt:
            cur["ghosts"][int(mt[1])] = int(mt[2])
            continue
        mt = re.match(r"\[rank (\d+)\] plan indegree=(-?\d+) outdegree=(-?\d+) "
                      r"send=(-?\d+) recv=(-?\d+)", line)
        if mt:
            cur["plan"][int(mt[1])] = tuple(int(mt[k]) for k in range(2, 6))
            continue
        mt = re.match(r"CC merge converged in (\d+) rounds", line)
        if mt:
            cur["rounds"] = int(mt[1])
            continue
        mt = re.match(r"Number of connected components: (\d+)", line)
        if mt:
            cur["components"] = int(mt[1])
            continue
        mt = re.match(r"Run (\d+): ([0-9.]+) seconds", line)
        if mt:
            cur["seconds"] = float(mt[2])
    for r in runs:
        nl = [r["n_local"].get(k, 0) for k in range(ranks)]
        r["bounds"] = [int(x) for x in np.concatenate([[0], np.cumsum(nl)])]
    return {"graph": graph, "runs": runs}


def ref_mpi_run(mat_path, ranks, threads=1, chunk=8192, exchange=1, runs=1, outdir=None,
                timeout=3600, extra_env=None):
    """Runs the reference's own mpi_cc_benchmark (compiled unmodified) at
    ``ranks`` fakempi ranks: ``-t threads -c chunk -e exchange -r runs``.
    Returns the parsed output (``parse_ref_mpi``) plus the raw text."""
    import tempfile
    if not have_ref_mpi():
        raise FileNotFoundError(f"{REF_MPI_BIN} missing; run `make -C oracle ref REF=...` "
                                "where the reference tree is available")
    env = dict(os.environ, FAKEMPI_NP=str(ranks))
    if extra_env:
        env.update(extra_env)
    with tempfile.TemporaryDirectory() as tmp:
        out = outdir or tmp
        cmd = [REF_MPI_BIN, "-t", str(threads), "-c", str(chunk), "-e", str(exchange),
               "-r", str(runs), "-o", out, mat_path]
        p = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"reference mpi_cc_benchmark failed ({p.returncode}): "
                           f"{p.stderr[-2000:]}")
    res = parse_ref_mpi(p.stdout, ranks)
    res["stdout"] = p.stdout
    return res
