"""Seeded synthetic graphs in the shapes the reference is benchmarked on.

The reference's own benchmark graph (com-Friendster) is not available, so
every workload is a seeded synthetic stand-in with the same shape:

* R-MAT (a=0.57, b=0.19, c=0.19, d=0.05), ``edge_factor * 2**scale`` edge
  samples, vertex ids scrambled by a seeded permutation (the Graph500
  convention) so that hubs are not clustered at low ids;
* 2-D 4-neighbour grids with a fraction of edges deleted uniformly;
* Erdos-Renyi graphs with a given average degree.

All graphs are returned as symmetric CSR (``row_ptr`` uint64[n+1], ``col_idx``
uint32[m]) with self loops and duplicate edges removed and every row sorted -
the input contract of the reference (its loader does neither, src/graph.c:17-18,
so inputs must already be symmetric).  numpy builders serve the CPU tests;
the ``*_torch`` builders make the large bench graphs directly in HBM.
"""
from __future__ import annotations

import numpy as np

RMAT_ABC = (0.57, 0.19, 0.19)


# --------------------------------------------------------------------- numpy


def csr_from_edges(n: int, src: np.ndarray, dst: np.ndarray):
    """Symmetrise, drop self loops and duplicates, sort rows -> CSR."""
    src = np.asarray(src, dtype=np.uint64)
    dst = np.asarray(dst, dtype=np.uint64)
    keep = src != dst
    s = np.concatenate([src[keep], dst[keep]])
    d = np.concatenate([dst[keep], src[keep]])
    key = np.unique((s << np.uint64(32)) | d)
    s = (key >> np.uint64(32)).astype(np.int64)
    col = (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    counts = np.bincount(s, minlength=n).astype(np.uint64)
    row_ptr = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(counts, out=row_ptr[1:])
    return row_ptr, col


def rmat_edges(scale: int, edge_factor: int = 16, seed: int = 1, abc=RMAT_ABC, permute=True):
    rng = np.random.default_rng(seed)
    m = edge_factor << scale
    a, b, c = abc
    src = np.zeros(m, dtype=np.uint64)
    dst = np.zeros(m, dtype=np.uint64)
    for lvl in range(scale):
        r = rng.random(m)
        sbit = r >= a + b
        dbit = ((r >= a) & (r < a + b)) | (r >= a + b + c)
        src |= sbit.astype(np.uint64) << np.uint64(lvl)
        dst |= dbit.astype(np.uint64) << np.uint64(lvl)
    if permute:
        perm = rng.permutation(1 << scale).astype(np.uint64)
        src, dst = perm[src], perm[dst]
    return src, dst


def rmat_csr(scale: int, edge_factor: int = 16, seed: int = 1, permute=True):
    s, d = rmat_edges(scale, edge_factor, seed, permute=permute)
    return csr_from_edges(1 << scale, s, d)


def grid_csr(rows: int, cols: int, p_delete: float = 0.1, seed: int = 1):
    """rows x cols 4-neighbour grid, row-major ids, each edge deleted with
    probability p_delete."""
    rng = np.random.default_rng(seed)
    ids = np.arange(rows * cols, dtype=np.uint64).reshape(rows, cols)
    h_keep = rng.random((rows, cols - 1)) >= p_delete
    v_keep = rng.random((rows - 1, cols)) >= p_delete
    src = np.concatenate([ids[:, :-1][h_keep], ids[:-1, :][v_keep]])
    dst = np.concatenate([ids[:, 1:][h_keep], ids[1:, :][v_keep]])
    return csr_from_edges(rows * cols, src, dst)


def er_csr(n: int, avg_degree: float = 8.0, seed: int = 1):
    rng = np.random.default_rng(seed)
    m = int(n * avg_degree / 2)
    src = rng.integers(0, n, m, dtype=np.uint64)
    dst = rng.integers(0, n, m, dtype=np.uint64)
    return csr_from_edges(n, src, dst)


def small_cases():
    """Hand-made graphs covering the edge cases the parity tests walk:
    empty, singletons, a path, a star, two components, isolated vertices,
    a long path (high diameter), hubs above the warp and heavy thresholds,
    and ids arranged so the min id of a component is far from its hub."""
    cases = {}

    def add(name, n, edges):
        e = np.asarray(edges, dtype=np.uint64).reshape(-1, 2)
        cases[name] = csr_from_edges(n, e[:, 0], e[:, 1])

    add("single", 1, [])
    add("isolated4", 4, [])
    add("pair", 2, [(0, 1)])
    add("path8", 8, [(i, i + 1) for i in range(7)])
    add("rpath8", 8, [(7 - i, 6 - i) for i in range(7)])
    add("star9", 9, [(4, i) for i in range(9) if i != 4])
    add("two_comps", 10, [(0, 2), (2, 4), (4, 6), (1, 3), (3, 5), (5, 7), (8, 9)])
    add("tri_iso", 6, [(1, 2), (2, 3), (3, 1)])
    add("long_path", 5000, [(i, i + 1) for i in range(4999)])
    # zig-zag path: consecutive ids are far apart along the path
    zz = [i // 2 if i % 2 == 0 else 2999 - i // 2 for i in range(3000)]
    add("zigzag", 3000, [(zz[i], zz[i + 1]) for i in range(2999)])
    rng = np.random.default_rng(7)
    # hub of degree 20000 plus a second component with a 300-degree hub
    hub = [(17, int(v)) for v in rng.choice(np.arange(40000, 60000), 20000, replace=False)]
    hub2 = [(30001, 30002 + i) for i in range(300)]
    add("hubs", 60000, hub + hub2 + [(5, 6)])
    cases["rmat10"] = rmat_csr(10, 16, seed=3)
    cases["rmat12"] = rmat_csr(12, 8, seed=4)
    cases["grid64"] = grid_csr(64, 64, 0.3, seed=5)
    cases["grid_sparse"] = grid_csr(40, 50, 0.55, seed=6)
    cases["er2k"] = er_csr(2000, 1.2, seed=8)
    return cases


def to_undirected_count(row_ptr: np.ndarray) -> int:
    return int(row_ptr[-1]) // 2


# --------------------------------------------------------------------- torch


def _csr_from_keys_torch(torch, n, key):
    """key: sorted unique int64 (src << 32 | dst) on the device."""
    src = key >> 32
    col = (key & 0xFFFFFFFF).to(torch.int32)
    counts = torch.bincount(src, minlength=n)
    row_ptr = torch.zeros(n + 1, dtype=torch.int64, device=key.device)
    torch.cumsum(counts, 0, out=row_ptr[1:])
    return row_ptr, col


def symmetric_csr_torch(torch, n, src, dst):
    keep = src != dst
    src, dst = src[keep], dst[keep]
    key = torch.cat([(src << 32) | dst, (dst << 32) | src])
    del src, dst, keep
    key = torch.unique(key, sorted=True)
    return _csr_from_keys_torch(torch, n, key)


def rmat_csr_torch(torch, scale, edge_factor=16, seed=1, device="cuda", abc=RMAT_ABC,
                   n=None, samples=None):
    """R-MAT on the device.  ``n`` < 2**scale truncates the id space after a
    seeded permutation (used for non-power-of-two vertex counts)."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    m = samples if samples is not None else edge_factor << scale
    a, b, c = abc
    src = torch.zeros(m, dtype=torch.int64, device=device)
    dst = torch.zeros(m, dtype=torch.int64, device=device)
    for lvl in range(scale):
        r = torch.rand(m, generator=g, device=device)
        src |= (r >= a + b).to(torch.int64) << lvl
        dst |= (((r >= a) & (r < a + b)) | (r >= a + b + c)).to(torch.int64) << lvl
        del r
    perm = torch.randperm(1 << scale, generator=g, device=device)
    src = perm[src]
    dst = perm[dst]
    del perm
    nv = (1 << scale) if n is None else n
    if nv < (1 << scale):
        keep = (src < nv) & (dst < nv)
        src, dst = src[keep], dst[keep]
    return symmetric_csr_torch(torch, nv, src, dst)


def _sort_unique_keys(torch, keys, bits):
    """Sorted distinct values of a device int64 tensor, through the library's
    radix sort (ccgpu_sort_keys / ccgpu_unique_keys)."""
    import ctypes as C
    from . import _lib
    L = _lib.lib()
    L.ccgpu_sort_keys.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_int,
                                  C.POINTER(C.c_int), C.c_void_p]
    L.ccgpu_unique_keys.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                    C.POINTER(C.c_uint64), C.c_void_p]
    n = keys.numel()
    alt = torch.empty_like(keys)
    in_alt = C.c_int(0)
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(L.ccgpu_sort_keys(None, keys.data_ptr(), alt.data_ptr(), n, bits, C.byref(in_alt),
                                 st))
    src, dst = (alt, keys) if in_alt.value else (keys, alt)
    cnt = C.c_uint64(0)
    _lib.check(L.ccgpu_unique_keys(None, src.data_ptr(), n, dst.data_ptr(), C.byref(cnt), st))
    del src
    return dst[:cnt.value]


def rmat_csr_big(torch, scale, n, target_undirected, seed=1, device="cuda", abc=RMAT_ABC,
                 chunk=1 << 27, keep_estimate=0.87):
    """Large R-MAT graph built chunk by chunk on the device: ids over 2**scale
    permuted by a seeded permutation and truncated to [0, n); enough samples
    for about `target_undirected` distinct undirected edges (the exact count
    is whatever remains after dropping self loops and duplicates).  Returns
    (row_ptr int64[n+1], col int32[m]) with sorted rows."""
    assert n <= (1 << scale) and n < (1 << 31)
    bits = max(1, (n - 1).bit_length())
    mask = (1 << bits) - 1
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    perm = torch.randperm(1 << scale, generator=g, device=device)
    a, b, c = abc
    samples = int(target_undirected / keep_estimate)
    keys = torch.empty(samples, dtype=torch.int64, device=device)
    w = 0
    for start in range(0, samples, chunk):
        cnt = min(chunk, samples - start)
        src = torch.zeros(cnt, dtype=torch.int64, device=device)
        dst = torch.zeros(cnt, dtype=torch.int64, device=device)
        for lvl in range(scale):
            r = torch.rand(cnt, generator=g, device=device)
            src |= (r >= a + b).to(torch.int64) << lvl
            dst |= (((r >= a) & (r < a + b)) | (r >= a + b + c)).to(torch.int64) << lvl
            del r
        src, dst = perm[src], perm[dst]
        keep = (src < n) & (dst < n) & (src != dst)
        lo = torch.minimum(src, dst)[keep]
        hi = torch.maximum(src, dst)[keep]
        del src, dst, keep
        k = (lo << bits) | hi
        keys[w:w + k.numel()] = k
        w += k.numel()
        del lo, hi, k
    del perm
    und = _sort_unique_keys(torch, keys[:w], 2 * bits).clone()
    del keys
    both = torch.empty(2 * und.numel(), dtype=torch.int64, device=device)
    both[:und.numel()] = und
    both[und.numel():] = ((und & mask) << bits) | (und >> bits)
    del und
    both = _sort_unique_keys(torch, both, 2 * bits)
    col = (both & mask).to(torch.int32)
    counts = torch.zeros(n, dtype=torch.int64, device=device)
    for start in range(0, both.numel(), chunk):
        counts += torch.bincount(both[start:start + chunk] >> bits, minlength=n)
    del both
    row_ptr = torch.zeros(n + 1, dtype=torch.int64, device=device)
    torch.cumsum(counts, 0, out=row_ptr[1:])
    return row_ptr, col


def grid_csr_torch(torch, rows, cols, p_delete=0.1, seed=1, device="cuda"):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    n = rows * cols
    h = torch.rand((rows, cols - 1), generator=g, device=device) >= p_delete
    v = torch.rand((rows - 1, cols), generator=g, device=device) >= p_delete
    # candidate neighbours in sorted order: up, left, right, down
    ids = torch.arange(n, dtype=torch.int64, device=device).view(rows, cols)
    valid = torch.zeros((rows, cols, 4), dtype=torch.bool, device=device)
    valid[1:, :, 0] = v
    valid[:, 1:, 1] = h
    valid[:, :-1, 2] = h
    valid[:-1, :, 3] = v
    del h, v
    counts = valid.view(n, 4).sum(1)
    row_ptr = torch.zeros(n + 1, dtype=torch.int64, device=device)
    torch.cumsum(counts, 0, out=row_ptr[1:])
    del counts
    off = torch.tensor([-cols, -1, 1, cols], dtype=torch.int64, device=device)
    nb = ids.view(n, 1) + off.view(1, 4)
    col = nb[valid.view(n, 4)].to(torch.int32)
    return row_ptr, col


def er_csr_torch(torch, n, avg_degree=8.0, seed=1, device="cuda"):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    m = int(n * avg_degree / 2)
    src = torch.randint(0, n, (m,), generator=g, device=device, dtype=torch.int64)
    dst = torch.randint(0, n, (m,), generator=g, device=device, dtype=torch.int64)
    return symmetric_csr_torch(torch, n, src, dst)
