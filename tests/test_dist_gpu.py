"""Parity of the partitioned path (ccgpu_dist_cc and the boundary sort) with
the oracle's restatement of the reference's distributed algorithm: labels
bit-exact, and - because both use the same round semantics - the same
round, exchange, pair, ghost and rep counts and the same bounds."""
import numpy as np
import pytest

import oracle
from cc_mpi_b200 import dist, graphs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    t.cuda.set_device(0)
    return t


def dev(torch, rp, col):
    d_rp = torch.from_numpy(rp.astype(np.int64)).cuda()
    d_col = torch.from_numpy(col.astype(np.int32)).cuda() if len(col) else \
        torch.zeros(1, dtype=torch.int32, device="cuda")
    return d_rp, d_col


def run(torch, rp, col, parts, kind, interval, chunk=2048):
    n = len(rp) - 1
    d_rp, d_col = dev(torch, rp, col)
    lab = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    st, bounds = dist.dist_cc_device(d_rp, d_col, n, int(rp[-1]), parts, kind, chunk, interval,
                                     d_labels=lab)
    torch.cuda.synchronize()
    return lab[:n].cpu().numpy().view(np.uint32), st, bounds


def check_against_oracle(torch, rp, col, parts, kind, interval, chunk=2048):
    got, st, bounds = run(torch, rp, col, parts, kind, interval, chunk)
    want, obounds, ost = oracle.dist_cc(rp, col, parts, kind, interval)
    assert (got == want).all()
    assert (bounds == obounds).all()
    assert st.roots == ost.roots
    assert st.boundary_raw == ost.boundary_raw
    assert st.pair_count == ost.pair_count
    assert st.ghost_count == ost.ghost_count
    assert st.rep_count == ost.rep_count
    assert st.rounds == ost.rounds, (st.rounds, ost.rounds)
    assert st.exchanges == ost.exchanges
    assert st.sent_pairs == ost.sent_pairs
    return st


@pytest.mark.parametrize("parts", [1, 2, 3, 4, 7])
@pytest.mark.parametrize("kind", [0, 1])
def test_small_cases(torch, small_cases, parts, kind):
    for name, (rp, col) in small_cases.items():
        if len(rp) - 1 < parts:
            continue
        for interval in (1, 2, 4):
            check_against_oracle(torch, rp, col, parts, kind, interval)


def test_golden_graphs(torch, golden_labels):
    for name, (rp, col, ref) in golden_labels.items():
        if len(rp) - 1 < 4:
            continue
        got, st, _ = run(torch, rp, col, 4, 1, 1)
        assert (got == ref).all(), name


@pytest.mark.parametrize("chunk", [1, 2048, 8192, 32768])
@pytest.mark.parametrize("interval", [1, 2, 4])
def test_rmat_chunks_and_intervals(torch, chunk, interval):
    rp, col = graphs.rmat_csr(14, 16, seed=31)
    st = check_against_oracle(torch, rp, col, 4, 1, interval, chunk)
    assert st.rounds >= 1


def test_grid_partitions(torch):
    rp, col = graphs.grid_csr(256, 256, 0.1, seed=9)
    for parts in (2, 4, 8):
        check_against_oracle(torch, rp, col, parts, 1, 2)


def test_many_partitions_and_er(torch):
    rp, col = graphs.er_csr(30000, 3.0, seed=4)
    for parts in (16, 64):
        check_against_oracle(torch, rp, col, parts, 1, 1)
        check_against_oracle(torch, rp, col, parts, 0, 3)


@pytest.mark.parametrize("parts", [5, 9, 17, 33])
def test_rmat_partition_widths(torch, parts):
    """Every code path by partition count: the partition lookup specialised
    for <= 4 / <= 8 / more partitions, the message scatter over sent
    messages (<= 16) or over all ghosts, and the giant masks (<= 32) or
    plain keys; R-MAT hubs put long rows across column tiles."""
    rp, col = graphs.rmat_csr(13, 16, seed=40 + parts)
    for interval in (1, 3):
        check_against_oracle(torch, rp, col, parts, 1, interval)


def test_unaligned_columns(torch):
    """A column array that starts 4 bytes past a 16-byte boundary takes the
    scalar column loads and gives the same labels and counts."""
    rp, col = graphs.rmat_csr(13, 16, seed=77)
    n, m = len(rp) - 1, len(col)
    d_rp = torch.from_numpy(rp.astype(np.int64)).cuda()
    buf = torch.zeros(m + 4, dtype=torch.int32, device="cuda")
    buf[1:m + 1] = torch.from_numpy(col.astype(np.int32)).cuda()
    d_col = buf[1:m + 1]
    assert d_col.data_ptr() % 16 == 4
    lab = torch.empty(n, dtype=torch.int32, device="cuda")
    st, bounds = dist.dist_cc_device(d_rp, d_col, n, m, 4, 1, 2048, 1, d_labels=lab)
    want, obounds, ost = oracle.dist_cc(rp, col, 4, 1, 1)
    assert (lab.cpu().numpy().view(np.uint32) == want).all()
    assert (bounds == obounds).all()
    assert st.boundary_raw == ost.boundary_raw and st.pair_count == ost.pair_count
    assert st.rounds == ost.rounds and st.sent_pairs == ost.sent_pairs


def test_sorted_row_mode_and_its_fallback(torch):
    """Ascending rows take the partition runs and the sorted-row boundary
    passes; the same graph with its rows shuffled falls back to the local
    CSR build and the gather pass.  A duplicated (mirrored) entry keeps the
    runs: the run counts of the local end see both copies.  Every variant
    matches the oracle."""
    rp, col = graphs.rmat_csr(12, 16, seed=91)
    st = check_against_oracle(torch, rp, col, 4, 1, 1)
    assert st.sorted_rows == 1 and st.row_runs == 1
    rng = np.random.default_rng(3)
    shuffled = col.copy()
    for v in range(len(rp) - 1):
        a, b = int(rp[v]), int(rp[v + 1])
        shuffled[a:b] = rng.permutation(shuffled[a:b])
    st = check_against_oracle(torch, rp, shuffled, 4, 1, 1)
    assert st.sorted_rows == 0 and st.row_runs == 0
    # duplicate the first cut edge found (both directions): rows stay
    # ascending but not strictly
    n = len(rp) - 1
    bounds = np.array(oracle.weighted_bounds(rp, 4), dtype=np.int64)
    part = np.searchsorted(bounds, np.arange(n), side="right") - 1
    src = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    cut = np.nonzero(part[src] != part[col])[0][0]
    u, v = int(src[cut]), int(col[cut])
    rows = [list(col[int(rp[x]):int(rp[x + 1])]) for x in range(n)]
    for a, b in ((u, v), (v, u)):
        rows[a].insert(rows[a].index(b), b)
    rp2 = np.zeros(n + 1, np.uint64)
    rp2[1:] = np.cumsum([len(r) for r in rows])
    col2 = np.array([x for r in rows for x in r], np.uint32)
    st = check_against_oracle(torch, rp2, col2, 4, 1, 1)
    assert st.sorted_rows == 1 and st.row_runs == 1


def test_asymmetric_input_takes_the_gather_pass(torch):
    """The run counts assume a symmetric graph (the reference's input); the
    row scan's symmetry sum catches a cut edge stored in one direction only
    and the pairs are made by the gather pass instead."""
    rp, col = graphs.rmat_csr(12, 16, seed=92)
    n = len(rp) - 1
    bounds = np.array(oracle.weighted_bounds(rp, 4), dtype=np.int64)
    part = np.searchsorted(bounds, np.arange(n), side="right") - 1
    src = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    cut = np.nonzero(part[src] != part[col])[0][:3]
    keep = np.ones(len(col), bool)
    keep[cut] = False
    col2 = col[keep]
    rp2 = np.zeros(n + 1, np.uint64)
    rp2[1:] = np.cumsum(np.bincount(src[keep], minlength=n))
    _, st, _ = run(torch, rp2, col2, 4, 1, 1)
    assert st.sorted_rows == 0 and st.row_runs == 1


@pytest.mark.parametrize("parts", [2, 5, 6, 8])
def test_partition_runs_every_width(torch, parts):
    """Ascending rows with 2 to 8 partitions take the in-place partition
    runs (no local CSR is built); counts and labels are the oracle's."""
    for rp, col in (graphs.rmat_csr(13, 16, seed=101), graphs.grid_csr(120, 90, 0.2, seed=102)):
        st = check_against_oracle(torch, rp, col, parts, 1, 2)
        assert st.sorted_rows == 1


def test_ids_beyond_n_are_ignored(torch):
    """Column ids >= n (the reference skips them, src/cc_mpi.c:269,389) sit
    at the end of ascending rows; the partition runs and the local CSR path
    both leave them out of the local subgraph and of the raw cut count."""
    rp, col = graphs.rmat_csr(12, 16, seed=103)
    n = len(rp) - 1
    rows = [list(col[int(rp[v]):int(rp[v + 1])]) for v in range(n)]
    rng = np.random.default_rng(4)
    for v in rng.choice(n, 300, replace=False):
        rows[v] += sorted(int(x) for x in rng.choice(np.arange(n, n + 50), 2, replace=False))
    rp2 = np.zeros(n + 1, np.uint64)
    rp2[1:] = np.cumsum([len(r) for r in rows])
    col2 = np.array([x for r in rows for x in r], np.uint32)
    for parts in (4, 9):
        check_against_oracle(torch, rp2, col2, parts, 1, 1)


def test_bounds_match_reference_restatement(torch):
    rp, col = graphs.rmat_csr(12, 8, seed=6)
    d_rp, _ = dev(torch, rp, col)
    for parts in (1, 2, 3, 5, 16):
        for kind in (0, 1):
            got = dist.partition_bounds_device(d_rp, len(rp) - 1, parts, kind)
            if kind and parts > 1:
                want = oracle.weighted_bounds(rp, parts)
            else:
                want = np.array([oracle.vertex_range(len(rp) - 1, parts, r)[0]
                                 for r in range(parts)] + [len(rp) - 1], dtype=np.uint32)
            assert (got == want).all(), (parts, kind)


def test_large_rmat_properties(torch):
    rp_d, col_d = graphs.rmat_csr_torch(torch, 20, 16, seed=5)
    n, m = rp_d.numel() - 1, col_d.numel()
    lab = torch.empty(n, dtype=torch.int32, device="cuda")
    st, bounds = dist.dist_cc_device(rp_d, col_d, n, m, 4, 1, 8192, 2, d_labels=lab)
    rp = rp_d.cpu().numpy().view(np.uint64)
    col = col_d.cpu().numpy().view(np.uint32)
    uf = oracle.uf_labels(rp, col)
    assert (lab.cpu().numpy().view(np.uint32) == uf).all()
    assert st.roots == oracle.count_components(uf)


def test_boundary_sort_golden(torch):
    import os
    from conftest import GOLDEN
    d = np.load(os.path.join(GOLDEN, "boundary_sort.npz"))
    for name in d["names"]:
        name = str(name)
        inp = d[f"{name}__in"]
        exp = d[f"{name}__out"]
        if len(inp) == 0:
            continue
        t = torch.from_numpy(inp.view(np.int64).copy()).cuda()
        dist.boundary_sort_device(t, len(inp))
        k = dist.boundary_dedup_device(t, len(inp))
        torch.cuda.synchronize()
        got = t[:k].cpu().numpy().view(np.uint64)
        assert k == len(exp), name
        assert (got == exp).all(), name


def test_boundary_sort_random_bits(torch):
    rng = np.random.default_rng(3)
    for n, rb, gb in [(100000, 20, 24), (70000, 32, 32), (5, 3, 3), (4097, 12, 1)]:
        pairs = np.empty(n, dtype=oracle.PAIR_DTYPE)
        pairs["rep"] = rng.integers(0, 1 << rb, n, dtype=np.uint64)
        pairs["remote"] = rng.integers(0, 1 << gb, n, dtype=np.uint64)
        want = oracle.boundary_sort_dedup(pairs)
        t = torch.from_numpy(pairs.view(np.int64).copy()).cuda()
        dist.boundary_sort_device(t, n, (1 << rb) - 1, (1 << gb) - 1)
        k = dist.boundary_dedup_device(t, n)
        torch.cuda.synchronize()
        assert k == len(want)
        assert (t[:k].cpu().numpy().view(np.uint64) == want.view(np.uint64)).all()


def test_host_and_device_driven_rounds_agree(torch):
    """After its first rounds a merge goes on as one CUDA graph (a while node
    over k_upd, the round bookkeeping and the exchange) unless the
    per-kernel profiler is on, when the host drives every round: both give
    the oracle's labels and the same round, exchange and sent-pair counts -
    on a graph with over a thousand rounds (zigzag), one with a few dozen
    (ER) and one with about ten (R-MAT)."""
    from cc_mpi_b200 import _lib
    L = _lib.lib()
    sc = graphs.small_cases()
    cases = {"zigzag": sc["zigzag"], "er": sc["er2k"], "rmat": graphs.rmat_csr(12, 8, seed=44)}
    for name, (rp, col) in cases.items():
        for parts, interval in ((7, 1), (4, 3)):
            dev_st = check_against_oracle(torch, rp, col, parts, 1, interval)
            _lib.check(L.ccgpu_prof_enable(None, 1))
            try:
                host_st = check_against_oracle(torch, rp, col, parts, 1, interval)
            finally:
                _lib.check(L.ccgpu_prof_enable(None, 0))
            assert dev_st.rounds == host_st.rounds and dev_st.exchanges == host_st.exchanges, name
            assert dev_st.sent_pairs == host_st.sent_pairs, name


@pytest.mark.gpu
def test_ghost_map_and_buckets_agree(torch, monkeypatch):
    """The merge finds a ghost's slot through a direct (partition, id) map
    when parts * n words fit the budget, else through id buckets and a
    binary search; CCGPU_GHOST_MAP_BYTES=0 forces the buckets.  Both give
    the oracle's labels and the same round, exchange and sent-pair counts."""
    sc = graphs.small_cases()
    cases = {"zigzag": sc["zigzag"], "er": sc["er2k"], "rmat": graphs.rmat_csr(12, 8, seed=45)}
    for name, (rp, col) in cases.items():
        for parts, interval in ((3, 1), (8, 2)):
            monkeypatch.delenv("CCGPU_GHOST_MAP_BYTES", raising=False)
            map_st = check_against_oracle(torch, rp, col, parts, 1, interval)
            monkeypatch.setenv("CCGPU_GHOST_MAP_BYTES", "0")
            bucket_st = check_against_oracle(torch, rp, col, parts, 1, interval)
            monkeypatch.delenv("CCGPU_GHOST_MAP_BYTES")
            assert map_st.rounds == bucket_st.rounds, name
            assert map_st.exchanges == bucket_st.exchanges, name
            assert map_st.sent_pairs == bucket_st.sent_pairs, name
