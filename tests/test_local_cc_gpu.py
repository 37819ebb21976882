"""Parity of the local-CC kernels (ccgpu_local_cc*, compute_connected_components
_pthreads) with the oracle: bit-exact labels on every case and option."""
import ctypes as C

import numpy as np
import pytest

import oracle
from cc_mpi_b200 import _lib, cc, graphs

pytestmark = pytest.mark.gpu

OPTION_GRID = [
    dict(chunk_size=4096, sample_rounds=2, heavy_degree=8192, skip_giant=1),
    dict(chunk_size=1, sample_rounds=2, heavy_degree=8192, skip_giant=1),      # static
    dict(chunk_size=2048, sample_rounds=0, heavy_degree=8192, skip_giant=0),   # no sampling
    dict(chunk_size=32768, sample_rounds=1, heavy_degree=64, skip_giant=1),    # heavy queue
    dict(chunk_size=100, sample_rounds=4, heavy_degree=33, skip_giant=0),      # odd chunk
    dict(chunk_size=8192, sample_rounds=8, heavy_degree=100000, skip_giant=1),
]
# every hook mode (first hook / lazy hook / cadence) on two schedules
OPTION_GRID += [dict(chunk_size=c, sample_rounds=r, heavy_degree=64, skip_giant=1, hook_mode=h)
                for h in range(16) for c, r in ((4096, 2), (1, 3))]


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    t.cuda.set_device(0)
    return t


def to_dev(torch, rp, col):
    d_rp = torch.from_numpy(rp.astype(np.int64)).cuda()
    d_col = torch.from_numpy(col.astype(np.int32)).cuda() if len(col) else \
        torch.zeros(1, dtype=torch.int32, device="cuda")
    return d_rp, d_col


def solve_dev(torch, rp, col, opts=None, stats=False):
    n = len(rp) - 1
    d_rp, d_col = to_dev(torch, rp, col)
    d_lab = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    st = cc.local_cc_device(d_rp, d_col, n, int(rp[-1]), d_lab, opts, stats=stats)
    torch.cuda.synchronize()
    lab = d_lab[:n].cpu().numpy().view(np.uint32)
    return (lab, st) if stats else lab


def test_golden_fixtures_device(torch, golden_labels):
    for name, (rp, col, ref) in golden_labels.items():
        for o in OPTION_GRID:
            lab = solve_dev(torch, rp, col, _lib.opts(**o))
            assert (lab == ref).all(), (name, o)


def test_golden_fixtures_host_path(golden_labels):
    for name, (rp, col, ref) in golden_labels.items():
        assert (cc.local_cc_host(rp, col) == ref).all(), name
        assert (cc.compute_connected_components_pthreads(rp, col, 8, 8192) == ref).all(), name
        assert (cc.compute_connected_components_pthreads(rp, col, 8, 1) == ref).all(), name


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_graphs_all_options(torch, seed):
    cases = [graphs.rmat_csr(14, 16, seed=seed), graphs.grid_csr(300, 200, 0.3, seed=seed),
             graphs.er_csr(50000, 1.5, seed=seed), graphs.rmat_csr(13, 4, seed=seed,
                                                                    permute=False)]
    for rp, col in cases:
        uf = oracle.uf_labels(rp, col)
        for o in OPTION_GRID:
            lab, st = solve_dev(torch, rp, col, _lib.opts(**o), stats=True)
            assert (lab == uf).all(), o
            assert st.components == oracle.count_components(uf)


def test_stats_fields(torch):
    rp, col = graphs.rmat_csr(14, 16, seed=9)
    uf = oracle.uf_labels(rp, col)
    lab, st = solve_dev(torch, rp, col, _lib.opts(heavy_degree=64), stats=True)
    assert (lab == uf).all()
    # the root picked after sampling lies in the largest component
    assert uf[st.giant_label] == np.bincount(uf).argmax()
    assert st.kernels >= 6
    assert st.finish_rows <= len(rp) - 1
    lab, st = solve_dev(torch, rp, col, _lib.opts(sample_rounds=0, skip_giant=0,
                                                   heavy_degree=64), stats=True)
    assert st.giant_label == 0xFFFFFFFF
    assert st.finish_rows == len(rp) - 1 and st.finish_edges == int(rp[-1])
    deg = np.diff(rp.astype(np.int64))
    assert st.heavy_rows == int((deg > 64).sum())


def test_unaligned_pointers(torch):
    """Column and label arrays that do not start on 16 bytes take the scalar
    paths and give the same labels."""
    rp, col = graphs.rmat_csr(12, 16, seed=5)
    n, m = len(rp) - 1, int(rp[-1])
    uf = oracle.uf_labels(rp, col)
    d_rp = torch.from_numpy(rp.astype(np.int64)).cuda()
    d_colbuf = torch.zeros(m + 3, dtype=torch.int32, device="cuda")
    d_colbuf[1:m + 1] = torch.from_numpy(col.astype(np.int32)).cuda()
    d_labbuf = torch.zeros(n + 3, dtype=torch.int32, device="cuda")
    for o in OPTION_GRID[:3]:
        cc.local_cc_device(d_rp.data_ptr(), d_colbuf.data_ptr() + 4, n, m,
                           d_labbuf.data_ptr() + 4, _lib.opts(**o))
        torch.cuda.synchronize()
        lab = d_labbuf[1:n + 1].cpu().numpy().view(np.uint32)
        assert (lab == uf).all(), o


def test_out_of_range_neighbours_are_ignored(torch):
    rp = np.array([0, 2, 4, 5, 6], dtype=np.uint64)
    col = np.array([1, 999, 0, 4000000000, 3, 2], dtype=np.uint32)
    lab = solve_dev(torch, rp, col)
    assert list(lab) == [0, 0, 2, 2]


def test_empty_and_error_statuses(torch):
    L = _lib.lib()
    assert L.ccgpu_local_cc(None, None, None, 0, 0, None, None, None, None) == 0
    rc = L.ccgpu_local_cc(None, None, None, 5, 0, None, None, None, None)
    assert rc == 1 and b"NULL" in L.ccgpu_last_error()
    bad = _lib.opts(sample_rounds=9)
    rp, col = graphs.rmat_csr(8, 4, seed=1)
    with pytest.raises(_lib.CCGPUError):
        solve_dev(torch, rp, col, bad)


def test_large_rmat_properties(torch):
    """Size-independent properties at a size the oracle still checks fast."""
    rp_d, col_d = graphs.rmat_csr_torch(torch, 20, 16, seed=77)
    n, m = rp_d.numel() - 1, col_d.numel()
    lab = torch.empty(n, dtype=torch.int32, device="cuda")
    st = cc.local_cc_device(rp_d, col_d, n, m, lab, stats=True)
    assert cc.check_labels_device(rp_d, col_d, n, m, lab) == 0
    uf = oracle.uf_labels(rp_d.cpu().numpy().view(np.uint64), col_d.cpu().numpy().view(np.uint32))
    assert st.components == oracle.count_components(uf)
    assert (lab.cpu().numpy().view(np.uint32) == uf).all()


def test_grid_high_diameter(torch):
    rp_d, col_d = graphs.grid_csr_torch(torch, 1024, 1024, 0.1, seed=3)
    n, m = rp_d.numel() - 1, col_d.numel()
    lab = torch.empty(n, dtype=torch.int32, device="cuda")
    cc.local_cc_device(rp_d, col_d, n, m, lab)
    torch.cuda.synchronize()
    uf = oracle.uf_labels(rp_d.cpu().numpy().view(np.uint64), col_d.cpu().numpy().view(np.uint32))
    assert (lab.cpu().numpy().view(np.uint32) == uf).all()


def test_profiler_and_launch_counter(torch):
    L = _lib.lib()
    rp, col = graphs.rmat_csr(12, 8, seed=4)
    before = L.ccgpu_ctx_launches(None)
    _lib.check(L.ccgpu_prof_enable(None, 1))
    solve_dev(torch, rp, col)
    k = L.ccgpu_prof_kernels()
    ms = (C.c_double * k)()
    cnt = (C.c_uint64 * k)()
    _lib.check(L.ccgpu_prof_collect(None, ms, cnt))
    _lib.check(L.ccgpu_prof_enable(None, 0))
    names = [L.ccgpu_prof_name(i).decode() for i in range(k)]
    got = {names[i]: cnt[i] for i in range(k) if cnt[i]}
    # default schedule: one sampling launch per sampled neighbour (cadence)
    assert got.get("sample") == 2 and got.get("link_rows") == 1
    assert L.ccgpu_ctx_launches(None) - before == sum(cnt)


def test_final_shortcut_race_regression(torch):
    """Long paths and tile-boundary vertices under every hook mode and
    schedule, repeated: a plain halving store once put an intermediate
    ancestor back over a root pointer written in the final shortcut pass."""
    cases = [graphs.csr_from_edges(20000, np.arange(19999), np.arange(1, 20000)),
             graphs.small_cases()["zigzag"], graphs.small_cases()["long_path"]]
    for rp, col in cases:
        uf = oracle.uf_labels(rp, col)
        for hm in range(16):
            for ch, sr in ((1, 0), (256, 0), (2048, 2), (4096, 1)):
                for _ in range(3):
                    lab = solve_dev(torch, rp, col, _lib.opts(chunk_size=ch, sample_rounds=sr,
                                                               hook_mode=hm))
                    assert (lab == uf).all(), (hm, ch, sr)


def test_plan_replays_match(torch):
    """The CUDA-graph plan gives the same labels on every replay."""
    L = _lib.lib()
    rp, col = graphs.rmat_csr(14, 16, seed=12)
    n, m = len(rp) - 1, int(rp[-1])
    d_rp, d_col = to_dev(torch, rp, col)
    lab = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    uf = oracle.uf_labels(rp, col)
    for o in (None, _lib.opts(chunk_size=1, hook_mode=5)):
        plan = C.c_void_p()
        _lib.check(L.ccgpu_local_cc_plan(d_rp.data_ptr(), d_col.data_ptr(), n, m,
                                         lab.data_ptr(), C.byref(o) if o else None,
                                         C.byref(plan)))
        assert L.ccgpu_plan_kernels(plan) >= 6
        for _ in range(3):
            lab.fill_(-1)
            _lib.check(L.ccgpu_plan_launch(plan, torch.cuda.current_stream().cuda_stream))
            torch.cuda.synchronize()
            assert (lab.cpu().numpy().view(np.uint32) == uf).all()
        L.ccgpu_plan_destroy(plan)
