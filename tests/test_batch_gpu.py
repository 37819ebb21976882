"""Batched CC (ccgpu_batch_*): every graph of a packed batch gets exactly the
labels of a single-graph solve - the oracle's labels on small batches, the
plain single-graph kernel's labels on a mixed batch of the bench's shapes -
under every schedule the autotuner can pick, through the eager kernel
sequence and through the CUDA-graph replay."""
import numpy as np
import pytest

import oracle
from cc_mpi_b200 import _lib, batch, cc, graphs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    t.cuda.set_device(0)
    return t


def small_batch(seed=11, count=60):
    """Edge cases (empty graph, single vertex, paths, hubs above the heavy
    threshold, ...) plus seeded ER / R-MAT / grid graphs of random sizes."""
    rng = np.random.default_rng(seed)
    gs = [(np.zeros(1, np.uint64), np.zeros(0, np.uint32))]  # n = 0
    gs += list(graphs.small_cases().values())
    while len(gs) < count:
        k = rng.integers(0, 3)
        n = int(rng.integers(1, 3000))
        if k == 0:
            gs.append(graphs.er_csr(n, float(rng.uniform(0.5, 10)), seed=int(rng.integers(1e9))))
        elif k == 1:
            gs.append(graphs.rmat_csr(int(rng.integers(2, 12)), 8, seed=int(rng.integers(1e9))))
        else:
            gs.append(graphs.grid_csr(int(rng.integers(1, 60)), int(rng.integers(1, 60)),
                                      float(rng.uniform(0, 0.6)), seed=int(rng.integers(1e9))))
    return gs


def to_device(torch, gs):
    vo, eo, rp, col = batch.pack(gs)
    d_rp = torch.from_numpy(rp.astype(np.int64)).cuda()
    d_col = torch.from_numpy(col.astype(np.int32)).cuda() if len(col) else \
        torch.zeros(1, dtype=torch.int32, device="cuda")
    d_lab = torch.full((max(int(vo[-1]), 1),), -1, dtype=torch.int32, device="cuda")
    return vo, eo, d_rp, d_col, d_lab


def check_oracle(torch, gs, vo, d_lab, comps=None, done=None):
    lab = d_lab.cpu().numpy().view(np.uint32)
    for g, (rp, col) in enumerate(gs):
        want = oracle.uf_labels(rp, col)
        got = batch.labels_of(lab, vo, g)
        assert (got == want).all(), g
        if comps is not None:
            assert comps[g] == oracle.count_components(want), g
    if done is not None:
        assert (done == 1).all()


def tuning_with(**kw):
    t = batch.default_tuning()
    for c in range(batch.CLASSES):
        for k, v in kw.items():
            if k == "heavy_degree":
                t.heavy_degree = v
            else:
                setattr(t.cls[c], k, v)
    return t


def test_small_batch_matches_oracle_eager_and_graph(torch):
    gs = small_batch()
    vo, eo, d_rp, d_col, d_lab = to_device(torch, gs)
    plan = batch.BatchPlan(vo, eo, d_rp, d_col, d_lab)
    assert plan.class_graphs().sum() == len(gs)
    plan.run()
    comps, done = plan.results()
    check_oracle(torch, gs, vo, d_lab, comps, done)
    for _ in range(2):  # graph replays start from a dirty label array
        d_lab.fill_(-7)
        plan.launch()
        torch.cuda.synchronize()
        comps, done = plan.results()
        check_oracle(torch, gs, vo, d_lab, comps, done)
    assert plan.kernels() > 0
    plan.close()


SCHEDULES = [dict(sample_rounds=0), dict(sample_rounds=1, cadence=0),
             dict(sample_rounds=3, cadence=1, tile=256), dict(sample_rounds=4, cadence=0,
                                                              tile=65536),
             dict(warp_degree=2), dict(warp_degree=1024, tile=1024),
             dict(heavy_degree=32, warp_degree=8), dict(heavy_degree=32, sample_rounds=0)]


@pytest.mark.parametrize("sched", SCHEDULES, ids=[str(s) for s in SCHEDULES])
def test_schedules_match_oracle(torch, sched):
    gs = small_batch(seed=23, count=40)
    vo, eo, d_rp, d_col, d_lab = to_device(torch, gs)
    plan = batch.BatchPlan(vo, eo, d_rp, d_col, d_lab, tuning=tuning_with(**sched))
    plan.launch()
    comps, done = plan.results()
    check_oracle(torch, gs, vo, d_lab, comps, done)
    plan.close()


def test_one_shot_call(torch):
    """ccgpu_batch_cc reuses its context's plan from call to call: batches
    that grow, shrink and change tuning all get the oracle's labels."""
    import ctypes as C
    L = batch._bind()
    cases = [(5, 20, None), (6, 70, tuning_with(sample_rounds=3, cadence=1)),
             (7, 10, None), (8, 90, tuning_with(sample_rounds=0))]
    for seed, count, tun in cases:
        gs = small_batch(seed=seed, count=count)
        vo, eo, d_rp, d_col, d_lab = to_device(torch, gs)
        b = batch.Batch()
        b.graphs = len(gs)
        b.h_vtx_off = vo.ctypes.data_as(C.POINTER(C.c_uint64))
        b.h_edge_off = eo.ctypes.data_as(C.POINTER(C.c_uint64))
        b.d_row_ptr, b.d_col, b.d_labels = d_rp.data_ptr(), d_col.data_ptr(), d_lab.data_ptr()
        comps = np.zeros(len(gs), np.uint32)
        _lib.check(L.ccgpu_batch_cc(None, C.byref(b), C.byref(tun) if tun else None,
                                    comps.ctypes.data, torch.cuda.current_stream().cuda_stream))
        check_oracle(torch, gs, vo, d_lab, comps)


def test_rejects_bad_offsets(torch):
    import ctypes as C
    L = batch._bind()
    vo = np.array([0, 5, 3], np.uint64)
    eo = np.array([0, 0, 0], np.uint64)
    d = torch.zeros(16, dtype=torch.int64, device="cuda")
    b = batch.Batch()
    b.graphs = 2
    b.h_vtx_off = vo.ctypes.data_as(C.POINTER(C.c_uint64))
    b.h_edge_off = eo.ctypes.data_as(C.POINTER(C.c_uint64))
    b.d_row_ptr, b.d_col, b.d_labels = d.data_ptr(), d.data_ptr(), d.data_ptr()
    p = C.c_void_p()
    assert L.ccgpu_batch_plan_create(None, C.byref(b), None, C.byref(p)) == 1
    t = tuning_with(tile=1000)  # not a power of two
    vo[2] = 7
    assert L.ccgpu_batch_plan_create(None, C.byref(b), C.byref(t), C.byref(p)) == 1


def test_mixed_batch_matches_plain_kernel_and_autotune(torch):
    spec = batch.mix_spec(graphs=90, n_min=1000, n_max=150_000, seed=3)
    vo, eo, d_rp, d_col, kinds = batch.build_batch_torch(torch, spec)
    G = len(spec)
    d_lab = torch.full((int(vo[-1]),), -1, dtype=torch.int32, device="cuda")
    want = torch.empty_like(d_lab)
    for g in range(G):
        a, b = int(vo[g]), int(vo[g + 1])
        n, m = b - a, int(eo[g + 1] - eo[g])
        cc.local_cc_device(d_rp[a + g:], d_col[int(eo[g]):] if m else d_col, n, m,
                           want[a:b] if n else want)
    plan = batch.BatchPlan(vo, eo, d_rp, d_col, d_lab)
    assert (plan.class_graphs() > 0).all()  # all three degree classes present
    plan.launch()
    torch.cuda.synchronize()
    assert torch.equal(d_lab, want)
    t = plan.autotune()
    for c in range(batch.CLASSES):
        o = t.cls[c]
        assert 0 <= o.sample_rounds <= 4 and o.tile in (1024, 4096, 16384)
    d_lab.fill_(-1)
    plan.launch()
    torch.cuda.synchronize()
    assert torch.equal(d_lab, want)
    comps, done = plan.results()
    assert (done == 1).all()
    # spot-check a few graphs against the oracle too
    lab = d_lab.cpu().numpy().view(np.uint32)
    rp_h = d_rp.cpu().numpy().view(np.uint64)
    col_h = d_col.cpu().numpy().view(np.uint32)
    for g in (0, 1, 2, G // 2, G - 1):
        a = int(vo[g])
        n = int(vo[g + 1]) - a
        rp = rp_h[a + g:a + g + n + 1]
        col = col_h[int(eo[g]):int(eo[g + 1])]
        ref = oracle.uf_labels(rp, col)
        assert (batch.labels_of(lab, vo, g) == ref).all(), g
        assert comps[g] == oracle.count_components(ref)
    plan.close()


def persistent(t=None, **kw):
    t = t or batch.default_tuning()
    t.persistent = 1
    for k, v in kw.items():
        setattr(t, k, v)
    return t


@pytest.mark.parametrize("sched", SCHEDULES[:6], ids=[str(s) for s in SCHEDULES[:6]])
def test_persistent_launch_matches_oracle(torch, sched):
    """One persistent launch per class (work items in phase order, per-graph
    phase counters) gives every graph the oracle's labels, replay after
    replay, under the schedules the autotuner can pick."""
    gs = small_batch(seed=29, count=50)
    vo, eo, d_rp, d_col, d_lab = to_device(torch, gs)
    plan = batch.BatchPlan(vo, eo, d_rp, d_col, d_lab,
                           tuning=persistent(tuning_with(**sched)))
    for _ in range(2):
        d_lab.fill_(-3)
        plan.launch()
        comps, done = plan.results()
        check_oracle(torch, gs, vo, d_lab, comps, done)
    assert plan.kernels() <= batch.CLASSES
    plan.close()


def test_persistent_mixed_batch_matches_phase_launches(torch):
    spec = batch.mix_spec(graphs=120, n_min=1000, n_max=200_000, seed=5)
    vo, eo, d_rp, d_col, kinds = batch.build_batch_torch(torch, spec)
    d_a = torch.full((int(vo[-1]),), -1, dtype=torch.int32, device="cuda")
    d_b = torch.full_like(d_a, -2)
    plan_a = batch.BatchPlan(vo, eo, d_rp, d_col, d_a)
    plan_b = batch.BatchPlan(vo, eo, d_rp, d_col, d_b, tuning=persistent(heavy_degree=256))
    plan_a.launch()
    plan_b.launch()
    torch.cuda.synchronize()
    assert torch.equal(d_a, d_b)
    comps_a, _ = plan_a.results()
    comps_b, done_b = plan_b.results()
    assert (comps_a == comps_b).all() and (done_b == 1).all()
    lab = d_b.cpu().numpy().view(np.uint32)
    for g in range(0, len(spec), 17):
        a, n = int(vo[g]), int(vo[g + 1] - vo[g])
        rp = d_rp[a + g:a + g + n + 1].cpu().numpy().view(np.uint64)
        col = d_col[int(eo[g]):int(eo[g + 1])].cpu().numpy().view(np.uint32)
        assert (batch.labels_of(lab, vo, g) == oracle.uf_labels(rp, col)).all(), g
    plan_a.close()
    plan_b.close()


def test_persistent_wait_runs_out_and_reports(torch):
    """A graph whose first wait can never be met (the stall_graph test aid):
    the bounded wait runs out after wait_ms, the launch ends, the results
    call returns CCGPU_ERR_TIMEOUT, and the same plan solves the batch
    afterwards once the aid is off."""
    import ctypes as C
    gs = small_batch(seed=31, count=30)
    vo, eo, d_rp, d_col, d_lab = to_device(torch, gs)
    stalled = next(g for g in range(len(gs)) if vo[g + 1] > vo[g])
    L = batch._bind()
    plan = batch.BatchPlan(vo, eo, d_rp, d_col, d_lab,
                           tuning=persistent(wait_ms=50, stall_graph=stalled))
    plan.launch()
    torch.cuda.synchronize()
    comps = np.zeros(len(gs), np.uint32)
    done = np.zeros(len(gs), np.uint32)
    rc = L.ccgpu_batch_plan_results(plan.p, comps.ctypes.data, done.ctypes.data,
                                    torch.cuda.current_stream().cuda_stream)
    assert rc == 4  # CCGPU_ERR_TIMEOUT
    assert done[stalled] == 0
    plan.close()
    plan = batch.BatchPlan(vo, eo, d_rp, d_col, d_lab, tuning=persistent(wait_ms=50))
    plan.launch()
    comps2, done2 = plan.results()
    check_oracle(torch, gs, vo, d_lab, comps2, done2)
    plan.close()
