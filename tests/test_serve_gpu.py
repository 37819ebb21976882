"""Request server (ccgpu_server_*): every request's labels are the oracle's
and the same as when the request is served alone, while requests that
arrive during other batches are admitted, batched together and overlap
them on the device; admission waits for pool memory and refuses graphs that
can never fit."""
import threading
import time

import numpy as np
import pytest

import oracle
from cc_mpi_b200 import _lib, graphs, serve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    t.cuda.set_device(0)
    return t


def request_mix(seed=3, count=120):
    rng = np.random.default_rng(seed)
    cases = list(graphs.small_cases().values())
    out = [(np.zeros(1, np.uint64), np.zeros(0, np.uint32))] + cases
    while len(out) < count:
        k = rng.integers(0, 3)
        if k == 0:
            out.append(graphs.er_csr(int(rng.integers(10, 20000)), 8.0,
                                     seed=int(rng.integers(1e9))))
        elif k == 1:
            out.append(graphs.rmat_csr(int(rng.integers(4, 14)), 16, seed=int(rng.integers(1e9))))
        else:
            out.append(graphs.grid_csr(int(rng.integers(2, 120)), int(rng.integers(2, 120)),
                                       0.1, seed=int(rng.integers(1e9))))
    return out


def test_mix_matches_oracle_and_alone(torch):
    reqs = request_mix()
    big = graphs.rmat_csr(17, 16, seed=99)  # keeps the first batch busy while others arrive
    srv = serve.Server(hbm_bytes=1 << 30, max_batch=32, streams=2)
    results = {}
    t_big = srv.submit(*big)

    def client(idx):
        rng = np.random.default_rng(idx)
        for i in range(idx, len(reqs), 3):
            t = srv.submit(*reqs[i])
            results[i] = t
            time.sleep(float(rng.uniform(0, 0.0005)))

    th = [threading.Thread(target=client, args=(k,)) for k in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    got = {}
    for i, t in results.items():
        lab, info = srv.wait(t, timeout=120)
        assert info.status == 0
        got[i] = (lab.copy(), info.components, info.batch_graphs)
    lab_big, info_big = srv.wait(t_big, timeout=120)
    st = srv.stats()
    srv.close()
    assert (lab_big == oracle.uf_labels(*big)).all()
    assert st.completed == len(reqs) + 1 and st.batches >= 2
    assert st.max_batch_seen > 1, "requests were never batched together"
    assert st.max_in_flight >= 2, "no batch overlapped another on the device"
    for i, (rp, col) in enumerate(reqs):
        want = oracle.uf_labels(rp, col)
        assert (got[i][0] == want).all(), i
        assert got[i][1] == oracle.count_components(want), i
    # the same requests one at a time (one slot, one graph per batch)
    alone = serve.Server(hbm_bytes=1 << 28, max_batch=1, streams=1)
    for i, (rp, col) in enumerate(reqs):
        lab, info = alone.wait(alone.submit(rp, col), timeout=60)
        assert info.batch_graphs == (1 if len(rp) > 1 else 0)
        assert (lab == got[i][0]).all(), i
    assert alone.stats().max_in_flight <= 1
    alone.close()


def test_admission_waits_for_pool_memory(torch):
    g = graphs.er_csr(30000, 8.0, seed=5)  # about 1.3 MB of CSR + labels
    srv = serve.Server(hbm_bytes=4 << 20, max_batch=64, streams=2)  # room for 2-3 at a time
    ts = [srv.submit(*g) for _ in range(24)]
    want = oracle.uf_labels(*g)
    for t in ts:
        lab, info = srv.wait(t, timeout=120)
        assert (lab == want).all()
        assert info.t_admit >= info.t_submit and info.t_done >= info.t_start >= info.t_admit
    st = srv.stats()
    assert st.pool_peak <= st.pool_bytes
    assert st.batches >= 8  # never more than a few resident: many batches
    srv.close()


def test_rejects_graph_larger_than_pool(torch):
    srv = serve.Server(hbm_bytes=1 << 20)
    g = graphs.er_csr(200000, 4.0, seed=1)
    with pytest.raises(_lib.CCGPUError) as e:
        srv.submit(*g)
    assert e.value.status == 5  # CCGPU_ERR_LIMIT
    # the server still serves graphs that fit
    t = srv.submit(*graphs.er_csr(1000, 4.0, seed=2))
    lab, info = srv.wait(t, timeout=60)
    assert info.status == 0
    srv.close()
