"""The reference's own MPI path, run here, pins the oracle's restatement of
the partitioned algorithm.

oracle/_ref/mpi_cc_benchmark is the reference's CLI and everything it calls
(src/mpi_cc_benchmark.c, cc_mpi.c, exchange_plan.c, graph_dist.c, graph.c,
cc_pthreads.c, boundary_sort.c, ...) compiled unmodified against the
fakempi / fakematio shims in oracle/.  What it prints per rank - local sizes
(src/cc_mpi.c:318), boundary raw and dedup counts (:417), ghost counts
(:461), plan degrees and sizes (:471) - and in total - merge rounds (:713),
component count (:742) - is compared with the oracle (oracle.c), which the
GPU path is compared with in tests/test_dist_gpu.py and
tests/test_ref_mpi_gpu.py.

With one pthread per rank (-t 1) the reference's merge update walks the
reps in order and reads labels written earlier in the same round
(src/cc_mpi.c:575-622, Gauss-Seidel), so its round count is deterministic
and equals the oracle's Gauss-Seidel restatement; the GPU rounds are
Jacobi and equal the oracle's Jacobi mode."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from cc_mpi_b200 import graphs

pytestmark = pytest.mark.skipif(not oracle.have_ref_mpi(),
                                reason="reference MPI build (oracle/_ref) absent")

ENV = {"FAKEMPI_TIMEOUT_S": "120"}


def _grid(rows, cols, p, seed):
    rng = np.random.default_rng(seed)
    ids = np.arange(rows * cols).reshape(rows, cols)
    e = [np.stack([ids[:, :-1].ravel(), ids[:, 1:].ravel()], 1),
         np.stack([ids[:-1, :].ravel(), ids[1:, :].ravel()], 1)]
    e = np.concatenate(e)
    e = e[rng.random(len(e)) >= p]
    return _csr_from_edges(rows * cols, e)


def _csr_from_edges(n, e):
    u = np.concatenate([e[:, 0], e[:, 1]])
    v = np.concatenate([e[:, 1], e[:, 0]])
    key = np.unique(u.astype(np.uint64) * n + v)
    u, v = key // n, key % n
    rp = np.zeros(n + 1, dtype=np.uint64)
    np.add.at(rp, u.astype(np.int64) + 1, 1)
    return np.cumsum(rp).astype(np.uint64), v.astype(np.uint32)


def _cases():
    out = {}
    out["rmat12"] = graphs.rmat_csr(12, 8, seed=5)
    out["rmat13"] = graphs.rmat_csr(13, 16, seed=7)
    out["grid48"] = _grid(48, 48, 0.1, 3)
    # many components: a grid with 45% of edges gone (long thin pieces)
    out["grid40_sparse"] = _grid(40, 40, 0.45, 11)
    return out


CASES = _cases()


def _mat(tmp_path, name):
    path = str(tmp_path / f"{name}.mat")
    if not os.path.exists(path):
        oracle.write_mat(path, *CASES[name])
    return path


def _expected_partition_stats(rp, col, parts):
    """Per-partition counts the reference prints, from the oracle."""
    P = [oracle.dist_partition(rp, col, parts, 1, p) for p in range(parts)]
    n = len(rp) - 1
    out = {"raw": [], "dedup": [], "ghosts": [], "m_local": [], "plan": [], "reps": []}
    need = np.zeros((parts, parts), dtype=np.int64)  # need[p][q]: ghosts p reads from q
    for p, d in enumerate(P):
        seg = d["seg"].astype(np.int64)
        for q in range(parts):
            need[p, q] = seg[q + 1] - seg[q] if q != p else 0
    for p, d in enumerate(P):
        s, e = d["v_start"], d["v_end"]
        rows = col[int(rp[s]):int(rp[e])]
        out["m_local"].append(int(((rows >= s) & (rows < e)).sum()))
        out["raw"].append(d["boundary_raw"])
        out["dedup"].append(len(d["pairs"]))
        out["ghosts"].append(len(d["ghosts"]))
        out["reps"].append(len(d["rep_list"]))
        ind = int((need[p] > 0).sum())
        outd = int((need[:, p] > 0).sum())
        out["plan"].append((ind, outd, int(need[:, p].sum()), int(need[p].sum())))
    assert n == P[-1]["v_end"]
    return out


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("ranks", [2, 3, 4])
def test_reference_mpi_matches_oracle(tmp_path, name, ranks):
    rp, col = CASES[name]
    res = oracle.ref_mpi_run(_mat(tmp_path, name), ranks, threads=1, chunk=64, exchange="1,2,4",
                             extra_env=ENV)
    n, m = len(rp) - 1, int(rp[-1])
    assert res["graph"]["n"] == n and res["graph"]["m"] == m
    assert len(res["runs"]) == 3
    want_labels = oracle.uf_labels(rp, col)
    comps = oracle.count_components(want_labels)
    bounds = [int(x) for x in oracle.weighted_bounds(rp, ranks)]
    ps = _expected_partition_stats(rp, col, ranks)
    for interval, run in zip((1, 2, 4), res["runs"]):
        assert run["components"] == comps
        assert run["bounds"] == bounds
        for r in range(ranks):
            assert run["raw"][r] == ps["raw"][r]
            assert run["dedup"][r] == ps["dedup"][r]
            assert run["ghosts"][r] == ps["ghosts"][r]
            assert run["m_local"][r] == ps["m_local"][r]
            assert run["plan"][r] == ps["plan"][r], (r, run["plan"][r], ps["plan"][r])
        assert run["reps0"] == ps["reps"][0]
        _, obounds, gs = oracle.dist_cc(rp, col, ranks, 1, interval, gauss_seidel=True)
        assert [int(x) for x in obounds] == bounds
        assert run["rounds"] == gs.rounds, (name, ranks, interval, run["rounds"], gs.rounds)
        assert gs.roots == comps


def test_reference_mpi_threads_and_chunks(tmp_path):
    """Several pthreads per rank (the threaded update is racy in its round
    count, not in its result) and the chunk sweep: the component count is
    the oracle's in every run."""
    rp, col = CASES["rmat13"]
    comps = oracle.count_components(oracle.uf_labels(rp, col))
    res = oracle.ref_mpi_run(_mat(tmp_path, "rmat13"), 4, threads=4, chunk="1,64,8192",
                             exchange=2, runs=2, extra_env=ENV)
    assert len(res["runs"]) == 6
    assert all(r["components"] == comps for r in res["runs"])
    assert all(r["seconds"] is not None and r["seconds"] > 0 for r in res["runs"])


def test_reference_reads_csrbin_through_the_matio_shim(tmp_path):
    """The CSR binary file (for graphs MAT v5 cannot hold) named *.mat gives
    the same run as the MAT file."""
    rp, col = CASES["grid48"]
    p = str(tmp_path / "grid48_bin.mat")
    oracle.write_csrbin(p, rp, col)
    a = oracle.ref_mpi_run(p, 2, extra_env=ENV)["runs"][0]
    b = oracle.ref_mpi_run(_mat(tmp_path, "grid48"), 2, extra_env=ENV)["runs"][0]
    for k in ("components", "rounds", "bounds", "raw", "dedup", "ghosts", "plan"):
        assert a[k] == b[k], k


def test_reference_failure_ends_every_rank(tmp_path):
    """A load error on rank 0 (src/mpi_cc_benchmark.c:181-186) aborts the
    whole job with a non-zero status instead of leaving ranks waiting."""
    bad = tmp_path / "missing.mat"
    p = subprocess.run([oracle.REF_MPI_BIN, "-o", str(tmp_path), str(bad)],
                       env=dict(os.environ, FAKEMPI_NP="3", FAKEMPI_TIMEOUT_S="30"),
                       capture_output=True, text=True, timeout=60)
    assert p.returncode != 0
    assert "Error loading graph" in p.stderr
