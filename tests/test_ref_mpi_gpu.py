"""The GPU partitioned path against the reference's own MPI path run here.

The same .mat file goes to the reference's unmodified mpi_cc_benchmark
(oracle/_ref, fakempi ranks, one pthread per rank) and to this library:
through the device API (ccgpu_dist_cc) and through this repository's CLI
(cc_mpi_b200/bin/mpi_cc_benchmark, the reference's flags and CSV layout).
Partition bounds, the totals of the per-rank boundary / dedup / ghost
counts the reference prints, and the component count must be identical;
the labels must equal the reference's cc_pthreads labels.  Round counts:
the reference's one-thread merge is Gauss-Seidel and the GPU's is Jacobi;
each equals the oracle's restatement of its order."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from cc_mpi_b200 import dist, graphs

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.have_ref_mpi(),
                                 reason="reference MPI build (oracle/_ref) absent")]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "cc_mpi_b200", "bin", "mpi_cc_benchmark")
ENV = {"FAKEMPI_TIMEOUT_S": "120"}


@pytest.fixture(scope="module")
def torch():
    import torch as t
    t.cuda.set_device(0)
    return t


def _cases():
    return {
        "rmat14": graphs.rmat_csr(14, 16, seed=41),
        "rmat16": graphs.rmat_csr(16, 8, seed=42),
        "grid": graphs.grid_csr(160, 120, 0.1, seed=43),
        "grid_sparse": graphs.grid_csr(90, 90, 0.45, seed=44),
    }


CASES = _cases()


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("ranks", [2, 4])
def test_device_path_matches_reference_mpi(torch, tmp_path, name, ranks):
    rp, col = CASES[name]
    n, m = len(rp) - 1, int(rp[-1])
    path = str(tmp_path / f"{name}.mat")
    oracle.write_mat(path, rp, col)
    res = oracle.ref_mpi_run(path, ranks, threads=1, chunk=8192, exchange="1,2,4",
                             extra_env=ENV)
    ref_labels = oracle.ref_pthreads_labels(rp, col, 4, 8192)
    d_rp = torch.from_numpy(rp.astype(np.int64)).cuda()
    d_col = torch.from_numpy(col.astype(np.int32)).cuda()
    lab = torch.empty(n, dtype=torch.int32, device="cuda")
    for interval, run in zip((1, 2, 4), res["runs"]):
        st, bounds = dist.dist_cc_device(d_rp, d_col, n, m, ranks, 1, 8192, interval,
                                         d_labels=lab)
        torch.cuda.synchronize()
        got = lab.cpu().numpy().view(np.uint32)
        assert (got == ref_labels).all()
        assert [int(x) for x in bounds] == run["bounds"]
        assert st.roots == run["components"]
        assert st.boundary_raw == sum(run["raw"].values())
        assert st.pair_count == sum(run["dedup"].values())
        assert st.ghost_count == sum(run["ghosts"].values())
        _, _, jac = oracle.dist_cc(rp, col, ranks, 1, interval)
        _, _, gs = oracle.dist_cc(rp, col, ranks, 1, interval, gauss_seidel=True)
        assert st.rounds == jac.rounds and st.exchanges == jac.exchanges
        assert run["rounds"] == gs.rounds


def test_cli_prints_what_the_reference_prints(tmp_path):
    """Both CLIs on one .mat with the same sweep: the same component count
    and round count lines per configuration where the orders agree, the same
    CSV file name and column names."""
    rp, col = CASES["rmat14"]
    path = str(tmp_path / "rmat14.mat")
    oracle.write_mat(path, rp, col)
    ref_out = tmp_path / "ref"
    res = oracle.ref_mpi_run(path, 4, threads=1, chunk="2048,8192", exchange="1,2", runs=2,
                             outdir=str(ref_out), extra_env=ENV)
    ours_out = tmp_path / "ours"
    p = subprocess.run([CLI, "-p", "4", "-c", "2048,8192", "-e", "1,2", "-r", "2", "-o",
                        str(ours_out), path], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    comps = [int(x) for x in re.findall(r"Number of connected components: (\d+)", p.stdout)]
    assert comps and set(comps) == {r["components"] for r in res["runs"]}
    ref_csv = (ref_out / "results_mpi_rmat14.csv").read_text().splitlines()
    our_csv = (ours_out / "results_mpi_rmat14.csv").read_text().splitlines()
    assert ref_csv[0] == our_csv[0]  # chunk_<c>_exchange_<e> columns, same order
    assert len(ref_csv) == len(our_csv) == 3
