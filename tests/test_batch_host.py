"""Host-side batch logic (no GPU): the packed CSR-of-CSRs layout and the
batched workload's size and type mix."""
import math

import numpy as np

from cc_mpi_b200 import batch, graphs


def test_pack_layout():
    gs = [graphs.er_csr(50, 3.0, seed=1), (np.zeros(1, np.uint64), np.zeros(0, np.uint32)),
          graphs.grid_csr(4, 5, 0.0, seed=2), graphs.rmat_csr(5, 4, seed=3)]
    vo, eo, rp, col = batch.pack(gs)
    assert vo[0] == 0 and eo[0] == 0 and len(vo) == len(gs) + 1
    assert len(rp) == vo[-1] + len(gs) and len(col) == eo[-1]
    for g, (r, c) in enumerate(gs):
        n = len(r) - 1
        assert vo[g + 1] - vo[g] == n and eo[g + 1] - eo[g] == len(c)
        a = int(vo[g]) + g
        assert (rp[a:a + n + 1] == r).all()
        assert (col[int(eo[g]):int(eo[g + 1])] == c).all()


def test_mix_spec_shape():
    spec = batch.mix_spec(graphs=4096, seed=7)
    assert len(spec) == 4096
    ns = np.array([n for _, n, _ in spec])
    assert ns.min() >= 1000 and ns.max() <= 2_000_000
    # log-uniform: the median sits near the geometric mean of the range
    assert abs(math.log(np.median(ns)) - 0.5 * math.log(1000 * 2e6)) < 0.3
    kinds = [k for k, _, _ in spec]
    for k in ("er", "rmat", "grid"):
        assert abs(kinds.count(k) - 4096 / 3) <= 1
    assert spec == batch.mix_spec(graphs=4096, seed=7)  # seeded
