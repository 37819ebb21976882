"""The partition-per-rank merge protocol (cc_mpi_b200/multi.py) with one
partition per process over gloo: world size 2, 3 and 4 on CPU.

Each rank's partition is a small numpy engine built from the oracle's
per-partition artefacts (local components, reps, deduplicated boundary
pairs, ghosts - oracle.dist_partition, the restatement of
src/cc_mpi.c:252-461).  Its merge round is the reference's INIT / HOOK /
UPD (src/cc_mpi.c:547-622, MAX_JUMPS = 4) in Jacobi order, the order of
the GPU solver, so the protocol's round, exchange and sent-pair counts must
equal the oracle's Jacobi restatement and the final labels the union-find
labels.  The engine is test scaffolding; what is under test is the
protocol: plan build by all_to_all, the delta exchange (pack below
prev_sent, counts, pairs, scatter) and the OR-reduced termination flags."""
import os
import socket

import numpy as np
import pytest

import oracle
from cc_mpi_b200 import graphs


class NumpyPartition:
    """One partition's merge state (src/cc_mpi.c:326-487), numpy arrays."""

    def __init__(self, rp, col, parts, p):
        d = oracle.dist_partition(rp, col, parts, 1, p)
        self.p, self.parts = p, parts
        self.v_start, self.v_end = d["v_start"], d["v_end"]
        self.comp_of = d["comp_of"].astype(np.int64)
        self.reps = d["rep_list"].astype(np.int64)
        self.pair_rep = d["pairs"]["rep"].astype(np.int64)
        self.pair_g = d["pairs"]["remote"].astype(np.int64)
        self.ghosts = d["ghosts"].astype(np.int64)
        self.seg = d["seg"].astype(np.int64)
        self.label = self.v_start + np.arange(self.v_end - self.v_start, dtype=np.int64)
        self.ghost_labels = self.ghosts.copy()
        self.send_to, self.prev_sent = None, None

    def has_work(self):
        return len(self.ghosts) > 0 and len(self.pair_rep) > 0 and len(self.reps) > 0

    def need_from(self, world):
        return [self.ghosts[self.seg[q]:self.seg[q + 1]].astype(np.uint32) if q != self.p
                else np.zeros(0, np.uint32) for q in range(world)]

    def set_send_to(self, lists):
        self.send_to = [x.astype(np.int64) for x in lists]
        self.prev_sent = [np.full(len(x), 0xFFFFFFFF, np.int64) for x in lists]

    def _label_of(self, x, cur):
        """get_vertex_label_global (src/cc_mpi.c:78-115) over arrays."""
        y = np.full(len(x), -1, np.int64)
        loc = (x >= self.v_start) & (x < self.v_end)
        y[loc] = cur[self.comp_of[x[loc] - self.v_start]]
        gi = np.searchsorted(self.ghosts, x)
        hit = ~loc & (gi < len(self.ghosts))
        hit[hit] = self.ghosts[gi[hit]] == x[hit]
        y[hit] = self.ghost_labels[gi[hit]]
        return y, loc | hit

    def round(self):
        cur = self.label.copy()
        cmin = cur.copy()
        np.minimum.at(cmin, self.pair_rep, self.ghost_labels[self.pair_g])
        x = cmin[self.reps]
        active = np.ones(len(x), bool)
        for _ in range(4):
            y, ok = self._label_of(x, cur)
            step = active & ok & (y >= 0) & (y < x)
            x = np.where(step, y, x)
            active = step
        new = np.minimum(cmin[self.reps], x)
        lower = new < cur[self.reps]
        self.label[self.reps[lower]] = new[lower]
        return bool(lower.any())

    def pack(self):
        out = []
        for q, ids in enumerate(self.send_to):
            if not len(ids):
                out.append(np.zeros(0, np.uint64))
                continue
            lbl = self.label[self.comp_of[ids - self.v_start]]
            go = lbl < self.prev_sent[q]
            self.prev_sent[q][go] = lbl[go]
            pos = np.nonzero(go)[0].astype(np.uint64)
            out.append((pos << np.uint64(32)) | lbl[go].astype(np.uint64))
        return out

    def scatter(self, src, msgs):
        pos = (msgs >> np.uint64(32)).astype(np.int64)
        lbl = (msgs & np.uint64(0xFFFFFFFF)).astype(np.int64)
        self.ghost_labels[self.seg[src] + pos] = lbl

    def roots(self):
        li = np.arange(self.v_end - self.v_start)
        return int((self.label[self.comp_of] == self.v_start + li).sum())

    def final_labels(self):
        return self.label[self.comp_of]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, case, interval, out_dir):
    import torch
    import torch.distributed as dist
    import datetime
    from cc_mpi_b200 import multi
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rp, col = CASES[case]()
        eng = NumpyPartition(rp, col, world, rank)
        res = multi.merge(eng, dist, torch, interval)
        np.save(os.path.join(out_dir, f"labels_{rank}.npy"), eng.final_labels())
        np.save(os.path.join(out_dir, f"stats_{rank}.npy"),
                np.array([res["rounds"], res["exchanges"], res["sent_pairs"],
                          res["components"]], np.int64))
    finally:
        dist.destroy_process_group()


CASES = {
    "rmat11": lambda: graphs.rmat_csr(11, 16, seed=61),
    "grid": lambda: graphs.grid_csr(40, 30, 0.3, seed=62),
    "path": lambda: graphs.small_cases()["long_path"],
}


@pytest.mark.parametrize("case,world,interval", [
    ("rmat11", 2, 1), ("rmat11", 2, 3), ("rmat11", 3, 2), ("rmat11", 4, 1),
    ("grid", 2, 1), ("grid", 4, 2), ("path", 3, 1)])
def test_partition_per_rank_protocol(tmp_path, case, world, interval):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(world, _free_port(), case, interval, str(tmp_path)),
                       nprocs=world, start_method="spawn")
    rp, col = CASES[case]()
    want, _, ost = oracle.dist_cc(rp, col, world, 1, interval)
    got = np.concatenate([np.load(tmp_path / f"labels_{r}.npy") for r in range(world)])
    assert (got.astype(np.uint32) == want).all()
    stats = [np.load(tmp_path / f"stats_{r}.npy") for r in range(world)]
    for s in stats:
        assert s[0] == ost.rounds and s[1] == ost.exchanges
        assert s[3] == ost.roots == oracle.count_components(oracle.uf_labels(rp, col))
    assert sum(int(s[2]) for s in stats) == ost.sent_pairs
