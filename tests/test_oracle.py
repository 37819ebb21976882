"""The CPU oracle, pinned against fixtures the reference's own code produced
(tests/golden/make_golden.py), and its distributed restatement checked
against independent labellings."""
import json
import os

import numpy as np
import pytest

import oracle
from cc_mpi_b200 import graphs

from conftest import GOLDEN


def test_golden_labels_union_find(golden_labels):
    for name, (rp, col, ref) in golden_labels.items():
        assert (oracle.uf_labels(rp, col) == ref).all(), name


def test_golden_labels_label_propagation(golden_labels):
    for name, (rp, col, ref) in golden_labels.items():
        lp, rounds = oracle.lp_labels(rp, col)
        assert (lp == ref).all(), name
        assert rounds >= 1


def test_golden_labels_are_min_ids(golden_labels):
    for name, (rp, col, ref) in golden_labels.items():
        n = len(rp) - 1
        v = np.arange(n, dtype=np.uint32)
        assert (ref <= v).all(), name
        assert (ref[ref] == ref).all(), name


def test_golden_boundary_sort():
    d = np.load(os.path.join(GOLDEN, "boundary_sort.npz"))
    for name in d["names"]:
        name = str(name)
        inp = d[f"{name}__in"].view(oracle.PAIR_DTYPE)
        exp = d[f"{name}__out"].view(oracle.PAIR_DTYPE)
        got = oracle.boundary_sort_dedup(inp)
        assert len(got) == len(exp), name
        assert (got.view(np.uint64) == exp.view(np.uint64)).all(), name


@pytest.mark.parametrize("parts", [1, 2, 3, 4, 7])
@pytest.mark.parametrize("kind", [0, 1])
def test_dist_restatement_matches_union_find(small_cases, parts, kind):
    for name, (rp, col) in small_cases.items():
        n = len(rp) - 1
        if n < parts:
            continue
        uf = oracle.uf_labels(rp, col)
        for interval in (1, 2, 4):
            for gs in (False, True):
                lab, bounds, st = oracle.dist_cc(rp, col, parts, kind, interval, gs)
                assert (lab == uf).all(), (name, parts, kind, interval, gs)
                assert st.roots == oracle.count_components(uf)
                assert bounds[0] == 0 and bounds[-1] == n
                assert (np.diff(bounds.astype(np.int64)) >= 0).all()


def test_dist_round_count_depends_on_interval_not_labels():
    rp, col = graphs.rmat_csr(11, 8, seed=21)
    uf = oracle.uf_labels(rp, col)
    rounds = {}
    for interval in (1, 2, 4, 8):
        lab, _, st = oracle.dist_cc(rp, col, 4, 1, interval)
        assert (lab == uf).all()
        rounds[interval] = (st.rounds, st.exchanges)
    assert rounds[1][1] >= 1


def test_weighted_bounds_edge_cases():
    # more parts than a balanced split would give: clamps keep every part non-empty
    rp = np.array([0, 100, 100, 100, 100, 100], dtype=np.uint64)
    b = oracle.weighted_bounds(rp, 4)
    assert list(b) == sorted(b) and b[0] == 0 and b[-1] == 5
    assert (np.diff(b.astype(np.int64)) >= 1).all()
    # every partition non-empty for n == parts
    rp = np.arange(0, 9, 2, dtype=np.uint64)
    b = oracle.weighted_bounds(rp, 4)
    assert list(b) == [0, 1, 2, 3, 4]


def test_owner_of_vertex_agrees_with_bounds():
    rp, col = graphs.rmat_csr(10, 8, seed=2)
    n = len(rp) - 1
    for parts in (2, 3, 4, 5):
        b = oracle.weighted_bounds(rp, parts)
        for v in range(0, n, 7):
            q = oracle.owner_of_vertex(v, n, parts, 1, b)
            assert b[q] <= v < b[q + 1]
        for v in range(0, n, 5):
            q = oracle.owner_of_vertex(v, n, parts, 0)
            s, e = oracle.vertex_range(n, parts, q)
            assert s <= v < e


def test_reference_pthreads_agrees_when_present(small_cases):
    if not oracle.have_ref():
        pytest.skip("reference checker not built on this machine")
    for name, (rp, col) in small_cases.items():
        assert (oracle.ref_pthreads_labels(rp, col, 3, 7) == oracle.uf_labels(rp, col)).all()


def test_opt_parser_golden_is_consistent():
    with open(os.path.join(GOLDEN, "opt_parser.json")) as f:
        d = json.load(f)
    for r in d["range_lists"]:
        if r["rc"] == 0:
            assert r["values"] == sorted(set(r["values"]))
