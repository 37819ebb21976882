"""The reference's per-rank exchange plan (include/exchange_plan.h) run as
one host thread per rank on a partition group: plan lists, the delta
exchange's prev_sent rule (src/exchange_plan.c:325-357) and the legacy full
exchange.  Host-only: no GPU involved."""
import ctypes as C
import threading

import numpy as np
import pytest

from cc_mpi_b200 import _lib, graphs

U32P = C.POINTER(C.c_uint32)
INTP = C.POINTER(C.c_int)
OWNER_FN = C.CFUNCTYPE(C.c_int, C.c_uint32, C.c_uint32, C.c_int)


class ExchangePlan(C.Structure):
    _fields_ = [("comm_size", C.c_int), ("comm_rank", C.c_int), ("indegree", C.c_int),
                ("outdegree", C.c_int), ("sources", INTP), ("dests", INTP),
                ("comm_graph", C.c_void_p), ("need_from_counts", INTP),
                ("send_to_counts", INTP), ("need_from_displs", INTP),
                ("send_to_displs", INTP), ("need_from_flat", U32P), ("send_to_flat", U32P),
                ("need_from_gidx_flat", U32P), ("total_need_from", C.c_int),
                ("total_send_to", C.c_int), ("sendcounts", INTP), ("sdispls", INTP),
                ("recvcounts", INTP), ("rdispls", INTP), ("send_labels_flat", U32P),
                ("recv_labels_flat", U32P)]


@pytest.fixture(scope="module")
def L():
    L = _lib.lib()
    vp = C.c_void_p
    _lib.declare("cc_group_create", vp, [C.c_int])
    _lib.declare("cc_group_free", None, [vp])
    _lib.declare("cc_group_view", vp, [vp, C.c_int])
    _lib.declare("ccb200_set_exit_on_error", C.c_int, [C.c_int])
    _lib.declare("exchangeplan_build", C.c_int, [C.POINTER(ExchangePlan), vp, C.c_uint32,
                                                 C.c_uint32, vp, OWNER_FN])
    _lib.declare("exchangeplan_free", None, [C.POINTER(ExchangePlan)])
    _lib.declare("exchangeplan_exchange_delta", None,
                 [C.POINTER(ExchangePlan), vp, vp, C.c_uint32, C.c_uint32, vp, vp, vp,
                  C.POINTER(C.POINTER(C.c_uint64)), INTP, C.POINTER(C.POINTER(C.c_uint64)),
                  INTP])
    _lib.declare("exchangeplan_exchange", None, [C.POINTER(ExchangePlan), vp, vp])
    L.ccb200_set_exit_on_error(0)
    return L


def arr(p, n):
    return np.ctypeslib.as_array(p, shape=(n,)).copy() if n else np.zeros(0, np.uint32)


def setup(P=4, n=3000, seed=2):
    rp, col = graphs.er_csr(n, 5.0, seed=seed)
    bounds = [n * r // P for r in range(P)] + [n]
    ghosts = []
    for r in range(P):
        lo, hi = bounds[r], bounds[r + 1]
        nb = col[int(rp[lo]):int(rp[hi])]
        ghosts.append(np.unique(nb[(nb < lo) | (nb >= hi)]).astype(np.uint32))
    return rp, col, bounds, ghosts


def run_ranks(P, fn):
    errs = []

    def wrap(r):
        try:
            fn(r)
        except Exception as e:  # pragma: no cover - reported below
            errs.append(e)

    th = [threading.Thread(target=wrap, args=(r,)) for r in range(P)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=120)
    assert not errs, errs


def test_plan_delta_and_legacy_exchange(L):
    P, n = 4, 3000
    rp, col, bounds, ghosts = setup(P, n)
    grp = L.cc_group_create(P)
    owner = OWNER_FN(lambda v, ng, size: int(np.searchsorted(bounds, v, side="right") - 1))
    plans = [ExchangePlan() for _ in range(P)]
    state = {}

    def rank(r):
        view = L.cc_group_view(grp, r)
        g = ghosts[r]
        assert L.exchangeplan_build(C.byref(plans[r]), g.ctypes.data, len(g), n, view,
                                    owner) == 0
        pl = plans[r]
        lo, hi = bounds[r], bounds[r + 1]
        comp_of = np.arange(hi - lo, dtype=np.uint32)          # every vertex its own rep
        comp_label = np.arange(lo, hi, dtype=np.uint32)        # label = own id
        prev = np.full(max(pl.total_send_to, 1), 0xFFFFFFFF, np.uint32)
        glab = np.full(max(len(g), 1), 0xFFFFFFFF, np.uint32)
        sb, sc = C.POINTER(C.c_uint64)(), C.c_int(0)
        rb, rc = C.POINTER(C.c_uint64)(), C.c_int(0)

        def delta():
            L.exchangeplan_exchange_delta(C.byref(pl), comp_label.ctypes.data,
                                          comp_of.ctypes.data, lo, hi, prev.ctypes.data,
                                          glab.ctypes.data, view, C.byref(sb), C.byref(sc),
                                          C.byref(rb), C.byref(rc))

        delta()  # everything is below UINT32_MAX: all labels travel
        first = glab[:len(g)].copy()
        # lower the label of every third vertex to 7: only those travel
        comp_label[::3] = np.minimum(comp_label[::3], 7)
        delta()
        second = glab[:len(g)].copy()
        delta()  # nothing changed since: ghost labels stay
        third = glab[:len(g)].copy()
        sent_after = prev[:pl.total_send_to].copy()
        # legacy full exchange of send_labels_flat
        send_to = arr(pl.send_to_flat, pl.total_send_to)
        if pl.total_send_to:
            lbl = np.where((send_to >= lo) & (send_to < hi),
                           comp_label[np.clip(send_to - lo, 0, hi - lo - 1)], send_to)
            lbl32 = np.ascontiguousarray(lbl, dtype=np.uint32)  # alive across the copy
            C.memmove(pl.send_labels_flat, lbl32.ctypes.data, 4 * len(lbl32))
        glab2 = np.zeros(max(len(g), 1), np.uint32)
        L.exchangeplan_exchange(C.byref(pl), glab2.ctypes.data, view)
        state[r] = dict(first=first, second=second, third=third, legacy=glab2[:len(g)].copy(),
                        sent_after=sent_after, send_to=send_to,
                        need=arr(pl.need_from_flat, pl.total_need_from),
                        gidx=arr(pl.need_from_gidx_flat, pl.total_need_from),
                        indeg=pl.indegree, outdeg=pl.outdegree, graph=pl.comm_graph)

    run_ranks(P, rank)
    final = np.arange(n, dtype=np.uint32)
    for r in range(P):
        lo, hi = bounds[r], bounds[r + 1]
        idx = np.arange(lo, hi)
        final[idx[::3]] = np.minimum(final[idx[::3]], 7)
    for r in range(P):
        s, g = state[r], ghosts[r]
        # need-from lists: the ghosts in order, grouped by owner
        assert sorted(s["need"].tolist()) == sorted(g.tolist())
        assert (g[s["gidx"]] == s["need"]).all()
        # what r sends to q is exactly what q needs from r, in q's order
        off = 0
        for q in range(P):
            if q == r:
                continue
            want = [v for v in state[q]["need"] if bounds[r] <= v < bounds[r + 1]]
            got = s["send_to"][off:off + len(want)].tolist()
            assert got == want, (r, q)
            off += len(want)
        assert (s["first"] == g).all()                 # first exchange: ids
        assert (s["second"] == final[g]).all()         # lowered labels arrived
        assert (s["third"] == s["second"]).all()
        assert (s["legacy"] == final[g]).all()
        assert (s["sent_after"] == final[s["send_to"]]).all()
        assert s["indeg"] > 0 and s["outdeg"] > 0 and s["graph"]
    for pl in plans:
        L.exchangeplan_free(C.byref(pl))
        assert pl.total_send_to == 0 and not pl.comm_graph
    L.cc_group_free(grp)


def test_rank_without_neighbours_skips(L):
    """Two ranks, no cut edge: no sources, no destinations, comm_graph NULL;
    the delta exchange returns at once without meeting the other rank."""
    grp = L.cc_group_create(2)
    owner = OWNER_FN(lambda v, ng, size: 0 if v < 10 else 1)
    pl = [ExchangePlan(), ExchangePlan()]

    def rank(r):
        view = L.cc_group_view(grp, r)
        empty = np.zeros(1, np.uint32)
        assert L.exchangeplan_build(C.byref(pl[r]), empty.ctypes.data, 0, 20, view, owner) == 0

    run_ranks(2, rank)
    for r in range(2):
        assert pl[r].indegree == 0 and pl[r].outdegree == 0 and not pl[r].comm_graph
        z = np.zeros(4, np.uint32)
        sb, sc = C.POINTER(C.c_uint64)(), C.c_int(0)
        rb, rc = C.POINTER(C.c_uint64)(), C.c_int(0)
        L.exchangeplan_exchange_delta(C.byref(pl[r]), z.ctypes.data, z.ctypes.data, 0, 10,
                                      z.ctypes.data, z.ctypes.data, None, C.byref(sb),
                                      C.byref(sc), C.byref(rb), C.byref(rc))
        L.exchangeplan_free(C.byref(pl[r]))
    L.cc_group_free(grp)
