"""ccgpu_local_cc_noalloc: the local CC solve for callers that cannot allocate
device memory (under an allocator that already reserved all of HBM, plug-ins
that must not own device memory, or where cudaMalloc's device-wide
synchronisation is not acceptable).  Its scratch is a fixed device array
inside the library, so the call allocates nothing; its labels must be the
same as the allocating entry point's, call after call.

This file sorts last so that a failure here comes after every other test
has run; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import oracle
from cc_mpi_b200 import _lib, cc, graphs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    L = _lib.lib()
    L.ccgpu_local_cc_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                         C.c_void_p, C.POINTER(_lib.CCOpts), C.c_void_p]
    L.ccgpu_local_cc_noalloc.restype = C.c_int
    L.ccgpu_local_cc_noalloc_capacity.restype = C.c_size_t
    L.ccgpu_local_cc_noalloc_required.argtypes = [C.c_uint32, C.c_uint64,
                                                  C.POINTER(_lib.CCOpts)]
    L.ccgpu_local_cc_noalloc_required.restype = C.c_size_t
    return L


@pytest.fixture(scope="module")
def torch():
    import torch as t
    t.cuda.set_device(0)
    return t


CASES = [("rmat14", lambda: graphs.rmat_csr(14, 16, seed=21)),
         ("grid", lambda: graphs.grid_csr(200, 150, 0.2, seed=22)),
         ("path", lambda: graphs.small_cases()["long_path"]),
         ("hubs", lambda: graphs.small_cases()["hubs"])]

OPTS = [None, dict(chunk_size=1), dict(heavy_degree=64, sample_rounds=0, skip_giant=0)]


def noalloc(L, d_rp, d_col, n, m, labels, opts, stream):
    return L.ccgpu_local_cc_noalloc(d_rp.data_ptr(), d_col.data_ptr(), n, m, labels.data_ptr(),
                                    C.byref(opts) if opts is not None else None, stream)


@pytest.mark.parametrize("name,make", CASES)
def test_noalloc_matches_allocating_call_twice(L, torch, name, make):
    rp, col = make()
    n, m = len(rp) - 1, int(rp[-1])
    d_rp = torch.from_numpy(rp.astype(np.int64)).cuda()
    d_col = torch.from_numpy(col.astype(np.int32)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for o in OPTS:
        opts = _lib.opts(**o) if o else None
        want = torch.empty(n, dtype=torch.int32, device="cuda")
        cc.local_cc_device(d_rp, d_col, n, m, want, opts)
        for _ in range(2):  # two calls in a row share the static scratch
            got = torch.full((n,), -1, dtype=torch.int32, device="cuda")
            assert noalloc(L, d_rp, d_col, n, m, got, opts, stream) == 0, L.ccgpu_last_error()
            torch.cuda.synchronize()
            assert torch.equal(got, want), (name, o)  # labels are integers: bit-exact
        assert (want.cpu().numpy().view(np.uint32) == oracle.uf_labels(rp, col)).all()


def test_noalloc_rejects_graphs_beyond_its_scratch(L):
    cap = L.ccgpu_local_cc_noalloc_capacity()
    assert cap == 1 << 20
    small = _lib.opts(heavy_degree=32)
    n, m = 1 << 30, 1 << 36
    assert L.ccgpu_local_cc_noalloc_required(n, m, C.byref(small)) > cap
    # sizes are checked before anything touches the (dummy, never read) pointers
    rc = L.ccgpu_local_cc_noalloc(C.c_void_p(16), C.c_void_p(16), n, m, C.c_void_p(16),
                                  C.byref(small), None)
    assert rc == 5  # CCGPU_ERR_LIMIT
    assert b"scratch" in L.ccgpu_last_error()
    assert L.ccgpu_local_cc_noalloc_required(1 << 24, 1 << 29, None) <= cap
    bad = _lib.opts(sample_rounds=9)  # above the limit of 8: invalid, never fits
    assert L.ccgpu_local_cc_noalloc_required(1000, 1000, C.byref(bad)) == C.c_size_t(-1).value


def test_noalloc_leaves_free_device_memory_unchanged(L, torch):
    """After the first call on the device (its set-up), a call takes no
    device memory: the free bytes the driver reports do not move."""
    rp, col = graphs.rmat_csr(15, 16, seed=23)
    n, m = len(rp) - 1, int(rp[-1])
    d_rp = torch.from_numpy(rp.astype(np.int64)).cuda()
    d_col = torch.from_numpy(col.astype(np.int32)).cuda()
    got = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert noalloc(L, d_rp, d_col, n, m, got, None, stream) == 0  # set-up call
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert noalloc(L, d_rp, d_col, n, m, got, None, stream) == 0, L.ccgpu_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert (got.cpu().numpy().view(np.uint32) == oracle.uf_labels(rp, col)).all()
