"""Host C layer of libccb200 without a GPU: the CLI helpers against fixtures
produced by the reference's own opt_parser.c / results_writer.c, and the
graph readers/writers (.mat level 5 incl. compressed, .mtx, .csrbin)."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from cc_mpi_b200 import _lib, graphs
from conftest import GOLDEN


class OptIntList(C.Structure):
    _fields_ = [("values", C.POINTER(C.c_int)), ("size", C.c_size_t),
                ("capacity", C.c_size_t)]


class CSR(C.Structure):
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint64), ("row_ptr", C.POINTER(C.c_uint64)),
                ("col_idx", C.POINTER(C.c_uint32))]


@pytest.fixture(scope="module")
def L():
    L = _lib.lib()
    L.opt_parse_range_list.argtypes = [C.c_char_p, C.POINTER(OptIntList), C.c_char_p]
    L.opt_int_list_free.argtypes = [C.POINTER(OptIntList)]
    L.opt_parse_positive_int.argtypes = [C.c_char_p, C.POINTER(C.c_int)]
    L.append_times_column.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_double), C.c_size_t]
    L.results_writer_build_results_path.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p,
                                                    C.c_char_p, C.c_char_p]
    L.results_writer_ensure_directory.argtypes = [C.c_char_p]
    for f in ("load_csr_from_mat", "load_csr_from_csrbin"):
        getattr(L, f).argtypes = [C.c_char_p, C.POINTER(CSR)]
    L.load_csr_from_file.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(CSR)]
    L.load_csr_from_mtx.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(CSR)]
    L.save_csr_to_mat.argtypes = [C.c_char_p, C.POINTER(CSR)]
    L.save_csr_to_csrbin.argtypes = [C.c_char_p, C.POINTER(CSR)]
    L.free_csr.argtypes = [C.POINTER(CSR)]
    return L


def test_opt_parser_matches_reference(L):
    with open(os.path.join(GOLDEN, "opt_parser.json")) as f:
        g = json.load(f)
    for case in g["range_lists"]:
        lst = OptIntList()
        rc = L.opt_parse_range_list(case["spec"].encode(), C.byref(lst), b"values")
        vals = [lst.values[i] for i in range(lst.size)] if rc == 0 else None
        L.opt_int_list_free(C.byref(lst))
        assert rc == case["rc"], case
        assert vals == case["values"], case
    for case in g["positive_ints"]:
        v = C.c_int(0)
        rc = L.opt_parse_positive_int(case["text"].encode(), C.byref(v))
        assert rc == case["rc"], case
        if rc == 0:
            assert v.value == case["value"]


def test_results_writer_matches_reference(L, tmp_path):
    with open(os.path.join(GOLDEN, "results_writer.json")) as f:
        g = json.load(f)
    for i, seq in enumerate(g["sequences"]):
        path = str(tmp_path / f"r{i}.csv")
        for col, vals in seq["ops"]:
            arr = (C.c_double * max(len(vals), 1))(*vals)
            assert L.append_times_column(path.encode(), col.encode(), arr, len(vals)) == 0
        assert open(path).read() == seq["csv"], seq["ops"]
    for case in g["paths"]:
        buf = C.create_string_buffer(4096)
        rc = L.results_writer_build_results_path(buf, 4096, case["dir"].encode(),
                                                 b"results_mpi", case["matrix"].encode())
        assert rc == case["rc"]
        assert buf.value.decode() == case["path"], case


def test_results_writer_mkdir(L, tmp_path):
    d = tmp_path / "a" / "b" / "c"
    assert L.results_writer_ensure_directory(str(d).encode() + b"/") == 0
    assert d.is_dir()


def csr_of(rp, col):
    rp = np.ascontiguousarray(rp, dtype=np.uint64)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    g = CSR(len(rp) - 1, int(rp[-1]), rp.ctypes.data_as(C.POINTER(C.c_uint64)),
            col.ctypes.data_as(C.POINTER(C.c_uint32)))
    return g, (rp, col)


def read_back(L, fn, path, *extra):
    out = CSR()
    rc = fn(path.encode(), *extra, C.byref(out))
    if rc != 0:
        return rc, None, None
    rp = np.ctypeslib.as_array(out.row_ptr, shape=(out.n + 1,)).copy()
    col = np.ctypeslib.as_array(out.col_idx, shape=(max(out.m, 1),))[:out.m].copy()
    L.free_csr(C.byref(out))
    return rc, rp, col


def test_mat_roundtrip_own_writer(L, tmp_path):
    rp, col = graphs.rmat_csr(10, 8, seed=2)
    g, keep = csr_of(rp, col)
    path = str(tmp_path / "g.mat")
    assert L.save_csr_to_mat(path.encode(), C.byref(g)) == 0
    rc, rp2, col2 = read_back(L, L.load_csr_from_mat, path)
    assert rc == 0 and (rp2 == rp).all() and (col2 == col).all()


@pytest.mark.parametrize("compress", [False, True])
@pytest.mark.parametrize("as_struct", [False, True])
def test_mat_written_by_scipy(L, tmp_path, compress, as_struct):
    sio = pytest.importorskip("scipy.io")
    sp = pytest.importorskip("scipy.sparse")
    rp, col = graphs.rmat_csr(9, 8, seed=5)
    n = len(rp) - 1
    A = sp.csr_matrix((np.ones(len(col), dtype=bool), col.astype(np.int64),
                       rp.astype(np.int64)), shape=(n, n))
    path = str(tmp_path / "s.mat")
    if as_struct:
        sio.savemat(path, {"Problem": {"title": "x", "A": A.tocsc()}}, do_compression=compress)
    else:
        sio.savemat(path, {"junk": np.arange(3.0), "G": A.tocsc()}, do_compression=compress)
    rc, rp2, col2 = read_back(L, L.load_csr_from_mat, path)
    assert rc == 0
    assert (rp2 == rp).all() and (col2 == col).all()


def test_mat_errors(L, tmp_path):
    sio = pytest.importorskip("scipy.io")
    assert read_back(L, L.load_csr_from_mat, str(tmp_path / "missing.mat"))[0] == 1
    path = str(tmp_path / "dense.mat")
    sio.savemat(path, {"x": np.eye(3)})
    assert read_back(L, L.load_csr_from_mat, path)[0] == 2


def test_file_dispatch_codes(L, tmp_path):
    out = CSR()
    for name, want in (("a.mtx", -1), ("a.txt", -1), ("a.xyz", 99)):
        assert L.load_csr_from_file(str(tmp_path / name).encode(), 1, 1, C.byref(out)) == want


def test_csrbin_roundtrip_and_bad_magic(L, tmp_path):
    rp, col = graphs.grid_csr(30, 40, 0.2, seed=1)
    g, keep = csr_of(rp, col)
    path = str(tmp_path / "g.csrbin")
    assert L.save_csr_to_csrbin(path.encode(), C.byref(g)) == 0
    rc, rp2, col2 = read_back(L, L.load_csr_from_file, path, 1, 1)
    assert rc == 0 and (rp2 == rp).all() and (col2 == col).all()
    bad = tmp_path / "bad.csrbin"
    bad.write_bytes(b"XXXX" + b"\0" * 64)
    assert read_back(L, L.load_csr_from_csrbin, str(bad))[0] == 5


def test_mtx_reader(L, tmp_path):
    sio = pytest.importorskip("scipy.io")
    sp = pytest.importorskip("scipy.sparse")
    rng = np.random.default_rng(0)
    r = rng.integers(0, 50, 300)
    c = rng.integers(0, 50, 300)
    A = sp.coo_matrix((np.ones(300), (r, c)), shape=(50, 50))
    path = str(tmp_path / "a.mtx")
    sio.mmwrite(path, A)
    rc, rp, col = read_back(L, L.load_csr_from_mtx, path, 1, 1)
    assert rc == 0
    want_rp, want_col = graphs.csr_from_edges(50, r, c)
    assert (rp == want_rp).all() and (col == want_col).all()
