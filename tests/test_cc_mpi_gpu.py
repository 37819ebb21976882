"""The reference-facing partitioned API (cc_mpi.h, graph_dist.h,
boundary_sort.h) and the mpi_cc_benchmark CLI, end to end on the GPU."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle
from cc_mpi_b200 import _lib, graphs
from cc_mpi_b200.dist import DistStats

pytestmark = pytest.mark.gpu


class CSR(C.Structure):
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint64), ("row_ptr", C.POINTER(C.c_uint64)),
                ("col_idx", C.POINTER(C.c_uint32))]


@pytest.fixture(scope="module")
def L():
    L = _lib.lib()
    vp = C.c_void_p
    L.cc_group_create.restype = vp
    L.cc_group_create.argtypes = [C.c_int]
    L.cc_group_free.argtypes = [vp]
    L.cc_group_set_verbose.argtypes = [vp, C.c_int]
    L.cc_group_last_stats.argtypes = [vp, C.POINTER(DistStats)]
    L.dist_csr_from_csr.argtypes = [C.POINTER(CSR), C.c_int, C.POINTER(_lib.DistCSRGraph), vp]
    L.free_dist_csr_view.argtypes = [C.POINTER(_lib.DistCSRGraph)]
    L.load_dist_csr_from_file.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int,
                                          C.POINTER(_lib.DistCSRGraph), vp]
    L.free_dist_csr.argtypes = [C.POINTER(_lib.DistCSRGraph)]
    L.cc_mpi_solve.argtypes = [C.POINTER(_lib.DistCSRGraph), vp, C.c_int, C.c_int, vp,
                               C.POINTER(DistStats)]
    L.compute_connected_components_mpi_advanced.argtypes = [C.POINTER(_lib.DistCSRGraph), vp,
                                                            C.c_int, C.c_int, vp]
    L.count_connected_components.argtypes = [vp, C.c_uint32]
    L.count_connected_components.restype = C.c_uint32
    L.boundary_edges_sort.argtypes = [vp, C.c_uint64]
    L.boundary_edges_dedup.argtypes = [vp, C.c_uint64]
    L.boundary_edges_dedup.restype = C.c_uint64
    L.save_csr_to_mat.argtypes = [C.c_char_p, C.POINTER(CSR)]
    L.ccb200_set_exit_on_error.argtypes = [C.c_int]
    L.ccb200_set_exit_on_error(0)
    return L


def csr_of(rp, col):
    rp = np.ascontiguousarray(rp, dtype=np.uint64)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    return CSR(len(rp) - 1, int(rp[-1]), rp.ctypes.data_as(C.POINTER(C.c_uint64)),
               col.ctypes.data_as(C.POINTER(C.c_uint32))), (rp, col)


@pytest.mark.parametrize("parts", [1, 2, 4, 5])
@pytest.mark.parametrize("use_edge", [0, 1])
def test_mpi_advanced_labels_and_stats(L, parts, use_edge):
    rp, col = graphs.rmat_csr(13, 8, seed=parts + 10 * use_edge)
    g, keep = csr_of(rp, col)
    grp = L.cc_group_create(parts)
    L.cc_group_set_verbose(grp, 0)
    Gd = _lib.DistCSRGraph()
    assert L.dist_csr_from_csr(C.byref(g), use_edge, C.byref(Gd), grp) == 0
    if use_edge and parts > 1:
        assert Gd.part_kind == 1 and Gd.part_size == parts
        b = np.ctypeslib.as_array(Gd.part_bounds, shape=(parts + 1,))
        assert (b == oracle.weighted_bounds(rp, parts)).all()
    else:
        assert Gd.part_kind == 0 and not Gd.part_bounds
    for interval in (1, 3):
        labels = np.zeros(len(rp) - 1, dtype=np.uint32)
        L.compute_connected_components_mpi_advanced(C.byref(Gd), labels.ctypes.data, 2048,
                                                    interval, grp)
        st = DistStats()
        assert L.cc_group_last_stats(grp, C.byref(st)) == 0
        want, _, ost = oracle.dist_cc(rp, col, parts, use_edge, interval)
        assert (labels == want).all()
        assert st.rounds == ost.rounds and st.roots == ost.roots
        assert L.count_connected_components(labels.ctypes.data, len(labels)) == ost.roots
    L.free_dist_csr_view(C.byref(Gd))
    L.cc_group_free(grp)


def test_mpi_advanced_null_labels_and_errors(L):
    rp, col = graphs.rmat_csr(10, 8, seed=1)
    g, keep = csr_of(rp, col)
    grp = L.cc_group_create(3)
    L.cc_group_set_verbose(grp, 0)
    Gd = _lib.DistCSRGraph()
    assert L.dist_csr_from_csr(C.byref(g), 1, C.byref(Gd), grp) == 0
    assert L.cc_mpi_solve(C.byref(Gd), None, 8192, 1, grp, None) == 0  # labels NULL is fine
    other = L.cc_group_create(2)
    assert L.cc_mpi_solve(C.byref(Gd), None, 8192, 1, other, None) == 1  # wrong group size
    part = _lib.DistCSRGraph()
    C.memmove(C.byref(part), C.byref(Gd), C.sizeof(part))
    part.n_local = 10
    assert L.cc_mpi_solve(C.byref(part), None, 8192, 1, grp, None) == 5  # one partition only
    L.free_dist_csr_view(C.byref(Gd))
    L.cc_group_free(grp)
    L.cc_group_free(other)


def test_load_dist_from_mat(L, tmp_path):
    rp, col = graphs.grid_csr(120, 90, 0.3, seed=2)
    g, keep = csr_of(rp, col)
    path = str(tmp_path / "grid.mat")
    assert L.save_csr_to_mat(path.encode(), C.byref(g)) == 0
    grp = L.cc_group_create(4)
    L.cc_group_set_verbose(grp, 0)
    Gd = _lib.DistCSRGraph()
    assert L.load_dist_csr_from_file(path.encode(), 1, 1, 1, C.byref(Gd), grp) == 0
    assert Gd.n_global == len(rp) - 1 and Gd.m_global == int(rp[-1])
    labels = np.zeros(Gd.n_global, dtype=np.uint32)
    L.compute_connected_components_mpi_advanced(C.byref(Gd), labels.ctypes.data, 1, 2, grp)
    assert (labels == oracle.uf_labels(rp, col)).all()
    L.free_dist_csr(C.byref(Gd))
    assert Gd.row_ptr is None or not Gd.row_ptr
    L.cc_group_free(grp)


def test_device_csc_to_csr_matches_host_loader(L, tmp_path):
    """The partitioned loader transposes a .mat's CSC on the device
    (ccgpu_graph_from_csc); the CSR it exposes equals the host loader's
    (load_csr_from_mat, the reference's count / scan / scatter,
    src/graph.c:91-117) entry for entry: rows in order, each row's
    neighbours ascending.  Cases: a symmetric graph written by scipy, a
    non-square matrix whose extra columns give ids >= n, empty rows and
    columns."""
    import scipy.io as sio
    import scipy.sparse as sp
    rp, col = graphs.rmat_csr(12, 8, seed=12)
    n = len(rp) - 1
    sym = sp.csc_matrix((np.ones(len(col), bool), col.astype(np.int64), rp.astype(np.int64)),
                        shape=(n, n))
    rect = sp.lil_matrix(sp.random(300, 420, density=0.02, random_state=14) != 0)
    rect[:, 7] = 0
    rect[11, :] = 0
    rect = sp.csc_matrix(rect)
    rect.eliminate_zeros()
    L.load_csr_from_mat.argtypes = [C.c_char_p, C.POINTER(CSR)]
    L.free_csr.argtypes = [C.POINTER(CSR)]
    for name, A, packed in (("sym", sym, True), ("rect", rect, False)):
        path = str(tmp_path / f"{name}.mat")
        sio.savemat(path, {"Problem": {"A": A}}, do_compression=packed)
        host = CSR()
        assert L.load_csr_from_mat(path.encode(), C.byref(host)) == 0
        grp = L.cc_group_create(2)
        L.cc_group_set_verbose(grp, 0)
        Gd = _lib.DistCSRGraph()
        assert L.load_dist_csr_from_file(path.encode(), 1, 1, 1, C.byref(Gd), grp) == 0
        assert Gd.n_global == host.n and Gd.m_global == host.m
        hr = np.ctypeslib.as_array(host.row_ptr, (host.n + 1,))
        hc = np.ctypeslib.as_array(host.col_idx, (max(host.m, 1),))[:host.m]
        dr = np.ctypeslib.as_array(Gd.row_ptr, (Gd.n_global + 1,))
        dc = np.ctypeslib.as_array(Gd.col_idx, (max(Gd.m_global, 1),))[:Gd.m_global]
        assert (hr == dr).all() and (hc == dc).all(), name
        want = sp.csr_matrix(A)
        want.sort_indices()
        assert (dr == want.indptr).all() and (dc == want.indices).all(), name
        L.free_dist_csr(C.byref(Gd))
        L.free_csr(C.byref(host))
        L.cc_group_free(grp)


def test_boundary_edges_host_api_golden(L):
    from conftest import GOLDEN
    d = np.load(os.path.join(GOLDEN, "boundary_sort.npz"))
    for name in d["names"]:
        name = str(name)
        a = d[f"{name}__in"].copy()
        exp = d[f"{name}__out"]
        if len(a) == 0:
            continue
        L.boundary_edges_sort(a.ctypes.data, len(a))
        k = L.boundary_edges_dedup(a.ctypes.data, len(a))
        assert k == len(exp) and (a[:k] == exp).all(), name


def test_cli_end_to_end(L, tmp_path):
    rp, col = graphs.rmat_csr(12, 16, seed=8)
    g, keep = csr_of(rp, col)
    mat = str(tmp_path / "rmat12.mat")
    assert L.save_csr_to_mat(mat.encode(), C.byref(g)) == 0
    out = tmp_path / "out"
    lab = tmp_path / "labels.bin"
    cli = _lib.CLI_PATH
    r = subprocess.run([cli, "-p", "4", "-c", "2048,8192", "-e", "1:2", "-r", "2", "-t", "8",
                        "-o", str(out), "-L", str(lab), mat], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    uf = oracle.uf_labels(rp, col)
    comps = oracle.count_components(uf)
    assert f"Number of connected components: {comps}" in r.stdout
    got = np.fromfile(lab, dtype=np.uint32)
    assert (got == uf).all()
    csv = (out / "results_mpi_rmat12.csv").read_text().splitlines()
    assert csv[0] == ("chunk_2048_exchange_1,chunk_2048_exchange_2,"
                      "chunk_8192_exchange_1,chunk_8192_exchange_2")
    assert len(csv) == 3
    for row in csv[1:]:
        vals = [float(x) for x in row.split(",")]
        assert all(v > 0 for v in vals) and all(len(x.split(".")[1]) == 6
                                                for x in row.split(","))
    # a second invocation appends rows below the existing ones
    r = subprocess.run([cli, "-p", "4", "-c", "2048", "-e", "1", "-q", "-o", str(out), mat],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    csv = (out / "results_mpi_rmat12.csv").read_text().splitlines()
    assert len(csv) == 4 and csv[3].startswith(csv[3].split(",")[0]) and csv[3].count(",") == 3


def test_cli_bad_input(tmp_path):
    cli = _lib.CLI_PATH
    r = subprocess.run([cli, "-r", "0", "x.mat"], capture_output=True, text=True)
    assert r.returncode != 0 and "Invalid runs" in r.stderr
    r = subprocess.run([cli, "-c", "5:1", str(tmp_path / "x.mat")], capture_output=True,
                       text=True)
    assert r.returncode != 0
    r = subprocess.run([cli, "-o", str(tmp_path), str(tmp_path / "missing.mat")],
                       capture_output=True, text=True)
    assert r.returncode != 0 and "Error loading graph" in r.stderr
