"""Regenerates the golden fixtures in this directory from the reference's own
code, compiled unmodified into oracle/_ref/libccref.so (``make -C oracle
ref``; needs the reference source tree, so this script runs where the tree
is, not on the GPU machines).

Fixtures:
  labels.npz          small graphs + labels from the reference's
                      compute_connected_components_pthreads (4 threads,
                      dynamic chunk 64 and static chunk 1)
  boundary_sort.npz   boundary pair arrays + the reference's
                      boundary_edges_sort/boundary_edges_dedup output
  opt_parser.json     range-list specs + opt_parse_range_list results
  results_writer.json append sequences + the CSV text append_times_column
                      leaves behind

Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from cc_mpi_b200 import graphs  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def make_labels():
    cases = graphs.small_cases()
    cases["grid100"] = graphs.grid_csr(100, 100, 0.35, seed=11)
    cases["er5k"] = graphs.er_csr(5000, 2.0, seed=12)
    arrays = {}
    names = []
    for name, (rp, col) in cases.items():
        dyn = oracle.ref_pthreads_labels(rp, col, threads=4, chunk=64)
        sta = oracle.ref_pthreads_labels(rp, col, threads=4, chunk=1)
        assert (dyn == sta).all(), name
        arrays[f"{name}__row_ptr"] = rp
        arrays[f"{name}__col"] = col
        arrays[f"{name}__labels"] = dyn
        names.append(name)
    arrays["names"] = np.array(names)
    np.savez_compressed(os.path.join(OUT, "labels.npz"), **arrays)


def make_boundary_sort():
    rng = np.random.default_rng(2024)
    cases = {}

    def pairs(rep, remote):
        a = np.empty(len(rep), dtype=oracle.PAIR_DTYPE)
        a["rep"] = rep
        a["remote"] = remote
        return a

    cases["empty"] = pairs([], [])
    cases["one"] = pairs([5], [9])
    cases["n64"] = pairs(rng.integers(0, 20, 64), rng.integers(0, 10, 64))
    cases["n65"] = pairs(rng.integers(0, 20, 65), rng.integers(0, 10, 65))
    cases["dups"] = pairs(np.repeat(rng.integers(0, 50, 300), 7), np.repeat(rng.integers(0, 50, 300), 7))
    cases["wide"] = pairs(rng.integers(0, 2**32, 5000, dtype=np.uint64),
                          rng.integers(0, 2**32, 5000, dtype=np.uint64))
    cases["same_remote"] = pairs(rng.integers(0, 1 << 20, 3000), np.full(3000, 123456))
    cases["same_rep"] = pairs(np.full(3000, 77), rng.integers(0, 1 << 24, 3000))
    cases["big"] = pairs(rng.integers(0, 1 << 18, 40000), rng.integers(0, 1 << 22, 40000))
    arrays = {}
    for name, a in cases.items():
        arrays[f"{name}__in"] = a.view(np.uint64) if len(a) else np.zeros(0, np.uint64)
        arrays[f"{name}__out"] = oracle.ref_boundary_sort_dedup(a).view(np.uint64) \
            if len(a) else np.zeros(0, np.uint64)
    arrays["names"] = np.array(list(cases))
    np.savez_compressed(os.path.join(OUT, "boundary_sort.npz"), **arrays)


class OptIntList(C.Structure):
    _fields_ = [("values", C.POINTER(C.c_int)), ("size", C.c_size_t), ("capacity", C.c_size_t)]


def make_opt_parser():
    L = oracle.rlib()
    L.opt_parse_range_list.argtypes = [C.c_char_p, C.POINTER(OptIntList), C.c_char_p]
    L.opt_int_list_free.argtypes = [C.POINTER(OptIntList)]
    L.opt_parse_positive_int.argtypes = [C.c_char_p, C.POINTER(C.c_int)]
    specs = ["2048", "1,2,4", "4,2,1,2", "1:8", "1:16:4", "2048,8192,32768", " 3 , 1 ",
             "1:3,2:6:2", "0", "-1", "abc", "5:1", "1:4:0", "", ",", "1,,2", "2147483647",
             "2147483646:2147483647", "1:10:3", "07", "3x", "1:2:3:4"]
    res = []
    for s in specs:
        lst = OptIntList()
        rc = L.opt_parse_range_list(s.encode(), C.byref(lst), b"values")
        vals = [lst.values[i] for i in range(lst.size)] if rc == 0 else None
        L.opt_int_list_free(C.byref(lst))
        res.append({"spec": s, "rc": rc, "values": vals})
    ints = []
    for s in ["1", "42", "0", "-3", "x", "", "2147483648", "12a", "+5"]:
        v = C.c_int(0)
        rc = L.opt_parse_positive_int(s.encode(), C.byref(v))
        ints.append({"text": s, "rc": rc, "value": v.value if rc == 0 else None})
    with open(os.path.join(OUT, "opt_parser.json"), "w") as f:
        json.dump({"range_lists": res, "positive_ints": ints}, f, indent=1)


def make_results_writer():
    L = oracle.rlib()
    L.append_times_column.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_double), C.c_size_t]
    L.results_writer_build_results_path.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p,
                                                    C.c_char_p, C.c_char_p]
    seqs = [
        [("chunk_2048_exchange_1", [0.5, 0.25])],
        [("a", [1.0]), ("b", [2.0, 3.0, 4.0])],
        [("a", [1.0, 2.0]), ("a", [3.0])],
        [("x", [0.1234567, 12.5]), ("y", [1e-7]), ("x", [2.0, 3.0, 4.0]), ("z", [])],
        [("chunk_8192_exchange_2", [52.414, 52.372, 52.407]),
         ("chunk_8192_exchange_4", [50.844])],
    ]
    out = []
    with tempfile.TemporaryDirectory() as d:
        for i, seq in enumerate(seqs):
            path = os.path.join(d, f"r{i}.csv")
            for col, vals in seq:
                arr = (C.c_double * max(len(vals), 1))(*vals)
                rc = L.append_times_column(path.encode(), col.encode(), arr, len(vals))
                assert rc == 0
            with open(path) as f:
                out.append({"ops": seq, "csv": f.read()})
    paths = []
    for od, mp in [("results", "data/com-Friendster.mat"), ("out/", "g.mat"), ("o", "x/y/z"),
                   ("o", "a.b.c.mat"), ("o", ""), ("o", ".mat"), ("o", "dir/")]:
        buf = C.create_string_buffer(4096)
        rc = L.results_writer_build_results_path(buf, 4096, od.encode(), b"results_mpi",
                                                 mp.encode())
        paths.append({"dir": od, "matrix": mp, "rc": rc, "path": buf.value.decode()})
    with open(os.path.join(OUT, "results_writer.json"), "w") as f:
        json.dump({"sequences": out, "paths": paths}, f, indent=1)


if __name__ == "__main__":
    oracle.build(ref=True)
    make_labels()
    make_boundary_sort()
    make_opt_parser()
    make_results_writer()
    print("golden fixtures written to", OUT)
