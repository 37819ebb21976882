"""libccb200.so loads without a GPU and exports every function the public
headers in include/ declare."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT

INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = {}
    for fn in sorted(os.listdir(INCLUDE)):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, fn)).read()
        text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
        text = re.sub(r"//[^\n]*", " ", text)
        text = re.sub(r"^\s*#.*$", " ", text, flags=re.M)
        # drop typedef'd structs / function-pointer typedefs
        text = re.sub(r"typedef[^;]*?\{.*?\}[^;]*;", " ", text, flags=re.S)
        text = re.sub(r"typedef[^;]*;", " ", text)
        text = re.sub(r'extern\s+"C"\s*\{|\}', " ", text)
        for m in re.finditer(r"([A-Za-z_]\w*)\s*\(([^;{}()]|\([^()]*\))*\)\s*;", text):
            names.setdefault(m.group(1), fn)
    return names


def test_headers_declare_reference_entry_points():
    names = declared_functions()
    for must in ("compute_connected_components_pthreads", "count_unique_labels",
                 "load_csr_from_file", "load_csr_from_mat", "free_csr", "ccgpu_local_cc"):
        assert must in names, must


def test_library_loads_and_exports_every_declared_symbol():
    from cc_mpi_b200 import _lib
    L = _lib.lib()  # loads without a GPU: no CUDA call happens at load time
    missing = []
    for name, header in declared_functions().items():
        try:
            getattr(L, name)
        except AttributeError:
            missing.append(f"{header}:{name}")
    assert not missing, missing


def test_nm_dynamic_symbols():
    from cc_mpi_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    for name in declared_functions():
        assert name in exported, name


def test_no_device_means_status_not_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    from cc_mpi_b200 import _lib
    L = _lib.lib()
    assert L.ccgpu_device_check() == 6  # CCGPU_ERR_NODEVICE
    assert b"device" in L.ccgpu_last_error()
    L.ccgpu_clear_error()
    assert L.ccgpu_last_error() == b""
    ctx = C.c_void_p()
    assert L.ccgpu_ctx_create(C.byref(ctx)) == 6


def test_prof_kernel_names():
    from cc_mpi_b200 import _lib
    L = _lib.lib()
    k = L.ccgpu_prof_kernels()
    names = [L.ccgpu_prof_name(i).decode() for i in range(k)]
    assert "sample" in names and "link_rows" in names and len(set(names)) == k
