"""cc_mpi_b200 - a B200-native connected-components engine with the entry
points of the CC_mpi reference.

The product is ``libccb200.so`` (sm_100a kernels behind a C ABI, plus the
reference-facing C API of include/cc.h, include/cc_mpi.h, include/graph.h,
include/graph_dist.h, include/boundary_sort.h and include/exchange_plan.h) and
the ``mpi_cc_benchmark`` CLI.  This Python package is a thin host-side mirror
used by the tests and the benchmark: it passes pointers to the C ABI and
never computes labels itself.
"""
from ._lib import CCGPUError, lib, check, opts, LIB_PATH, CLI_PATH  # noqa: F401
from . import cc  # noqa: F401

__all__ = ["CCGPUError", "lib", "check", "opts", "LIB_PATH", "CLI_PATH", "cc"]
