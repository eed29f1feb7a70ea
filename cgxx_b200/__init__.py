"""cgxx_b200: a B200-native (sm_100a) conjugate-gradient solver behind the
hahnjo/CGxx interface.

The product is native: libcgb200.so (CUDA kernels + the C ABI of
include/cgx.h) and the cg_b200 executable (the reference's CG class surface
in C++, cgxx_b200/host/). This Python package is a thin ctypes binding used by
the tests, the benchmark and the training driver of the learned
preconditioner; it loads the in-tree library and fails loudly if it is
missing.
"""
from ._lib import (  # noqa: F401
    CgxError, Gnn, Handle, default_options, device_count, load, mtx_read,
    mtx_write_symmetric_crs, pinned_empty,
    FORMAT_COO, FORMAT_CRS, FORMAT_ELL,
    PRECOND_NONE, PRECOND_JACOBI, PRECOND_LEARNED,
    PRECISION_FP64, PRECISION_MIXED,
    LOOP_GRAPH, LOOP_CHUNKED, LOOP_KERNELS, LOOP_PERSISTENT, LOOP_PERSISTENT_SPLIT,
    VECTOR_K, VECTOR_X, VECTOR_P, VECTOR_Q, VECTOR_R, VECTOR_Z,
)
