"""ctypes binding of the CPU oracle (oracle/build/liboracle.so) and helpers to
run the reference's own binaries from oracle/_ref/.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker. The product never imports it.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


class _Matrix(C.Structure):
    _fields_ = [
        ("format", C.c_int), ("N", C.c_int), ("nz", C.c_int),
        ("I", C.c_void_p), ("J", C.c_void_p), ("V", C.c_void_p),
        ("ptr", C.c_void_p), ("index", C.c_void_p), ("value", C.c_void_p),
        ("length", C.c_void_p), ("data", C.c_void_p),
    ]


class _Coo(C.Structure):
    _fields_ = [("N", C.c_int), ("nz", C.c_int), ("I", C.POINTER(C.c_int)),
                ("J", C.POINTER(C.c_int)), ("V", C.POINTER(C.c_double)),
                ("nzPerRow", C.POINTER(C.c_int))]


def build():
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = C.CDLL(LIB_PATH)
        P = C.c_void_p
        lib.orc_cg_solve.argtypes = [C.POINTER(_Matrix), P, P, P, C.c_int, C.c_double,
                                     C.POINTER(C.c_double)]
        lib.orc_cg_solve.restype = C.c_int
        lib.orc_mixed_ir_solve.argtypes = [C.c_int, P, P, P, P, P, P, C.c_int, C.c_double,
                                           C.c_double, C.c_int, C.POINTER(C.c_int),
                                           C.POINTER(C.c_double)]
        lib.orc_mixed_ir_solve.restype = C.c_int
        lib.orc_matvec_crs.argtypes = [C.c_int, P, P, P, P, P]
        lib.orc_matvec_ell.argtypes = [C.c_int, P, P, P, P, P]
        lib.orc_matvec_coo.argtypes = [C.c_int, C.c_int, P, P, P, P, P]
        lib.orc_axpy.argtypes = [C.c_int, C.c_double, P, P]
        lib.orc_xpay.argtypes = [C.c_int, P, C.c_double, P]
        lib.orc_dot.argtypes = [C.c_int, P, P]
        lib.orc_dot.restype = C.c_double
        lib.orc_jacobi_apply.argtypes = [C.c_int, P, P, P]
        lib.orc_read_mtx.argtypes = [C.c_char_p, C.POINTER(_Coo)]
        lib.orc_read_mtx.restype = C.c_int
        lib.orc_coo_free.argtypes = [C.POINTER(_Coo)]
        lib.orc_check_ones.argtypes = [C.c_int, P, C.c_double]
        lib.orc_check_ones.restype = C.c_int
        lib.orc_coo_to_crs.argtypes = [C.POINTER(_Coo), P, P, P]
        lib.orc_coo_to_ell.argtypes = [C.POINTER(_Coo), C.c_int, P, P, P]
        lib.orc_jacobi_init.argtypes = [C.POINTER(_Coo), P]
        lib.orc_rhs_ones.argtypes = [C.POINTER(_Coo), P]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# --- kernels (serial/SerialCG.cpp) -------------------------------------------

def matvec_crs(ptr, index, value, x):
    ptr, index, value, x = _c(ptr, np.int32), _c(index, np.int32), _c(value, np.float64), _c(x, np.float64)
    y = np.empty(len(ptr) - 1)
    load().orc_matvec_crs(len(ptr) - 1, _p(ptr), _p(index), _p(value), _p(x), _p(y))
    return y


def matvec_ell(N, length, index, data, x):
    length, index, data, x = _c(length, np.int32), _c(index, np.int32), _c(data, np.float64), _c(x, np.float64)
    y = np.empty(N)
    load().orc_matvec_ell(N, _p(length), _p(index), _p(data), _p(x), _p(y))
    return y


def matvec_coo(N, I, J, V, x):
    I, J, V, x = _c(I, np.int32), _c(J, np.int32), _c(V, np.float64), _c(x, np.float64)
    y = np.empty(N)
    load().orc_matvec_coo(N, len(I), _p(I), _p(J), _p(V), _p(x), _p(y))
    return y


def axpy(a, x, y):
    x, y = _c(x, np.float64), _c(y, np.float64).copy()
    load().orc_axpy(len(x), a, _p(x), _p(y))
    return y


def xpay(x, a, y):
    x, y = _c(x, np.float64), _c(y, np.float64).copy()
    load().orc_xpay(len(x), _p(x), a, _p(y))
    return y


def dot(a, b):
    a, b = _c(a, np.float64), _c(b, np.float64)
    return load().orc_dot(len(a), _p(a), _p(b))


def jacobi_apply(Cd, x):
    Cd, x = _c(Cd, np.float64), _c(x, np.float64)
    y = np.empty_like(x)
    load().orc_jacobi_apply(len(x), _p(Cd), _p(x), _p(y))
    return y


# --- solvers ------------------------------------------------------------------

def cg_solve_crs(ptr, index, value, k, Cdiag=None, x0=None, max_iter=1000, tol=1e-9):
    """CG::solve (CG.cpp:284-385) on a CRS matrix. Returns (x, iterations,
    residual)."""
    ptr, index, value = _c(ptr, np.int32), _c(index, np.int32), _c(value, np.float64)
    N = len(ptr) - 1
    m = _Matrix(format=1, N=N, nz=int(ptr[-1]), ptr=_p(ptr), index=_p(index), value=_p(value))
    return _solve(m, N, k, Cdiag, x0, max_iter, tol, keep=(ptr, index, value))


def cg_solve_ell(N, nz, length, index, data, k, Cdiag=None, x0=None, max_iter=1000, tol=1e-9):
    length, index, data = _c(length, np.int32), _c(index, np.int32), _c(data, np.float64)
    m = _Matrix(format=2, N=N, nz=nz, length=_p(length), index=_p(index), data=_p(data))
    return _solve(m, N, k, Cdiag, x0, max_iter, tol, keep=(length, index, data))


def cg_solve_coo(N, I, J, V, k, Cdiag=None, x0=None, max_iter=1000, tol=1e-9):
    I, J, V = _c(I, np.int32), _c(J, np.int32), _c(V, np.float64)
    m = _Matrix(format=0, N=N, nz=len(I), I=_p(I), J=_p(J), V=_p(V))
    return _solve(m, N, k, Cdiag, x0, max_iter, tol, keep=(I, J, V))


def _solve(m, N, k, Cdiag, x0, max_iter, tol, keep):
    k = _c(k, np.float64)
    x = np.zeros(N) if x0 is None else _c(x0, np.float64).copy()
    Cd = None if Cdiag is None else _c(Cdiag, np.float64)
    res = C.c_double(0)
    it = load().orc_cg_solve(C.byref(m), _p(Cd), _p(k), _p(x), max_iter, tol, C.byref(res))
    return x, it, res.value


def mixed_ir_solve(ptr, index, value, Cdiag, b, max_iter=10000, tol=1e-9,
                   inner_tol=3e-6, max_outer=30):
    """FP32-inner / FP64-refinement restatement (see cg_oracle.h), with the
    library's default floor of the inner tolerance. Returns (x, total_inner,
    outer, true_residual)."""
    ptr, index, value = _c(ptr, np.int32), _c(index, np.int32), _c(value, np.float64)
    Cd, b = _c(Cdiag, np.float64), _c(b, np.float64)
    N = len(ptr) - 1
    x = np.zeros(N)
    outer = C.c_int(0)
    tr = C.c_double(0)
    it = load().orc_mixed_ir_solve(N, _p(ptr), _p(index), _p(value), _p(Cd), _p(b), _p(x),
                                   max_iter, tol, inner_tol, max_outer, C.byref(outer),
                                   C.byref(tr))
    return x, it, outer.value, tr.value


def read_mtx(path):
    """MatrixCOO::MatrixCOO restated. Returns (status, N, I, J, V)."""
    c = _Coo()
    st = load().orc_read_mtx(os.fsencode(path), C.byref(c))
    if st != 0:
        return st, 0, None, None, None
    n = c.nz
    I = np.ctypeslib.as_array(c.I, shape=(n,)).copy()
    J = np.ctypeslib.as_array(c.J, shape=(n,)).copy()
    V = np.ctypeslib.as_array(c.V, shape=(n,)).copy()
    N = c.N
    load().orc_coo_free(C.byref(c))
    return 0, N, I, J, V


# --- the reference's own binaries (built into oracle/_ref by the Makefile) ----

def ref_binary(name):
    p = os.path.join(REF_DIR, name)
    return p if os.path.exists(p) else None


_SUMMARY = {
    "iterations": re.compile(r"^Iterations:\s+(\d+)", re.M),
    "residual": re.compile(r"^Residual:\s+(\S+)", re.M),
    "solve_time": re.compile(r"^Solve time:\s+(\S+)", re.M),
    "io_time": re.compile(r"^IO time:\s+(\S+)", re.M),
}


def parse_summary(text):
    """Reads the labels printed by CG::printSummary (CG.cpp:417-520); with
    several repetitions, lists of values."""
    out = {}
    for k, rx in _SUMMARY.items():
        vals = rx.findall(text)
        conv = int if k == "iterations" else float
        out[k] = [conv(v) for v in vals]
    out["correct"] = text.count("Solution is correct!")
    out["incorrect"] = re.findall(r"^(\d+) elements are incorrect!", text, re.M)
    return out


def run_ref_harness(mtx, rhs=None, backend="serial", reps=1, env=None, x_out=None,
                    threads=None, timeout=3600):
    """Runs oracle/_ref/ref_harness_<backend>: the reference's CG on `mtx`,
    optionally with right-hand side `rhs` (numpy), returning (summary, x)."""
    exe = ref_binary(f"ref_harness_{backend}")
    if exe is None:
        raise FileNotFoundError(f"oracle/_ref/ref_harness_{backend} is not built")
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        cmd = [exe, mtx, "--reps", str(reps)]
        if rhs is not None:
            rp = os.path.join(td, "k.bin")
            np.ascontiguousarray(rhs, dtype=np.float64).tofile(rp)
            cmd += ["--rhs", rp]
        xp = x_out or os.path.join(td, "x.bin")
        cmd += ["--x-out", xp]
        e = dict(os.environ)
        if env:
            e.update(env)
        if threads:
            e["OMP_NUM_THREADS"] = str(threads)
        p = subprocess.run(cmd, capture_output=True, text=True, env=e, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"{cmd} failed: {p.stderr}")
        x = np.fromfile(xp, dtype=np.float64)
        return parse_summary(p.stdout), x


def coo_to_crs(N, I, J, V):
    """DataMatrix<CRS>::convert restated (Matrix.cpp:203-228)."""
    lib = load()
    c = _coo_struct(N, I, J, V)
    ptr = np.empty(N + 1, np.int32)
    index = np.empty(max(1, len(I)), np.int32)
    value = np.empty(max(1, len(I)), np.float64)
    lib.orc_coo_to_crs(C.byref(c[0]), _p(ptr), _p(index), _p(value))
    return ptr, index[:len(I)], value[:len(I)]


def coo_to_ell(N, I, J, V):
    """DataMatrix<ELL>::convert restated (Matrix.cpp:339-361); padding 0."""
    lib = load()
    c = _coo_struct(N, I, J, V)
    max_nz = int(np.bincount(I, minlength=N).max()) if len(I) else 0
    length = np.empty(N, np.int32)
    index = np.zeros(max(1, max_nz * N), np.int32)
    data = np.zeros(max(1, max_nz * N), np.float64)
    lib.orc_coo_to_ell(C.byref(c[0]), max_nz, _p(length), _p(index), _p(data))
    return max_nz, length, index[:max_nz * N], data[:max_nz * N]


def jacobi_init(N, I, J, V):
    """Jacobi::init restated (Preconditioner.cpp:13-23), C zero-initialised."""
    lib = load()
    c = _coo_struct(N, I, J, V)
    Cd = np.zeros(N)
    lib.orc_jacobi_init(C.byref(c[0]), _p(Cd))
    return Cd


def rhs_ones(N, I, J, V):
    """k = A * 1 in COO order (CG.cpp:256-261)."""
    lib = load()
    c = _coo_struct(N, I, J, V)
    k = np.empty(N)
    lib.orc_rhs_ones(C.byref(c[0]), _p(k))
    return k


def _coo_struct(N, I, J, V):
    I = np.ascontiguousarray(I, np.int32)
    J = np.ascontiguousarray(J, np.int32)
    V = np.ascontiguousarray(V, np.float64)
    nzr = np.bincount(I, minlength=N).astype(np.int32)
    s = _Coo(N=N, nz=len(I), I=I.ctypes.data_as(C.POINTER(C.c_int)),
             J=J.ctypes.data_as(C.POINTER(C.c_int)),
             V=V.ctypes.data_as(C.POINTER(C.c_double)),
             nzPerRow=nzr.ctypes.data_as(C.POINTER(C.c_int)))
    return s, (I, J, V, nzr)  # keep the arrays alive with the struct
