"""ctypes binding of libcgb200.so (the C ABI declared in include/cgx.h).

The library is built in-tree by cgxx_b200.build; loading fails loudly if it
is missing -- there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcgb200.so")

SUCCESS = 0
STATUS_NAMES = {
    0: "SUCCESS", 1: "INVALID_ARGUMENT", 2: "INVALID_STATE", 3: "UNSUPPORTED",
    4: "CUDA", 5: "OUT_OF_MEMORY", 6: "DEVICE", 7: "IO", 8: "NUMERICAL",
}

# cgx_vector (CG::Vector order, CG.h:22-35)
VECTOR_K, VECTOR_X, VECTOR_P, VECTOR_Q, VECTOR_R, VECTOR_Z = range(6)
VECTORS = {"K": 0, "X": 1, "P": 2, "Q": 3, "R": 4, "Z": 5}
# cgx_format (CG::MatrixFormat order, CG.h:38-47)
FORMAT_COO, FORMAT_CRS, FORMAT_ELL = range(3)
PRECOND_NONE, PRECOND_JACOBI, PRECOND_LEARNED = range(3)
PRECISION_FP64, PRECISION_MIXED = range(2)
LOOP_GRAPH, LOOP_CHUNKED, LOOP_KERNELS, LOOP_PERSISTENT, LOOP_PERSISTENT_SPLIT = range(5)


class Options(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_int),
        ("tolerance", C.c_double),
        ("preconditioner", C.c_int),
        ("precision", C.c_int),
        ("loop", C.c_int),
        ("inner_tolerance", C.c_double),
        ("max_outer", C.c_int),
        ("compute_true_residual", C.c_int),
    ]


class Result(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("residual", C.c_double),
        ("true_residual", C.c_double),
        ("converged", C.c_int),
        ("outer_iterations", C.c_int),
        ("solve_ms", C.c_double),
        ("spmv_ms", C.c_double),
        ("update_ms", C.c_double),
        ("direction_ms", C.c_double),
        ("spmv_launches", C.c_int),
        ("update_launches", C.c_int),
        ("direction_launches", C.c_int),
        ("fell_back", C.c_int),
        ("inner_form", C.c_int),
        ("inner_launches", C.c_int),
        ("inner_ms", C.c_double),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class CgxError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_PI = C.POINTER(C.c_int)
_PD = C.POINTER(C.c_double)

# name -> argtypes (restype is the int status unless listed in _RESTYPE)
PROTOTYPES = {
    "cgx_version": [_PI, _PI],
    "cgx_status_string": [_I],
    "cgx_last_error": [],
    "cgx_device_count": [_PI],
    "cgx_default_options": [C.POINTER(Options)],
    "cgx_create": [C.POINTER(_P), _I],
    "cgx_destroy": [_P],
    "cgx_set_stream": [_P, _P],
    "cgx_synchronize": [_P],
    "cgx_upload_crs": [_P, _I, _I, _P, _P, _P],
    "cgx_upload_ell": [_P, _I, _I, _I, _P, _P, _P],
    "cgx_upload_coo": [_P, _I, _I, _P, _P, _P],
    "cgx_upload_jacobi": [_P, _P],
    "cgx_jacobi_from_matrix": [_P],
    "cgx_set_vector": [_P, _I, _P],
    "cgx_get_vector": [_P, _I, _P],
    "cgx_fill_vector": [_P, _I, _D],
    "cgx_matrix_info": [_P, _PI, _PI, _PI],
    "cgx_copy": [_P, _I, _I],
    "cgx_matvec": [_P, _I, _I],
    "cgx_axpy": [_P, _D, _I, _I],
    "cgx_xpay": [_P, _I, _D, _I],
    "cgx_dot": [_P, _I, _I, _PD],
    "cgx_apply_jacobi": [_P, _I, _I],
    "cgx_solve": [_P, C.POINTER(Options), C.POINTER(Result)],
    "cgx_true_residual": [_P, _PD],
    "cgx_time_spmv": [_P, _I, _I, _PD],
    "cgx_check_wait_timeout": [_P, _I, C.POINTER(C.c_int)],
    "cgx_inner_layout": [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                         C.POINTER(C.c_longlong)],
    "cgx_inner_band": [_P, _PI, _PI],
    "cgx_learned_apply": [_P, _P, _P],
    "cgx_inner_matvec": [_P, _P, _P],
    "cgx_mtx_read": [C.c_char_p, _PI, _PI, C.POINTER(_PI), C.POINTER(_PI),
                     C.POINTER(_PD)],
    "cgx_mtx_write_symmetric_crs": [C.c_char_p, _I, _P, _P, _P],
    "cgx_free": [_P],
    "cgx_host_alloc": [C.POINTER(_P), C.c_size_t],
    "cgx_host_free": [_P],
    "cgx_dot_noalloc": [_P, _P, _I, _P, _P],
    "cgx_upload_coo_as": [_P, _I, _I, _P, _P, _P, _I],
    "cgx_download_crs": [_P, _P, _P, _P],
    "cgx_download_ell": [_P, _PI, _P, _P, _P],
    "cgx_gnn_param_count": [],
    "cgx_gnn_set_probes": [_P, _I, _I, C.c_float, _I],
    "cgx_learned_capture_residual": [_P, _I],
    "cgx_gnn_create": [C.POINTER(_P), _I, _P],
    "cgx_gnn_destroy": [_P],
    "cgx_gnn_set_params": [_P, _P],
    "cgx_gnn_get_params": [_P, _P],
    "cgx_update_crs_values": [_P, _P],
    "cgx_learned_setup": [_P],
    "cgx_learned_factor": [_P, _P, _D],
    "cgx_learned_get_factor": [_P, _PI, _P, _P, _P],
    "cgx_gnn_loss_grad": [_P, _P, _P, C.c_ulonglong, C.POINTER(C.c_float), _P],
    "cgx_gnn_train_step": [_P, _P, C.c_ulonglong, C.c_float, C.POINTER(C.c_float)],
}
_RESTYPE = {"cgx_version": None, "cgx_status_string": C.c_char_p,
            "cgx_last_error": C.c_char_p, "cgx_free": None,
            "cgx_gnn_param_count": C.c_int}

_lib = None


def load():
    """Loads libcgb200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m cgxx_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, args in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, C.c_int)
        _lib = lib
    return _lib


def check(status):
    if status != SUCCESS:
        msg = load().cgx_last_error().decode(errors="replace")
        raise CgxError(status, msg)


def device_count():
    n = C.c_int(0)
    check(load().cgx_device_count(C.byref(n)))
    return n.value


def _arr(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a, a.ctypes.data_as(C.c_void_p)


def default_options(**kw):
    o = Options()
    check(load().cgx_default_options(C.byref(o)))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class Handle:
    """One device-resident problem: matrix, Jacobi C and the vectors K..Z."""

    def __init__(self, device=0):
        self._lib = load()
        self._h = C.c_void_p()
        check(self._lib.cgx_create(C.byref(self._h), device))
        self.N = 0

    def close(self):
        if self._h:
            check(self._lib.cgx_destroy(self._h))
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- uploads (CGCUDA::doTransferTo) ---
    def upload_crs(self, ptr, index, value):
        ptr, pp = _arr(ptr, np.int32)
        index, pi = _arr(index, np.int32)
        value, pv = _arr(value, np.float64)
        N = len(ptr) - 1
        check(self._lib.cgx_upload_crs(self._h, N, len(index), pp, pi, pv))
        self.N = N

    def upload_ell(self, N, nz, max_nz, length, index, data):
        length, pl = _arr(length, np.int32)
        index, pi = _arr(index, np.int32)
        data, pd = _arr(data, np.float64)
        check(self._lib.cgx_upload_ell(self._h, N, nz, max_nz, pl, pi, pd))
        self.N = N

    def upload_coo(self, N, I, J, V):
        I, pI = _arr(I, np.int32)
        J, pJ = _arr(J, np.int32)
        V, pV = _arr(V, np.float64)
        check(self._lib.cgx_upload_coo(self._h, N, len(I), pI, pJ, pV))
        self.N = N

    def upload_coo_as(self, N, I, J, V, fmt):
        """COO entries in file order, converted on the device into `fmt`
        (FORMAT_COO, FORMAT_CRS or FORMAT_ELL)."""
        I, pI = _arr(I, np.int32)
        J, pJ = _arr(J, np.int32)
        V, pV = _arr(V, np.float64)
        check(self._lib.cgx_upload_coo_as(self._h, N, len(I), pI, pJ, pV, fmt))
        self.N = N

    def matrix_info(self):
        """(N, nz, format) of the uploaded matrix."""
        N, nz, fmt = C.c_int(0), C.c_int(0), C.c_int(0)
        check(self._lib.cgx_matrix_info(self._h, C.byref(N), C.byref(nz), C.byref(fmt)))
        return N.value, nz.value, fmt.value

    def download_crs(self):
        """The device's row layout (ptr, index, value)."""
        N, nz, _ = self.matrix_info()
        ptr = np.empty(N + 1, np.int32)
        index = np.empty(max(nz, 1), np.int32)
        value = np.empty(max(nz, 1), np.float64)
        check(self._lib.cgx_download_crs(self._h, ptr.ctypes.data_as(C.c_void_p),
                                         index.ctypes.data_as(C.c_void_p),
                                         value.ctypes.data_as(C.c_void_p)))
        return ptr, index[:nz], value[:nz]

    def download_ell(self):
        """The device's ELL matrix in the reference's column-major layout
        (max_nz, length, index, data); padding slots read 0."""
        N, _, _ = self.matrix_info()
        w = C.c_int(0)
        check(self._lib.cgx_download_ell(self._h, C.byref(w), None, None, None))
        length = np.empty(N, np.int32)
        index = np.empty(max(1, w.value * N), np.int32)
        data = np.empty(max(1, w.value * N), np.float64)
        check(self._lib.cgx_download_ell(self._h, None, length.ctypes.data_as(C.c_void_p),
                                         index.ctypes.data_as(C.c_void_p),
                                         data.ctypes.data_as(C.c_void_p)))
        return w.value, length, index[:w.value * N], data[:w.value * N]

    def upload_jacobi(self, Cdiag):
        Cdiag, pc = _arr(Cdiag, np.float64)
        check(self._lib.cgx_upload_jacobi(self._h, pc))

    def jacobi_from_matrix(self):
        check(self._lib.cgx_jacobi_from_matrix(self._h))

    # --- vectors ---
    def set_vector(self, v, host):
        host, p = _arr(host, np.float64)
        assert host.size == self.N
        check(self._lib.cgx_set_vector(self._h, VECTORS.get(v, v), p))

    def get_vector(self, v, out=None):
        """The vector as N doubles; `out` (a contiguous float64 array of N,
        e.g. from pinned_empty) receives it instead of a new array."""
        if out is None:
            out = np.empty(self.N, dtype=np.float64)
        elif out.dtype != np.float64 or out.size != self.N or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of N elements")
        check(self._lib.cgx_get_vector(self._h, VECTORS.get(v, v),
                                       out.ctypes.data_as(C.c_void_p)))
        return out

    def fill_vector(self, v, value):
        check(self._lib.cgx_fill_vector(self._h, VECTORS.get(v, v), float(value)))

    # --- per-kernel interface (CG.h:224-237) ---
    def copy(self, dst, src):
        check(self._lib.cgx_copy(self._h, VECTORS.get(dst, dst), VECTORS.get(src, src)))

    def matvec(self, x, y):
        check(self._lib.cgx_matvec(self._h, VECTORS.get(x, x), VECTORS.get(y, y)))

    def axpy(self, a, x, y):
        check(self._lib.cgx_axpy(self._h, float(a), VECTORS.get(x, x), VECTORS.get(y, y)))

    def xpay(self, x, a, y):
        check(self._lib.cgx_xpay(self._h, VECTORS.get(x, x), float(a), VECTORS.get(y, y)))

    def dot(self, a, b):
        r = C.c_double()
        check(self._lib.cgx_dot(self._h, VECTORS.get(a, a), VECTORS.get(b, b), C.byref(r)))
        return r.value

    def apply_jacobi(self, x, y):
        check(self._lib.cgx_apply_jacobi(self._h, VECTORS.get(x, x), VECTORS.get(y, y)))

    def synchronize(self):
        check(self._lib.cgx_synchronize(self._h))

    def set_stream(self, stream_ptr):
        """Run all work on an existing cudaStream_t (an int handle, e.g.
        torch.cuda.Stream().cuda_stream); 0/None restores the own stream."""
        check(self._lib.cgx_set_stream(self._h, C.c_void_p(stream_ptr or None)))

    # --- solve (CG::solve) ---
    def solve(self, options=None, **kw):
        o = options if options is not None else default_options(**kw)
        r = Result()
        check(self._lib.cgx_solve(self._h, C.byref(o), C.byref(r)))
        return r.as_dict()

    def true_residual(self):
        r = C.c_double()
        check(self._lib.cgx_true_residual(self._h, C.byref(r)))
        return r.value

    def time_spmv(self, precision, reps=20):
        """Average device time (us) of one launch of the solver's fused
        SpMV (PRECISION_FP64 or PRECISION_MIXED), timed back to back in a
        CUDA graph; overwrites Q and the last solve's scalars."""
        us = C.c_double()
        check(self._lib.cgx_time_spmv(self._h, int(precision), int(reps), C.byref(us)))
        return us.value

    def check_wait_timeout(self, which):
        """Runs a wait that cannot complete (0: the persistent solves' grid
        barrier, 1: the staged products' mbarrier) until it gives up; returns
        (status, error bits). The status is 6 (DEVICE) by design."""
        bits = C.c_int(0)
        st = self._lib.cgx_check_wait_timeout(self._h, int(which), C.byref(bits))
        return st, bits.value

    def inner_layout(self):
        """(value_slots, uniform_slices, slices) of A's FP32 copy for the
        inner SpMV; value_slots == 0 means FP32 CRS."""
        a, b, c = C.c_longlong(), C.c_longlong(), C.c_longlong()
        check(self._lib.cgx_inner_layout(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def inner_band(self):
        """Offsets (ascending from 0) stored per row by the symmetric band
        form of A's FP32 copy; empty when the inner SpMV uses another form."""
        k = C.c_int()
        offs = (C.c_int * 4)()
        check(self._lib.cgx_inner_band(self._h, C.byref(k), offs))
        return [offs[i] for i in range(k.value)]

    def inner_matvec(self, x):
        """y = A x (float32) by the inner FP32 SpMV of the mixed paths."""
        x, px = _arr(x, np.float32)
        y = np.empty_like(x)
        check(self._lib.cgx_inner_matvec(self._h, px, y.ctypes.data_as(C.c_void_p)))
        return y

    # --- learned preconditioner ---
    def update_crs_values(self, value):
        value, pv = _arr(value, np.float64)
        check(self._lib.cgx_update_crs_values(self._h, pv))

    def update_crs_values_ptr(self, device_ptr):
        """Same as update_crs_values with the values in device memory."""
        check(self._lib.cgx_update_crs_values(self._h, C.c_void_p(device_ptr)))

    def learned_setup(self):
        check(self._lib.cgx_learned_setup(self._h))

    def learned_capture_residual(self, col):
        """Store r = K - A X (Jacobi-scaled, unit RMS) as probe column col
        of the learned state (see Gnn.set_probes)."""
        check(self._lib.cgx_learned_capture_residual(self._h, int(col)))

    def learned_factor(self, gnn, eps=0.0):
        check(self._lib.cgx_learned_factor(self._h, gnn._g, float(eps)))

    def learned_apply(self, r):
        """z = G (G^T r) + eps C r (float32), as the inner solve applies it."""
        r, pr = _arr(r, np.float32)
        z = np.empty_like(r)
        check(self._lib.cgx_learned_apply(self._h, pr, z.ctypes.data_as(C.c_void_p)))
        return z

    def learned_get_factor(self):
        """(ghat, rows, cols) of the unscaled factor on its pattern."""
        n = C.c_int()
        check(self._lib.cgx_learned_get_factor(self._h, C.byref(n), None, None, None))
        g = np.empty(n.value, np.float32)
        r = np.empty(n.value, np.int32)
        c = np.empty(n.value, np.int32)
        check(self._lib.cgx_learned_get_factor(
            self._h, C.byref(n), g.ctypes.data_as(C.c_void_p),
            r.ctypes.data_as(C.c_void_p), c.ctypes.data_as(C.c_void_p)))
        return g, r, c


class Gnn:
    """Parameters (and Adam state) of the learned preconditioner's network on
    one device."""

    def __init__(self, device=0, params=None):
        self._lib = load()
        self._g = C.c_void_p()
        self.nparams = self._lib.cgx_gnn_param_count()
        p = None
        if params is not None:
            params = np.ascontiguousarray(params, np.float32)
            assert params.size == self.nparams
            p = params.ctypes.data_as(C.c_void_p)
        check(self._lib.cgx_gnn_create(C.byref(self._g), device, p))

    def close(self):
        if self._g:
            check(self._lib.cgx_gnn_destroy(self._g))
            self._g = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params):
        params = np.ascontiguousarray(params, np.float32)
        assert params.size == self.nparams
        check(self._lib.cgx_gnn_set_params(self._g, params.ctypes.data_as(C.c_void_p)))

    def get_params(self):
        out = np.empty(self.nparams, np.float32)
        check(self._lib.cgx_gnn_get_params(self._g, out.ctypes.data_as(C.c_void_p)))
        return out

    def loss_grad(self, handle, probes=None, seed=0):
        loss = C.c_float()
        grad = np.empty(self.nparams, np.float32)
        pp = None
        if probes is not None:
            probes = np.ascontiguousarray(probes, np.float32)
            pp = probes.ctypes.data_as(C.c_void_p)
        check(self._lib.cgx_gnn_loss_grad(self._g, handle._h, pp, seed, C.byref(loss),
                                          grad.ctypes.data_as(C.c_void_p)))
        return loss.value, grad

    def set_probes(self, smooth_steps=0, smooth_cols=0, smooth_scale=1.0, residual_cols=0):
        """Probe recipe of loss_grad (probes=None) and train_step: the last
        residual_cols columns are the handle's residual snapshots, the
        smooth_cols before them Rademacher columns smoothed by smooth_steps
        damped-Jacobi steps on Ahat and scaled by smooth_scale."""
        check(self._lib.cgx_gnn_set_probes(self._g, int(smooth_steps), int(smooth_cols),
                                           float(smooth_scale), int(residual_cols)))

    def train_step(self, handle, seed, lr):
        loss = C.c_float()
        check(self._lib.cgx_gnn_train_step(self._g, handle._h, seed, float(lr),
                                           C.byref(loss)))
        return loss.value


def pinned_empty(n, dtype):
    """numpy array of n elements in page-locked host memory (cgx_host_alloc);
    the memory is released when the array is garbage collected."""
    dt = np.dtype(dtype)
    lib = load()
    p = C.c_void_p()
    check(lib.cgx_host_alloc(C.byref(p), max(1, n * dt.itemsize)))
    buf = (C.c_byte * max(1, n * dt.itemsize)).from_address(p.value)
    arr = np.frombuffer(buf, dtype=dt, count=n)

    class _Owner:
        def __init__(self, ptr):
            self.ptr = ptr

        def __del__(self):
            try:
                lib.cgx_host_free(self.ptr)
            except Exception:
                pass

    # keep the owner alive as long as the array
    arr = arr.view(type=_PinnedArray)
    arr._owner = _Owner(p)
    return arr


class _PinnedArray(np.ndarray):
    _owner = None


def mtx_read(path):
    """MatrixMarket reader with the reference's entry order (Matrix.cpp:13-111).
    Returns (N, I, J, V) as numpy arrays."""
    lib = load()
    N = C.c_int()
    nz = C.c_int()
    I = _PI()
    J = _PI()
    V = _PD()
    check(lib.cgx_mtx_read(os.fsencode(path), C.byref(N), C.byref(nz),
                           C.byref(I), C.byref(J), C.byref(V)))
    try:
        n = nz.value
        Ia = np.ctypeslib.as_array(I, shape=(n,)).copy() if n else np.zeros(0, np.int32)
        Ja = np.ctypeslib.as_array(J, shape=(n,)).copy() if n else np.zeros(0, np.int32)
        Va = np.ctypeslib.as_array(V, shape=(n,)).copy() if n else np.zeros(0, np.float64)
    finally:
        lib.cgx_free(C.cast(I, C.c_void_p))
        lib.cgx_free(C.cast(J, C.c_void_p))
        lib.cgx_free(C.cast(V, C.c_void_p))
    return N.value, Ia, Ja, Va


def mtx_write_symmetric_crs(path, ptr, index, value):
    ptr, pp = _arr(ptr, np.int32)
    index, pi = _arr(index, np.int32)
    value, pv = _arr(value, np.float64)
    check(load().cgx_mtx_write_symmetric_crs(os.fsencode(path), len(ptr) - 1, pp, pi, pv))
