"""The oracle pinned against the reference (CPU only).

tests/golden/reference_runs.json holds what the reference's own cg_serial
printed and computed (tests/golden/make_golden.py); the C restatement must
reproduce every case bit for bit: iteration count, printed residual, solution
bytes. Where oracle/_ref is built (reference tree present), extra seeded
cases are compared live against the reference's serial and OpenMP binaries.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from cgxx_b200 import generators as G
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
RUNS = json.load(open(os.path.join(GOLD, "reference_runs.json")))


def sha(x):
    return hashlib.sha256(np.ascontiguousarray(x, dtype="<f8").tobytes()).hexdigest()


def oracle_solve_file(path, fmt, pc, max_iter, tol=1e-9, rhs=None):
    st, N, I, J, V = O.read_mtx(path)
    assert st == 0
    k = O.rhs_ones(N, I, J, V) if rhs is None else rhs
    Cd = O.jacobi_init(N, I, J, V) if pc == "jacobi" else None
    if fmt == "CRS":
        ptr, idx, val = O.coo_to_crs(N, I, J, V)
        return O.cg_solve_crs(ptr, idx, val, k, Cd, max_iter=max_iter, tol=tol)
    if fmt == "ELL":
        m, length, idx, data = O.coo_to_ell(N, I, J, V)
        return O.cg_solve_ell(N, len(I), length, idx, data, k, Cd, max_iter=max_iter, tol=tol)
    return O.cg_solve_coo(N, I, J, V, k, Cd, max_iter=max_iter, tol=tol)


@pytest.mark.parametrize("case", RUNS["cases"],
                         ids=lambda c: f"{c['matrix']}-{c['format']}-{c['preconditioner']}-{c['max_iter']}")
def test_oracle_matches_reference_golden(case):
    x, it, res = oracle_solve_file(os.path.join(GOLD, case["matrix"]), case["format"],
                                   case["preconditioner"], case["max_iter"])
    assert it == case["iterations"]
    assert "%e" % res == "%e" % case["residual_printed"]
    assert sha(x) == case["x_sha256"]
    if case["x"] is not None:
        assert np.array_equal(x, np.array(case["x"]))
    assert (O.load().orc_check_ones(len(x), x.ctypes.data_as(__import__("ctypes").c_void_p),
                                    1e-5) == 0) == case["correct"]


def test_poisson256_golden(tmp_path):
    g = RUNS["poisson256"]
    A = G.poisson2d(256)
    p = str(tmp_path / "p256.mtx")
    G.write_mtx_symmetric_py(p, A)
    assert hashlib.sha256(open(p, "rb").read()).hexdigest() == g["mtx_sha256"]
    x, it, res = oracle_solve_file(p, "CRS", "jacobi", 1000)
    assert it == g["iterations"] == 482
    assert "%e" % res == "%e" % g["residual_printed"]
    assert sha(x) == g["x_sha256"]


def test_generator_order_matches_reader():
    # The CRS the generators build equals the reference reader + conversion
    # applied to the file the generators write.
    for path, A in [("poisson16.mtx", G.poisson2d(16)),
                    ("diffusion27_8.mtx",
                     G.diffusion3d(8, stencil=27, sigma=1.0, corr_len=3.0, seed=5))]:
        st, N, I, J, V = O.read_mtx(os.path.join(GOLD, path))
        I2, J2, V2 = G.symmetric_file_coo(A)
        assert np.array_equal(I, I2) and np.array_equal(J, J2) and np.array_equal(V, V2)
        ptr, idx, val = O.coo_to_crs(N, I, J, V)
        assert np.array_equal(ptr, A.ptr) and np.array_equal(idx, A.index)
        assert np.array_equal(val, A.value)


def test_ell_conversion_matches_generator():
    A = G.diffusion3d(8, stencil=27, sigma=1.0, corr_len=3.0, seed=5)
    st, N, I, J, V = O.read_mtx(os.path.join(GOLD, "diffusion27_8.mtx"))
    m, length, idx, data = O.coo_to_ell(N, I, J, V)
    m2, l2, i2, d2 = G.to_ell(A)
    assert m == m2 and np.array_equal(length, l2)
    assert np.array_equal(idx, i2) and np.array_equal(data, d2)


def test_rhs_ones_matches_generator():
    A = G.diffusion3d(8, stencil=7, seed=1)
    I, J, V = G.symmetric_file_coo(A)
    assert np.array_equal(O.rhs_ones(A.N, I, J, V), G.rhs_ones(A))


@pytest.mark.parametrize("name,status", [("bad_banner.mtx", 2), ("bad_storage.mtx", 3),
                                         ("not_square.mtx", 4), ("does_not_exist.mtx", 1)])
def test_oracle_reader_errors(name, status):
    st, *_ = O.read_mtx(os.path.join(GOLD, name))
    assert st == status


def test_mixed_oracle_converges():
    A = G.diffusion3d(12, stencil=7, seed=3)
    b, xs = G.rhs_for(A, seed=1)
    Cd = 1 / A.diagonal()
    x, it, outer, tr = O.mixed_ir_solve(A.ptr, A.index, A.value, Cd, b)
    assert tr <= 1e-9 and outer >= 2
    assert np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b) <= 1e-9


# --- live comparison with the reference binaries (where they were built) -------

needs_ref = pytest.mark.skipif(O.ref_binary("ref_harness_serial") is None,
                               reason="oracle/_ref not built (reference tree absent)")


@needs_ref
@pytest.mark.parametrize("seed", [1, 2])
def test_live_reference_random_rhs(tmp_path, seed):
    A = G.diffusion3d(10, stencil=7, sigma=1.5, corr_len=4.0, seed=seed)
    p = str(tmp_path / "d.mtx")
    G.write_mtx_symmetric_py(p, A)
    b, _ = G.rhs_for(A, seed=seed)
    summ, xr = O.run_ref_harness(p, rhs=b, backend="serial")
    x, it, res = O.cg_solve_crs(A.ptr, A.index, A.value, b, 1 / A.diagonal())
    assert it == summ["iterations"][0]
    assert np.array_equal(x, xr)


@needs_ref
def test_live_reference_openmp_close_to_serial(tmp_path):
    A = G.diffusion3d(12, stencil=7, seed=4)
    p = str(tmp_path / "d.mtx")
    G.write_mtx_symmetric_py(p, A)
    s1, x1 = O.run_ref_harness(p, backend="serial")
    s2, x2 = O.run_ref_harness(p, backend="omp", threads=4)
    assert abs(s1["iterations"][0] - s2["iterations"][0]) <= 1
    assert np.linalg.norm(x1 - x2) / np.linalg.norm(x1) < 1e-10
