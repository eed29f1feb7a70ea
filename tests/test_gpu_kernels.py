"""Per-kernel parity of the device library against the oracle, through the C
ABI (the reference's per-kernel interface, CG.h:224-237).

SpMV (CRS, ELL, COO), axpy, xpay and the Jacobi apply keep the reference's
operation order and rounding (serial/SerialCG.cpp:79-174), so they are
compared bit for bit. Dot products sum in a different order: relative
tolerance 1e-13.
"""
import numpy as np
import pytest

from conftest import random_crs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = [1, 31, 33, 257, 1000, 4099]


def _x(N, seed=1):
    return np.random.default_rng(seed).standard_normal(N)


@pytest.mark.parametrize("N", SIZES)
def test_spmv_crs_bitexact(handle, N):
    A = random_crs(N, 0, 40, seed=N)
    handle.upload_crs(A.ptr, A.index, A.value)
    x = _x(N)
    handle.set_vector("X", x)
    handle.matvec("X", "Q")
    q = handle.get_vector("Q")
    assert np.array_equal(q, O.matvec_crs(A.ptr, A.index, A.value, x))


def test_spmv_crs_long_rows(handle):
    # Tiles above the staging capacity take the direct-load path.
    from cgxx_b200 import generators as G
    rng = np.random.default_rng(5)
    N = 3000
    lens = rng.integers(0, 8, N)
    lens[17] = 9000
    lens[2500:2510] = 700
    rows = np.repeat(np.arange(N), lens)
    cols = rng.integers(0, N, lens.sum())
    A = G.crs_from_unsorted(N, rows, cols, rng.standard_normal(lens.sum()))
    handle.upload_crs(A.ptr, A.index, A.value)
    x = _x(N, 2)
    handle.set_vector("X", x)
    handle.matvec("X", "Q")
    assert np.array_equal(handle.get_vector("Q"), O.matvec_crs(A.ptr, A.index, A.value, x))


@pytest.mark.parametrize("N", SIZES)
def test_spmv_ell_bitexact(handle, N):
    from cgxx_b200 import generators as G
    A = random_crs(N, 0, 40, seed=N + 7)
    max_nz, length, index, data = G.to_ell(A)
    handle.upload_ell(N, A.nz, max_nz, length, index, data)
    x = _x(N)
    handle.set_vector("X", x)
    handle.matvec("X", "Q")
    assert np.array_equal(handle.get_vector("Q"), O.matvec_ell(N, length, index, data, x))


@pytest.mark.parametrize("width", [1, 7, 16])
@pytest.mark.parametrize("N", SIZES)
def test_spmv_ell_staged_bitexact(handle, N, width):
    # Widths up to 16 take the bulk-copy staged kernel. The reference leaves
    # padding slots uninitialised (Matrix.cpp:339-361): they hold NaN values
    # and out-of-range indices here, which must never be read. Empty rows and
    # sizes that are not a multiple of the 256-row tile are included.
    from cgxx_b200 import generators as G
    A = random_crs(N, 0, width, seed=N + width)
    max_nz, length, index, data = G.to_ell(A)
    assert max_nz <= width
    slot = np.arange(max_nz)[:, None]
    pad = (slot >= length[None, :]).reshape(-1)
    index = index.copy()
    data = data.copy()
    index[pad] = -(N + 3)
    data[pad] = np.nan
    handle.upload_ell(N, A.nz, max_nz, length, index, data)
    x = _x(N, 3)
    handle.set_vector("X", x)
    handle.matvec("X", "Q")
    assert np.array_equal(handle.get_vector("Q"), O.matvec_ell(N, length, index, data, x))


@pytest.mark.parametrize("N", SIZES)
def test_spmv_coo_bitexact(handle, N):
    rng = np.random.default_rng(N)
    nz = 7 * N
    I = rng.integers(0, N, nz).astype(np.int32)  # unsorted, repeated rows
    J = rng.integers(0, N, nz).astype(np.int32)
    V = rng.standard_normal(nz)
    handle.upload_coo(N, I, J, V)
    x = _x(N)
    handle.set_vector("X", x)
    handle.matvec("X", "Q")
    assert np.array_equal(handle.get_vector("Q"), O.matvec_coo(N, I, J, V, x))


def test_spmv_poisson_large(handle):
    from cgxx_b200 import generators as G
    A = G.poisson2d(700)
    handle.upload_crs(A.ptr, A.index, A.value)
    x = _x(A.N, 3)
    handle.set_vector("X", x)
    handle.matvec("X", "Q")
    assert np.array_equal(handle.get_vector("Q"), O.matvec_crs(A.ptr, A.index, A.value, x))


@pytest.mark.parametrize("N", [1, 2, 3, 1001, 100003])
def test_blas1_bitexact(handle, N):
    A = random_crs(N, 1, 3, seed=3)
    handle.upload_crs(A.ptr, A.index, A.value)
    rng = np.random.default_rng(N)
    a, b, c = rng.standard_normal(N), rng.standard_normal(N), rng.uniform(0.5, 2, N)
    handle.set_vector("P", a)
    handle.set_vector("Q", b)
    handle.axpy(0.37, "P", "Q")
    assert np.array_equal(handle.get_vector("Q"), O.axpy(0.37, a, b))
    handle.set_vector("Q", b)
    handle.xpay("P", -1.25, "Q")
    assert np.array_equal(handle.get_vector("Q"), O.xpay(a, -1.25, b))
    handle.upload_jacobi(c)
    handle.apply_jacobi("P", "Z")
    assert np.array_equal(handle.get_vector("Z"), O.jacobi_apply(c, a))
    handle.copy("R", "P")
    assert np.array_equal(handle.get_vector("R"), a)
    d = handle.dot("P", "Q")
    ref = O.dot(a, handle.get_vector("Q"))
    assert abs(d - ref) <= 1e-13 * max(1.0, np.abs(a).dot(np.abs(handle.get_vector("Q"))))


def test_jacobi_from_matrix(handle):
    A = random_crs(2000, 0, 9, seed=11)
    handle.upload_crs(A.ptr, A.index, A.value)
    handle.jacobi_from_matrix()
    rng = np.random.default_rng(0)
    x = rng.standard_normal(A.N)
    handle.set_vector("R", x)
    handle.apply_jacobi("R", "Z")
    # Reference semantics: last diagonal entry of the row wins (file order).
    Cd = np.zeros(A.N)
    rows = A.rows()
    for j in np.nonzero(A.index == rows)[0]:
        Cd[rows[j]] = 1 / A.value[j]
    assert np.array_equal(handle.get_vector("Z"), Cd * x)


def test_invalid_matrix_rejected(handle):
    import cgxx_b200
    ptr = np.array([0, 2, 3], np.int32)
    with pytest.raises(cgxx_b200.CgxError) as e:
        handle.upload_crs(ptr, np.array([0, 5, 1], np.int32), np.ones(3))
    assert e.value.status == 1
    with pytest.raises(cgxx_b200.CgxError):
        handle.upload_crs(np.array([0, 2, 1], np.int32), np.array([0, 1], np.int32), np.ones(2))


def test_ell_upload_checks_lengths_against_nz(handle):
    """nz sizes the row-layout copies that the mixed and learned paths build
    from an ELL matrix, so an upload whose nz is not the sum of the row
    lengths, or with a length outside [0, maxNz], is rejected on the host and
    leaves the previous matrix in place."""
    import cgxx_b200 as cg
    from cgxx_b200 import generators as G
    A = random_crs(257, 0, 9, seed=41)
    max_nz, length, index, data = G.to_ell(A)
    handle.upload_ell(A.N, A.nz, max_nz, length, index, data)
    x = _x(A.N)
    handle.set_vector("X", x)
    for nz, lens in ((A.nz + 1, length), (A.nz, np.where(np.arange(A.N) == 5, max_nz + 1, length))):
        with pytest.raises(cg.CgxError) as e:
            handle.upload_ell(A.N, nz, max_nz, lens.astype(np.int32), index, data)
        assert e.value.status == 1 and "invalid ELL matrix" in e.value.message
    handle.matvec("X", "Q")
    assert np.array_equal(handle.get_vector("Q"), O.matvec_ell(A.N, length, index, data, x))
