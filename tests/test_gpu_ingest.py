"""COO -> CRS / ELL on the device (cgx_upload_coo_as) against the reference's
conversion on the host (DataMatrix<CRS>::convert, Matrix.cpp:203-228, and
DataMatrix<ELL>::convert, Matrix.cpp:339-361, as the oracle restates them):
bit for bit, from the COO the reference's reader produces (entry order =
file order, symmetric entries mirrored right after each stored one).
"""
import os

import numpy as np
import pytest

import cgxx_b200 as cg
from cgxx_b200 import generators as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _check(N, I, J, V):
    ptr, idx, val = O.coo_to_crs(N, I, J, V)
    w, length, eidx, edat = O.coo_to_ell(N, I, J, V)
    with cg.Handle(0) as h:
        for fmt in (cg.FORMAT_CRS, cg.FORMAT_COO):
            h.upload_coo_as(N, I, J, V, fmt)
            p, i, v = h.download_crs()
            assert np.array_equal(p, ptr) and np.array_equal(i, idx)
            assert np.array_equal(v.view(np.int64), val.view(np.int64))
        h.upload_coo_as(N, I, J, V, cg.FORMAT_ELL)
        dw, dl, di, dd = h.download_ell()
        assert dw == w and np.array_equal(dl, length)
        used = (np.arange(w)[:, None] < length[None, :]).ravel()  # slot j of row i at j*N+i
        assert np.array_equal(di[used], eidx[used])
        assert np.array_equal(dd[used].view(np.int64), edat[used].view(np.int64))
        p, i, v = h.download_crs()  # the row layout kept for the mixed paths
        assert np.array_equal(p, ptr) and np.array_equal(i, idx)


@pytest.mark.parametrize("name", ["poisson16.mtx", "spd_ragged300.mtx", "diffusion27_8.mtx"])
def test_golden_files(name):
    st, N, I, J, V = O.read_mtx(os.path.join(GOLDEN, name))
    assert st == 0
    _check(N, I, J, V)


@pytest.mark.parametrize("N,nz,seed", [(1, 3, 0), (37, 1000, 1), (5000, 70001, 2),
                                       (300000, 250000, 3)])
def test_unsorted_entries_with_repeats_and_empty_rows(N, nz, seed):
    """Entries in random order, several per (row, column), rows without
    entries: each row keeps its entries' file order, repeats included."""
    rng = np.random.default_rng(seed)
    I = rng.integers(0, N, nz).astype(np.int32)
    J = rng.integers(0, N, nz).astype(np.int32)
    V = rng.standard_normal(nz)
    _check(N, I, J, V)


def test_benchmark_matrix_160():
    """The 7-point 160^3 benchmark matrix (28.5M entries, 3 radix passes)."""
    A = G.diffusion3d(160, 7, sigma=1.0, corr_len=8.0, seed=2024)
    I, J, V = G.symmetric_file_coo(A)
    _check(A.N, I, J, V)


def test_invalid_indices_are_rejected():
    with cg.Handle(0) as h:
        for I, J, what in (([0, 5], [0, 0], "row index"), ([0, 1], [0, -1], "column index")):
            with pytest.raises(cg.CgxError) as e:
                h.upload_coo_as(3, np.array(I), np.array(J), np.ones(2), cg.FORMAT_CRS)
            assert e.value.status == 1 and what in e.value.message


def test_solve_after_device_conversion_equals_host_upload():
    A = G.diffusion3d(20, 7, seed=3)
    b, _ = G.rhs_for(A, seed=4)
    I, J, V = G.symmetric_file_coo(A)
    Cd = 1.0 / A.diagonal()
    xs = []
    with cg.Handle(0) as h:
        for up in (lambda: h.upload_crs(A.ptr, A.index, A.value),
                   lambda: h.upload_coo_as(A.N, I, J, V, cg.FORMAT_CRS),
                   lambda: h.upload_coo_as(A.N, I, J, V, cg.FORMAT_ELL)):
            up()
            h.upload_jacobi(Cd)
            h.set_vector("K", b)
            h.fill_vector("X", 0.0)
            r = h.solve(max_iterations=5000, tolerance=1e-9)
            assert r["converged"] == 1
            xs.append(h.get_vector("X"))
    assert np.array_equal(xs[0], xs[1])  # the same layout: the same bits
    # ELL runs another SpMV kernel, whose dot products add the partial sums
    # in another grouping.
    assert np.linalg.norm(xs[2] - xs[0]) <= 1e-10 * np.linalg.norm(xs[0])
