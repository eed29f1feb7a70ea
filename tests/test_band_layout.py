"""The symmetric band form of A's FP32 copy, restated in numpy (no GPU).

When A is symmetric and its column offsets col - row form one set D closed
under negation, the device stores U[i][k] = A(i, i + d_k) for the
non-negative offsets d_0 = 0 < d_1 < ... and reads each lower entry from the
row above: A(i, i - d_k) = U[i - d_k][k]. These tests check that identity on
the matrices the band form takes, and that it fails for a matrix whose
values are not symmetric, which is why the device build checks them before
using the form.
"""
import numpy as np

from cgxx_b200 import generators as G


def _offsets(A):
    rows = np.repeat(np.arange(A.N), np.diff(A.ptr))
    return np.unique(A.index - rows)


def _band(A):
    D = _offsets(A)
    up = [0] + [int(d) for d in D if d > 0]
    U = np.zeros((A.N, len(up)))
    rows = np.repeat(np.arange(A.N), np.diff(A.ptr))
    for r, c, v in zip(rows, A.index, A.value):
        if c >= r:
            U[r, up.index(int(c - r))] = v
    return up, U


def _band_matvec(up, U, x):
    N = len(x)
    y = np.zeros(N)
    i = np.arange(N)
    for k, d in enumerate(up):
        j = i + d
        ok = j < N
        y[ok] += U[ok, k] * x[j[ok]]          # diagonal and upper half
        if d > 0:
            j = i - d
            ok = j >= 0
            y[ok] += U[j[ok], k] * x[j[ok]]   # lower half from the rows above
    return y


def _symmetric_offsets(A):
    D = set(int(d) for d in _offsets(A))
    return all(-d in D for d in D)


def test_band_identity_on_the_matrices_it_takes():
    rng = np.random.default_rng(3)
    cases = [G.diffusion3d(11, stencil=7, seed=1), G.poisson2d(23),
             G.diffusion3d(7, stencil=27, seed=2)]
    for A in cases:
        assert _symmetric_offsets(A)
        up, U = _band(A)
        x = rng.standard_normal(A.N)
        y = _band_matvec(up, U, x)
        assert np.allclose(y, A.matvec(x), rtol=1e-13, atol=1e-13)
    # The 7-point stencil stores 4 offsets per row (the device form's limit),
    # the 27-point one 14 (left to SELL-U).
    assert len(_band(cases[0])[0]) == 4 and len(_band(cases[2])[0]) == 14


def test_band_identity_needs_symmetric_values():
    A = G.diffusion3d(9, stencil=7, seed=4)
    value = A.value.copy()
    rows = np.repeat(np.arange(A.N), np.diff(A.ptr))
    j = int(np.nonzero((rows == A.N // 2) & (A.index > rows))[0][0])
    value[j] *= 1.5  # one upper entry changed, its mirror not
    B = G.Crs(A.N, A.ptr, A.index, value)
    up, U = _band(B)
    x = np.random.default_rng(5).standard_normal(A.N)
    assert not np.allclose(_band_matvec(up, U, x), B.matvec(x), rtol=1e-13, atol=1e-13)
