"""Parity of the fused device solve (cgx_solve) with the oracle's CG::solve.

Bar (from the project's goal): the solution's relative difference to the
oracle's is <= 1e-8, the iteration count is within 2 %, and the reference's
CG_CHECK_TOLERANCE check (|x_i - 1| <= 1e-5 for k = A*1) passes.
"""
import numpy as np
import pytest

import cgxx_b200 as cg
from cgxx_b200 import generators as G
from conftest import random_crs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

X_TOL = 1e-8


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def upload(h, A, fmt):
    if fmt == "CRS":
        h.upload_crs(A.ptr, A.index, A.value)
    elif fmt == "ELL":
        m, l, i, d = G.to_ell(A)
        h.upload_ell(A.N, A.nz, m, l, i, d)
    else:
        I, J, V = G.symmetric_file_coo(A)
        h.upload_coo(A.N, I, J, V)


def solve_case(h, A, k, fmt="CRS", precond="jacobi", loop=cg.LOOP_GRAPH, max_iter=1000,
               tol=1e-9):
    upload(h, A, fmt)
    Cd = 1.0 / A.diagonal()
    if precond == "jacobi":
        h.upload_jacobi(Cd)
    h.set_vector("K", k)
    h.fill_vector("X", 0.0)
    pc = cg.PRECOND_JACOBI if precond == "jacobi" else cg.PRECOND_NONE
    res = h.solve(max_iterations=max_iter, tolerance=tol, preconditioner=pc, loop=loop)
    x = h.get_vector("X")
    xo, ito, reso = O.cg_solve_crs(A.ptr, A.index, A.value, k,
                                   Cd if precond == "jacobi" else None,
                                   max_iter=max_iter, tol=tol)
    return res, x, xo, ito, reso


@pytest.mark.parametrize("loop", [cg.LOOP_GRAPH, cg.LOOP_CHUNKED, cg.LOOP_KERNELS])
@pytest.mark.parametrize("fmt", ["CRS", "ELL", "COO"])
def test_poisson256_matches_reference(handle, fmt, loop):
    A = G.poisson2d(256)
    k = G.rhs_ones(A)
    res, x, xo, ito, reso = solve_case(handle, A, k, fmt=fmt, loop=loop)
    assert ito == 482  # the reference's cg_serial on this matrix
    assert abs(res["iterations"] - ito) <= 0.02 * ito
    assert res["converged"] == 1
    assert res["residual"] <= 1e-9
    assert rel(x, xo) <= X_TOL
    assert np.sum(np.abs(x - 1.0) > 1e-5) == 0  # CG::check


@pytest.mark.parametrize("precond", ["jacobi", "none"])
@pytest.mark.parametrize("N", [1, 2, 33, 1000, 20000])
def test_random_spd(handle, N, precond):
    A = random_crs(N, 0, 40, seed=N, spd=True)
    b, xs = G.rhs_for(A, seed=N)
    res, x, xo, ito, reso = solve_case(handle, A, b, precond=precond, max_iter=5000)
    assert abs(res["iterations"] - ito) <= max(1, 0.02 * ito)
    assert rel(x, xo) <= X_TOL


@pytest.mark.parametrize("stencil", [7, 27])
def test_diffusion3d(handle, stencil):
    A = G.diffusion3d(24, stencil=stencil, sigma=1.0, corr_len=4.0, seed=3)
    b, xs = G.rhs_for(A, seed=4)
    for fmt in ("CRS", "ELL"):
        res, x, xo, ito, reso = solve_case(handle, A, b, fmt=fmt, max_iter=3000)
        assert abs(res["iterations"] - ito) <= max(1, 0.02 * ito)
        assert rel(x, xo) <= X_TOL
        assert rel(x, xs) <= 1e-6


def test_iteration_limit(handle):
    A = G.poisson2d(64)
    k = G.rhs_ones(A)
    for loop in (cg.LOOP_GRAPH, cg.LOOP_CHUNKED, cg.LOOP_KERNELS):
        res, x, xo, ito, reso = solve_case(handle, A, k, max_iter=17, loop=loop)
        assert res["iterations"] == 17 == ito
        assert res["converged"] == 0
        assert rel(x, xo) <= 1e-10
        assert abs(res["residual"] - reso) <= 1e-8 * reso


def test_repeat_solve_is_deterministic(handle):
    A = G.diffusion3d(20, stencil=7, seed=9)
    b, _ = G.rhs_for(A, seed=1)
    r1, x1, *_ = solve_case(handle, A, b)
    handle.fill_vector("X", 0.0)
    r2 = handle.solve(max_iterations=1000, tolerance=1e-9)
    x2 = handle.get_vector("X")
    assert r1["iterations"] == r2["iterations"]
    assert np.array_equal(x1, x2)


def test_mixed_precision_reaches_fp64_tolerance(handle):
    A = G.diffusion3d(32, stencil=7, sigma=1.0, corr_len=8.0, seed=2)
    b, xs = G.rhs_for(A, seed=2)
    handle.upload_crs(A.ptr, A.index, A.value)
    Cd = 1.0 / A.diagonal()
    handle.upload_jacobi(Cd)
    handle.set_vector("K", b)
    handle.fill_vector("X", 0.0)
    res = handle.solve(max_iterations=5000, tolerance=1e-9, precision=cg.PRECISION_MIXED)
    x = handle.get_vector("X")
    assert res["converged"] == 1
    assert res["outer_iterations"] >= 2
    # FP64 true residual computed independently on the CPU.
    tr = np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)
    assert tr <= 1e-9
    # Error against a tight FP64 oracle solve.
    xo, _, _ = O.cg_solve_crs(A.ptr, A.index, A.value, b, Cd, max_iter=20000, tol=1e-13)
    assert rel(x, xo) <= 1e-6
    # Oracle of the mixed scheme: same number of refinement steps, inner
    # iteration total within 5 %.
    _, it_o, outer_o, tr_o = O.mixed_ir_solve(A.ptr, A.index, A.value, Cd, b)
    assert res["outer_iterations"] == outer_o
    assert abs(res["iterations"] - it_o) <= 0.05 * it_o + 2


def test_mixed_loops_agree(handle):
    A = G.diffusion3d(16, stencil=27, seed=5)
    b, _ = G.rhs_for(A, seed=3)
    handle.upload_crs(A.ptr, A.index, A.value)
    handle.upload_jacobi(1.0 / A.diagonal())
    handle.set_vector("K", b)
    out = []
    for loop in (cg.LOOP_GRAPH, cg.LOOP_CHUNKED, cg.LOOP_KERNELS):
        handle.fill_vector("X", 0.0)
        r = handle.solve(max_iterations=5000, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                         loop=loop)
        out.append((r["iterations"], handle.get_vector("X")))
        assert r["converged"] == 1
    assert out[0][0] == out[1][0] == out[2][0]
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][1], out[2][1])


def _shuffle_rows(A, seed):
    """The same matrix with every row's entries in a random order."""
    rng = np.random.default_rng(seed)
    index, value = A.index.copy(), A.value.copy()
    for i in range(A.N):
        a, b = A.ptr[i], A.ptr[i + 1]
        p = a + rng.permutation(b - a)
        index[a:b], value[a:b] = A.index[p], A.value[p]
    return G.Crs(A.N, A.ptr, index, value)


def _asymmetric(A, rel=1e-4):
    """A with the entry above the diagonal in row N/2 scaled by 1 + rel: no
    longer exactly symmetric, close enough for CG to converge."""
    value = A.value.copy()
    i = A.N // 2
    a, b = A.ptr[i], A.ptr[i + 1]
    j = a + int(np.nonzero(A.index[a:b] > i)[0][0])
    value[j] *= 1.0 + rel
    return G.Crs(A.N, A.ptr, A.index, value)


# Inner SpMV form per case: the symmetric band for the 7-point stencil
# (unsorted rows included), the 2D 5-point stencil and a tridiagonal matrix
# (3 and 2 stored offsets: padding slots), SELL-U for the 27-point stencil
# (14 stored offsets) and for a 7-point stencil whose values are not exactly
# symmetric, FP32 CRS for matrices whose slices would be mostly per-row.
_IRREGULAR = {
    "ragged": "crs",
    "unsorted": "band",
    "poisson2d": "band",
    "tridiagonal": "band",
    "wide": "crs",
    "stencil27_odd": "sellu",
    "stencil7_asym": "sellu",
}


def _tridiagonal(N, seed):
    """SPD tridiagonal matrix with random couplings (offsets -1, 0, 1)."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.5, 2.0, N - 1)
    rows = np.concatenate([np.arange(N), np.arange(N - 1), np.arange(1, N)])
    cols = np.concatenate([np.arange(N), np.arange(1, N), np.arange(N - 1)])
    diag = np.zeros(N)
    diag[:-1] += c
    diag[1:] += c
    vals = np.concatenate([diag + 0.01, -c, -c])
    return G.crs_from_unsorted(N, rows, cols, vals)


def _irregular_matrix(case):
    if case == "ragged":
        return random_crs(1007, max_len=12, seed=3, spd=True)
    if case == "unsorted":
        return _shuffle_rows(G.diffusion3d(13, stencil=7, seed=4), seed=5)
    if case == "wide":
        return random_crs(777, max_len=80, seed=4, spd=True)
    if case == "stencil27_odd":
        return G.diffusion3d(11, stencil=27, seed=6)
    if case == "poisson2d":
        return G.poisson2d(37)
    if case == "tridiagonal":
        return _tridiagonal(1999, seed=8)
    return _asymmetric(G.diffusion3d(11, stencil=7, seed=6))


def _expected_band(A):
    """The offsets d >= 0 of A's entries (col - row), ascending."""
    rows = np.repeat(np.arange(A.N), np.diff(A.ptr))
    return sorted(set(int(d) for d in np.unique(A.index - rows) if d >= 0))


def _check_inner_form(handle, A, form):
    slots, uniform, slices = handle.inner_layout()
    band = handle.inner_band()
    if form == "band":
        assert band == _expected_band(A) and slots == 0
    elif form == "sellu":
        assert band == [] and slices == (A.N + 31) // 32 and uniform == slices
        assert slots >= A.nz
    else:
        assert band == [] and slots == 0


@pytest.mark.parametrize("case", sorted(_IRREGULAR))
def test_inner_product_on_every_form(handle, case):
    """y = A x by the FP32 inner SpMV, on each of its forms, against the FP64
    product of the same FP32 x: within 4e-6 of sum |a_ij x_j| per row. x has
    large entries at both ends, where the band form masks the rows above row
    0 and clamps the columns past N - 1."""
    A = _irregular_matrix(case)
    handle.upload_crs(A.ptr, A.index, A.value)
    handle.upload_jacobi(1.0 / A.diagonal())
    x = np.random.default_rng(11).standard_normal(A.N).astype(np.float32)
    x[:3] = 1e3
    x[-3:] = -1e3
    y = handle.inner_matvec(x)
    _check_inner_form(handle, A, _IRREGULAR[case])
    xd = x.astype(np.float64)
    ref = A.matvec(xd)
    absA = G.Crs(A.N, A.ptr, A.index, np.abs(A.value))
    bound = 4e-6 * absA.matvec(np.abs(xd)) + 1e-30
    assert np.all(np.abs(y.astype(np.float64) - ref) <= bound)


@pytest.mark.parametrize("case", sorted(_IRREGULAR))
def test_mixed_on_irregular_patterns(handle, case):
    """The mixed solve on every form of the FP32 inner SpMV: the symmetric
    band for the 7-point stencil (rows stored out of order), SELL-U for the
    27-point stencil and when the values are not exactly symmetric (uniform
    slices with zero-filled missing neighbours at the boundary, a last slice
    shorter than 32 rows), and FP32 CRS for matrices whose slices would be
    mostly per-row (ragged random rows, rows whose offsets span more than 32
    slots)."""
    A = _irregular_matrix(case)
    b, _ = G.rhs_for(A, seed=7)
    handle.upload_crs(A.ptr, A.index, A.value)
    Cd = 1.0 / A.diagonal()
    handle.upload_jacobi(Cd)
    handle.set_vector("K", b)
    handle.fill_vector("X", 0.0)
    res = handle.solve(max_iterations=20000, tolerance=1e-9, precision=cg.PRECISION_MIXED)
    x = handle.get_vector("X")
    assert res["converged"] == 1
    tr = np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)
    assert tr <= 1e-9
    _, it_o, outer_o, _ = O.mixed_ir_solve(A.ptr, A.index, A.value, Cd, b)
    assert abs(res["iterations"] - it_o) <= 0.05 * it_o + 2
    _check_inner_form(handle, A, _IRREGULAR[case])


def test_band_returns_after_an_asymmetric_refresh(handle):
    """A value refresh that fails the band's symmetry check moves the inner
    SpMV to SELL-U; a later refresh with symmetric values on the same pattern
    brings the band back (the planned offsets are kept)."""
    A = G.diffusion3d(13, stencil=7, seed=14)
    b, _ = G.rhs_for(A, seed=15)
    handle.upload_crs(A.ptr, A.index, A.value)
    forms = []
    for vals in (A.value, _asymmetric(A).value, A.value * 1.5):
        handle.update_crs_values(vals)
        M = G.Crs(A.N, A.ptr, A.index, vals)
        handle.upload_jacobi(1.0 / M.diagonal())
        handle.set_vector("K", b)
        handle.fill_vector("X", 0.0)
        res = handle.solve(max_iterations=20000, tolerance=1e-9,
                           precision=cg.PRECISION_MIXED)
        x = handle.get_vector("X")
        assert res["converged"] == 1
        assert np.linalg.norm(b - M.matvec(x)) / np.linalg.norm(b) <= 1e-9
        forms.append(handle.inner_band())
    assert forms[0] == _expected_band(A)
    assert forms[1] == []
    assert forms[2] == _expected_band(A)


def _strided_band(N, seed):
    """SPD matrix with offsets 0, +-2, +-9: a band form whose d_1 is not 1
    (no lane shuffles)."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [np.arange(N)], [np.arange(N)], [np.full(N, 5.0)]
    for off in (2, 9):
        r = np.arange(N - off)
        w = rng.uniform(0.2, 1.0, N - off)
        rows += [r, r + off]
        cols += [r + off, r]
        vals += [-w, -w]
    return G.crs_from_unsorted(N, np.concatenate(rows), np.concatenate(cols),
                               np.concatenate(vals))


@pytest.mark.parametrize("case", ["diffusion7_24", "diffusion7_37x23x11", "poisson2d_65",
                                  "tridiagonal", "strided"])
def test_band_loops_agree(handle, case):
    """The mixed solve on band forms (the 7-point grids, the 2-D 5-point
    form, a tridiagonal matrix and offsets 2 and 9) in every loop mode:
    per-iteration kernels in a graph, in chunks and one launch at a time,
    and the fused and split persistent inner solves. Every mode reaches the
    FP64 tolerance with inner iteration counts within 2 % and the same
    solution."""
    A = {"diffusion7_24": lambda: G.diffusion3d(24, 7, sigma=1.0, corr_len=8.0, seed=31),
         "diffusion7_37x23x11": lambda: _grid7(37, 23, 11, seed=37),
         "poisson2d_65": lambda: G.poisson2d(65),
         "tridiagonal": lambda: _tridiagonal(20001, seed=32),
         "strided": lambda: _strided_band(30011, seed=33)}[case]()
    b, _ = G.rhs_for(A, seed=34)
    handle.upload_crs(A.ptr, A.index, A.value)
    handle.upload_jacobi(1.0 / A.diagonal())
    handle.set_vector("K", b)
    out = {}
    for loop in (cg.LOOP_GRAPH, cg.LOOP_CHUNKED, cg.LOOP_KERNELS, cg.LOOP_PERSISTENT,
                 cg.LOOP_PERSISTENT_SPLIT):
        handle.fill_vector("X", 0.0)
        r = handle.solve(max_iterations=50000, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                         loop=loop)
        x = handle.get_vector("X")
        assert r["converged"] == 1 and r["fell_back"] == 0, (loop, r)
        assert np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b) <= 1e-9
        out[loop] = (r, x)
    assert handle.inner_band() == _expected_band(A)
    rg, xg = out[cg.LOOP_GRAPH]
    for loop in (cg.LOOP_CHUNKED, cg.LOOP_KERNELS, cg.LOOP_PERSISTENT,
                 cg.LOOP_PERSISTENT_SPLIT):
        rl, xl = out[loop]
        assert abs(rl["iterations"] - rg["iterations"]) <= 0.02 * rg["iterations"] + 2
        assert rel(xl, xg) <= 1e-6


def _grid7(nx, ny, nz, seed):
    """SPD 7-point matrix on an nx x ny x nz grid (x fastest)."""
    rng = np.random.default_rng(seed)
    N = nx * ny * nz
    idx = np.arange(N).reshape(nz, ny, nx)
    rows, cols, vals = [np.arange(N)], [np.arange(N)], [np.full(N, 7.0)]
    for axis in (2, 1, 0):
        a_ = idx.take(range(idx.shape[axis] - 1), axis=axis).ravel()
        b_ = idx.take(range(1, idx.shape[axis]), axis=axis).ravel()
        w = rng.uniform(0.2, 1.0, len(a_))
        rows += [a_, b_]
        cols += [b_, a_]
        vals += [-w, -w]
    return G.crs_from_unsorted(N, np.concatenate(rows), np.concatenate(cols),
                               np.concatenate(vals))


def test_learned_loops_agree(handle):
    """The learned path on the 7-point band in every loop mode (the graph
    of per-iteration kernels, chunks, single launches, and the fused and
    split persistent inner solves): the same iterations within 2 % and
    solutions."""
    from cgxx_b200 import learned as LRN
    A = _grid7(41, 19, 13, seed=35)
    b, _ = G.rhs_for(A, seed=36)
    handle.upload_crs(A.ptr, A.index, A.value)
    handle.upload_jacobi(1.0 / A.diagonal())
    handle.set_vector("K", b)
    handle.learned_setup()
    net = cg.Gnn(0, LRN.load_weights(LRN.DEFAULT_WEIGHTS)[0])
    handle.learned_factor(net, 1e-4)
    net.close()
    out = {}
    for loop in (cg.LOOP_GRAPH, cg.LOOP_CHUNKED, cg.LOOP_KERNELS, cg.LOOP_PERSISTENT,
                 cg.LOOP_PERSISTENT_SPLIT):
        handle.fill_vector("X", 0.0)
        r = handle.solve(max_iterations=20000, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                         preconditioner=cg.PRECOND_LEARNED, loop=loop)
        x = handle.get_vector("X")
        assert r["converged"] == 1 and r["fell_back"] == 0, (loop, r)
        assert np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b) <= 1e-9
        out[loop] = (r["iterations"], x)
    ig, xg = out[cg.LOOP_GRAPH]
    for loop in (cg.LOOP_CHUNKED, cg.LOOP_KERNELS, cg.LOOP_PERSISTENT,
                 cg.LOOP_PERSISTENT_SPLIT):
        il, xl = out[loop]
        assert abs(il - ig) <= 0.02 * ig + 2, (loop, il, ig)
        assert rel(xl, xg) <= 1e-6, loop


@pytest.mark.parametrize("learned", [False, True])
def test_sell_loops_agree(handle, learned):
    """The mixed solves on the SELL-U inner form (27-point matrix: no band
    form, every slice uniform) in every loop mode: the default and the split
    persistent mode run the persistent SELL-U inner solve (inner_form 3), the
    others the graph of per-iteration kernels; the same iterations within
    2 % and the same solution."""
    from cgxx_b200 import learned as LRN
    A = G.diffusion3d(22, stencil=27, sigma=1.0, corr_len=4.0, seed=41)
    b, _ = G.rhs_for(A, seed=42)
    handle.upload_crs(A.ptr, A.index, A.value)
    handle.upload_jacobi(1.0 / A.diagonal())
    handle.set_vector("K", b)
    pc = cg.PRECOND_JACOBI
    if learned:
        handle.learned_setup()
        net = cg.Gnn(0, LRN.load_weights(LRN.DEFAULT_WEIGHTS)[0])
        handle.learned_factor(net, 1e-4)
        net.close()
        pc = cg.PRECOND_LEARNED
    out = {}
    for loop in (cg.LOOP_GRAPH, cg.LOOP_CHUNKED, cg.LOOP_KERNELS, cg.LOOP_PERSISTENT,
                 cg.LOOP_PERSISTENT_SPLIT):
        handle.fill_vector("X", 0.0)
        r = handle.solve(max_iterations=20000, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                         preconditioner=pc, loop=loop)
        x = handle.get_vector("X")
        assert r["converged"] == 1 and r["fell_back"] == 0, (loop, r)
        assert np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b) <= 1e-9
        out[loop] = (r, x)
    assert not handle.inner_band()
    assert out[cg.LOOP_GRAPH][0]["inner_form"] == 3
    assert out[cg.LOOP_PERSISTENT_SPLIT][0]["inner_form"] == 3
    assert out[cg.LOOP_PERSISTENT][0]["inner_form"] == 0  # no band: the graph
    assert out[cg.LOOP_GRAPH][0]["inner_launches"] == out[cg.LOOP_GRAPH][0]["outer_iterations"]
    rk, xk = out[cg.LOOP_KERNELS]
    for loop in (cg.LOOP_GRAPH, cg.LOOP_CHUNKED, cg.LOOP_PERSISTENT, cg.LOOP_PERSISTENT_SPLIT):
        rl, xl = out[loop]
        assert abs(rl["iterations"] - rk["iterations"]) <= 0.02 * rk["iterations"] + 2, loop
        assert rel(xl, xk) <= 1e-6, loop


def test_time_spmv_measures_the_fused_product(handle):
    """cgx_time_spmv times the solver's own SpMV (FP64 and the FP32 inner
    one) back to back, and a solve afterwards is unaffected."""
    A = G.diffusion3d(24, stencil=7, seed=8)
    b, _ = G.rhs_for(A, seed=8)
    handle.upload_crs(A.ptr, A.index, A.value)
    handle.upload_jacobi(1.0 / A.diagonal())
    handle.set_vector("K", b)
    handle.fill_vector("X", 0.0)
    r1 = handle.solve(max_iterations=5000, tolerance=1e-9)
    x1 = handle.get_vector("X")
    handle.fill_vector("X", 0.0)
    handle.solve(max_iterations=5000, tolerance=1e-9, precision=cg.PRECISION_MIXED)
    t64 = handle.time_spmv(cg.PRECISION_FP64, reps=5)
    t32 = handle.time_spmv(cg.PRECISION_MIXED, reps=5)
    assert 0 < t32 < 1e4 and 0 < t64 < 1e4
    # q = A p of the last FP64 product, checked against the CPU.
    p = handle.get_vector("P")
    assert np.allclose(handle.get_vector("Q"), A.matvec(p), rtol=1e-12, atol=0)
    handle.fill_vector("X", 0.0)
    r2 = handle.solve(max_iterations=5000, tolerance=1e-9)
    assert r2["iterations"] == r1["iterations"]
    assert np.array_equal(handle.get_vector("X"), x1)
    with pytest.raises(cg.CgxError):
        handle.time_spmv(cg.PRECISION_FP64, reps=0)


def test_reused_blocks_give_fresh_results():
    """A handle keeps the device blocks of a replaced matrix and hands them
    out again (uploads of the same size then allocate nothing). Whatever a
    reused block held before must not reach a result: a sequence of uploads
    of different sizes and formats, with the mixed and learned solves that
    build further buffers, gives exactly what a fresh handle gives for each
    matrix."""
    mats = [G.diffusion3d(14, stencil=7, seed=11), random_crs(3001, max_len=12, seed=12, spd=True),
            G.diffusion3d(14, stencil=7, seed=13), G.diffusion3d(9, stencil=27, seed=14)]

    def run(h, A, fmt, precision):
        b, _ = G.rhs_for(A, seed=A.N)
        if fmt == "ELL":
            m, length, index, data = G.to_ell(A)
            h.upload_ell(A.N, A.nz, m, length, index, data)
        else:
            h.upload_crs(A.ptr, A.index, A.value)
        h.upload_jacobi(1.0 / A.diagonal())
        h.set_vector("K", b)
        h.fill_vector("X", 0.0)
        r = h.solve(max_iterations=5000, tolerance=1e-9, precision=precision)
        return r["iterations"], h.get_vector("X")

    plan = [(0, "CRS", cg.PRECISION_MIXED), (1, "CRS", cg.PRECISION_MIXED),
            (2, "ELL", cg.PRECISION_FP64), (0, "CRS", cg.PRECISION_FP64),
            (3, "CRS", cg.PRECISION_MIXED), (2, "CRS", cg.PRECISION_MIXED)]
    from cgxx_b200 import learned as LRN

    def run_learned(h, A):
        b, _ = G.rhs_for(A, seed=A.N)
        h.upload_crs(A.ptr, A.index, A.value)
        h.upload_jacobi(1.0 / A.diagonal())
        h.set_vector("K", b)
        h.learned_setup()
        net = cg.Gnn(0, LRN.init_params(0))
        h.learned_factor(net, 1e-4)
        net.close()
        h.fill_vector("X", 0.0)
        r = h.solve(max_iterations=5000, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                    preconditioner=cg.PRECOND_LEARNED)
        return r["iterations"], h.get_vector("X")

    with cg.Handle(0) as h:
        for k, fmt, prec in plan:
            it, x = run(h, mats[k], fmt, prec)
            with cg.Handle(0) as fresh:
                it0, x0 = run(fresh, mats[k], fmt, prec)
            assert it == it0 and np.array_equal(x, x0), (k, fmt, prec)
        for k in (0, 1, 0):
            it, x = run_learned(h, mats[k])
            with cg.Handle(0) as fresh:
                it0, x0 = run_learned(fresh, mats[k])
            assert it == it0 and np.array_equal(x, x0), ("learned", k)


def test_mixed_and_learned_accept_every_format():
    """The mixed and learned paths and the device Jacobi set-up read the row
    layout: COO holds it from the upload (grouped by row), ELL builds it on
    first use. The COO form as the reference's reader produces it (lower
    triangle, then the mirrored entries) and the ELL form solve as the CRS
    form does: the same iteration counts and solutions within 1e-10 (only
    the order of entries inside a row may differ)."""
    from cgxx_b200 import learned as LRN
    A = G.diffusion3d(16, stencil=7, seed=21)
    b, xs = G.rhs_for(A, seed=22)
    I, J, V = G.symmetric_file_coo(A)
    out = {}
    for fmt in ("CRS", "COO", "ELL"):
        with cg.Handle(0) as h:
            if fmt == "CRS":
                h.upload_crs(A.ptr, A.index, A.value)
            elif fmt == "COO":
                h.upload_coo(A.N, I, J, V)
            else:
                m, length, index, data = G.to_ell(A)
                h.upload_ell(A.N, A.nz, m, length, index, data)
            h.jacobi_from_matrix()
            h.set_vector("K", b)
            h.fill_vector("X", 0.0)
            rm = h.solve(max_iterations=5000, tolerance=1e-9, precision=cg.PRECISION_MIXED)
            xm = h.get_vector("X")
            h.learned_setup()
            net = cg.Gnn(0, LRN.load_weights(LRN.DEFAULT_WEIGHTS)[0])
            h.learned_factor(net, 1e-4)
            net.close()
            h.fill_vector("X", 0.0)
            rl = h.solve(max_iterations=5000, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                         preconditioner=cg.PRECOND_LEARNED)
            out[fmt] = (rm["iterations"], xm, rl["iterations"], h.get_vector("X"), h.inner_band())
    im, xm, il, xl, band = out["CRS"]
    assert band == [0, 1, 16, 256] and il < 0.75 * im
    assert rel(xm, xs) <= 1e-6 and rel(xl, xs) <= 1e-6
    for fmt in ("COO", "ELL"):
        im2, xm2, il2, xl2, band2 = out[fmt]
        assert band2 == band and im2 == im and il2 == il, fmt
        assert rel(xm2, xm) <= 1e-10 and rel(xl2, xl) <= 1e-10, fmt


@pytest.mark.parametrize("case", ["graph", "stencil27", "band7"])
def test_value_refresh_keeps_graphs_and_results(case):
    """A value refresh of the same pattern keeps the captured inner-solve
    graphs (they hold pointers and layout choices, not values). The mixed
    and learned solves after each refresh give exactly what a fresh handle
    gives for those values: on the graph of per-iteration kernels (FP32 CRS
    and per-row SELL-U), on the persistent SELL-U form and on the band, and
    in the chunked loop's captured graph on each."""
    from cgxx_b200 import learned as LRN
    if case == "graph":
        # the same points with new weights: same pattern, symmetric scaling
        base = G.geometric_graph(6000, seed=31)
        rng = np.random.default_rng(5)
        rows = np.repeat(np.arange(base.N), np.diff(base.ptr))
        f = rng.uniform(0.5, 2.0, base.N)
        v = base.value * np.sqrt(f[rows] * f[base.index])
        mats = [base, G.Crs(base.N, base.ptr, base.index, v)]
    elif case == "stencil27":
        mats = [G.diffusion3d(12, stencil=27, seed=s) for s in (33, 34)]
    else:
        mats = [G.diffusion3d(13, stencil=7, seed=s) for s in (35, 36)]
    assert np.array_equal(mats[0].index, mats[1].index)
    net = cg.Gnn(0, LRN.init_params(2))

    def solves(h, A):
        b, _ = G.rhs_for(A, seed=7)
        h.upload_jacobi(1.0 / A.diagonal())
        h.set_vector("K", b)
        out = []
        for pc in (cg.PRECOND_JACOBI, cg.PRECOND_LEARNED):
            if pc == cg.PRECOND_LEARNED:
                h.learned_setup()
                h.learned_factor(net, 1e-4)
            # the default loop, and the chunked graph (captured on every form)
            for loop in (cg.LOOP_GRAPH, cg.LOOP_CHUNKED):
                h.fill_vector("X", 0.0)
                r = h.solve(max_iterations=5000, tolerance=1e-9,
                            precision=cg.PRECISION_MIXED, preconditioner=pc, loop=loop)
                out.append((r["iterations"], r["inner_form"], h.get_vector("X")))
        return out

    with cg.Handle(0) as h:
        h.upload_crs(mats[0].ptr, mats[0].index, mats[0].value)
        for k in (0, 1, 0, 1):
            h.update_crs_values(mats[k].value)
            got = solves(h, mats[k])
            with cg.Handle(0) as fresh:
                fresh.upload_crs(mats[k].ptr, mats[k].index, mats[k].value)
                ref = solves(fresh, mats[k])
            for (it, form, x), (it0, form0, x0) in zip(got, ref):
                assert it == it0 and form == form0 and np.array_equal(x, x0), (case, k)
    net.close()
