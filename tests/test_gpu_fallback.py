"""Failure handling of the mixed-precision paths: an FP32 refinement step that
breaks down or stalls is undone and the solve finishes with plain FP64
Jacobi-CG (the reference's algorithm, CG.cpp:284-385) from the restored x.

The failures are made on the host, in the matrix or the network parameters
handed to the library; no GPU fault is involved. Every solve here has a
bounded iteration budget, so a matrix on which no method converges ends with
a status, not a hang.
"""
import numpy as np
import pytest

import cgxx_b200 as cg
from cgxx_b200 import generators as G
from oracle import gnn_oracle as GO

pytestmark = pytest.mark.gpu


def _true_rel(A, b, x):
    return np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)


def _mixed(h, A, b, precond=cg.PRECOND_JACOBI, max_iter=20000, loop=cg.LOOP_GRAPH):
    h.set_vector("K", b)
    h.fill_vector("X", 0.0)
    r = h.solve(max_iterations=max_iter, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                preconditioner=precond, loop=loop)
    return r, h.get_vector("X")


@pytest.mark.parametrize("loop", [cg.LOOP_GRAPH, cg.LOOP_CHUNKED, cg.LOOP_KERNELS,
                                  cg.LOOP_PERSISTENT, cg.LOOP_PERSISTENT_SPLIT])
def test_fp32_overflow_falls_back_to_fp64(loop):
    """Every value of A is beyond the FP32 range (A scaled by 1e39; finite in
    FP64), so A's FP32 copy holds infinities and the inner solve cannot take a
    step. The Jacobi-mixed solve undoes that step and converges in FP64."""
    A0 = G.diffusion3d(16, 7, sigma=1.0, corr_len=4.0, seed=21)
    A = G.Crs(A0.N, A0.ptr, A0.index, A0.value * 1e39)
    b, _ = G.rhs_for(A, seed=22)
    with cg.Handle(0) as h:
        h.upload_crs(A.ptr, A.index, A.value)
        h.upload_jacobi(1.0 / A.diagonal())
        r, x = _mixed(h, A, b, loop=loop)
        assert r["fell_back"] == 1 and r["converged"] == 1, r
        assert _true_rel(A, b, x) <= 1e-9
        # The plain FP64 path on the same system for comparison: the fallback
        # starts from x = 0 (the undone step), so it repeats that solve.
        h.fill_vector("X", 0.0)
        rp = h.solve(max_iterations=20000, tolerance=0.5e-9)
        assert abs(r["iterations"] - rp["iterations"]) <= 5, (r, rp)


def test_fp32_overflow_learned_falls_back_to_fp64():
    """The same matrix on the learned path: the factor itself is finite (it
    is built from the Jacobi-scaled matrix), but A's FP32 copy is not."""
    A0 = G.diffusion3d(14, 7, sigma=1.0, corr_len=4.0, seed=23)
    A = G.Crs(A0.N, A0.ptr, A0.index, A0.value * 1e39)
    b, _ = G.rhs_for(A, seed=24)
    net = cg.Gnn(0, GO.init_params(0))
    with cg.Handle(0) as h:
        h.upload_crs(A.ptr, A.index, A.value)
        h.upload_jacobi(1.0 / A.diagonal())
        h.learned_setup()
        h.learned_factor(net, 1e-4)
        r, x = _mixed(h, A, b, precond=cg.PRECOND_LEARNED)
        assert r["fell_back"] == 1 and r["converged"] == 1, r
        assert _true_rel(A, b, x) <= 1e-9
    net.close()


def test_corrupted_network_falls_back_to_fp64():
    """A NaN network parameter makes every factor value NaN; the learned step
    is undone and plain FP64 Jacobi-CG finishes the solve."""
    A = G.diffusion3d(16, 7, seed=6)
    b, _ = G.rhs_for(A, seed=2)
    p = GO.init_params(0)
    p[GO.param_count() - 1] = np.nan  # the head bias -> NaN factor
    net = cg.Gnn(0, p)
    with cg.Handle(0) as h:
        h.upload_crs(A.ptr, A.index, A.value)
        h.upload_jacobi(1.0 / A.diagonal())
        h.learned_setup()
        h.learned_factor(net, 0.0)
        r, x = _mixed(h, A, b, precond=cg.PRECOND_LEARNED)
        assert r["fell_back"] == 1 and r["converged"] == 1, r
        assert _true_rel(A, b, x) <= 1e-9
        # x is the FP64 solve from x = 0: the same iterations as the plain path.
        h.fill_vector("X", 0.0)
        rp = h.solve(max_iterations=20000, tolerance=0.5e-9)
        assert abs(r["iterations"] - rp["iterations"]) <= 5, (r, rp)
    net.close()


def test_singular_inconsistent_system_ends_without_convergence():
    """The graph Laplacian of a 32x32 grid (rows sum to zero: singular) with a
    right-hand side that is mostly the constant null vector: no x solves it.
    The first refinement step cannot halve the residual, so the solve falls
    back to FP64, which runs out its budget. Documented outcome: status
    CGX_SUCCESS, converged = 0, fell_back = 1, and no hang."""
    n = 32
    P = G.poisson2d(n)
    rows = np.repeat(np.arange(P.N), np.diff(P.ptr))
    off = P.index != rows
    deg = np.bincount(rows[off], minlength=P.N).astype(np.float64)
    vals = np.where(off, P.value, deg[rows])
    A = G.Crs(P.N, P.ptr, P.index, vals)
    rng = np.random.default_rng(5)
    b = 1.0 + 1e-3 * A.matvec(rng.standard_normal(A.N))
    budget = 400
    with cg.Handle(0) as h:
        h.upload_crs(A.ptr, A.index, A.value)
        h.upload_jacobi(1.0 / A.diagonal())
        r, x = _mixed(h, A, b, max_iter=budget)
    assert r["converged"] == 0 and r["fell_back"] == 1, r
    assert r["iterations"] <= 2 * budget + 2
    assert _true_rel(A, b, x) > 1e-3  # the null-space part of b remains


def test_indefinite_matrix_ends_with_a_consistent_status():
    """A 2-D Poisson matrix shifted by -0.05 I has three negative eigenvalues
    (its diagonal stays positive, so Jacobi is defined). CG has no guarantee
    here. Documented outcome: the call returns with status CGX_SUCCESS and no
    hang; converged = 1 only if the FP64 true residual (checked here on the
    CPU) is within the tolerance, and otherwise the FP64 fallback has run or
    the budget is spent."""
    P = G.poisson2d(32)
    rows = np.repeat(np.arange(P.N), np.diff(P.ptr))
    A = G.Crs(P.N, P.ptr, P.index, np.where(P.index == rows, P.value - 0.05, P.value))
    b, _ = G.rhs_for(A, seed=31)
    budget = 3000
    with cg.Handle(0) as h:
        h.upload_crs(A.ptr, A.index, A.value)
        h.upload_jacobi(1.0 / A.diagonal())
        r, x = _mixed(h, A, b, max_iter=budget)
    tr = _true_rel(A, b, x) if np.all(np.isfinite(x)) else np.inf
    if r["converged"]:
        assert tr <= 1e-9, (r, tr)
    else:
        assert r["fell_back"] == 1 or r["iterations"] >= budget, r
    assert r["iterations"] <= 2 * budget + 2


@pytest.mark.parametrize("which,bit", [(0, 4), (1, 1)])
def test_bounded_wait_gives_up_and_the_handle_stays_usable(which, bit):
    """A wait that nothing can complete (0: the grid barrier of the
    persistent inner solves, whose target the arrivals never reach; 1: an
    mbarrier of the staged products that nobody arrives on) gives up after
    its limit: the kernel sets its error bit and returns, the call reports
    CGX_ERROR_DEVICE, and the same handle then solves correctly in every
    form that uses those waits."""
    A = G.diffusion3d(16, 7, sigma=1.0, corr_len=4.0, seed=31)
    b, _ = G.rhs_for(A, seed=32)
    with cg.Handle(0) as h:
        h.upload_crs(A.ptr, A.index, A.value)
        h.upload_jacobi(1.0 / A.diagonal())
        h.set_vector("K", b)
        status, bits = h.check_wait_timeout(which)
        assert status == 6 and bits & bit, (status, bits)
        for prec in (cg.PRECISION_FP64, cg.PRECISION_MIXED):
            h.fill_vector("X", 0.0)
            r = h.solve(max_iterations=5000, tolerance=1e-9, precision=prec)
            x = h.get_vector("X")
            assert r["converged"] == 1, r
            assert np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b) <= 1e-9
