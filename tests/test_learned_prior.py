"""The learned factor against its bounds, on the CPU (oracle only).

The factor's head carries no hand-set prior: the untrained network (a head
near zero) emits Ghat close to I, so G G^T is close to D^-1 and PCG needs
nearly Jacobi's iteration count. Training has to learn the off-diagonal
values. The reference point for what training
can reach on the pattern of tril(A) is the factorized sparse approximate
inverse (FSAI) on that pattern, the factor that minimises the Kaporin
condition number for it; the shipped weights must reach its quality (and so
about half of Jacobi's iterations) on a field they were not trained on.
"""
import numpy as np
import scipy.sparse as sp

from cgxx_b200 import generators as G
from oracle import gnn_oracle as GO


def pcg_iterations(A, b, apply_m, tol=1e-9, maxit=5000):
    x = np.zeros_like(b)
    r = b.copy()
    z = apply_m(r)
    p = z.copy()
    rz = r @ z
    n0 = np.linalg.norm(r)
    for it in range(1, maxit + 1):
        q = A @ p
        a = rz / (p @ q)
        x += a * p
        r -= a * q
        if np.linalg.norm(r) / n0 <= tol:
            return it
        z = apply_m(r)
        rzn = r @ z
        p = z + (rzn / rz) * p
        rz = rzn
    return maxit


def fsai_lower(A):
    """FSAI with G lower on tril(A) and G G^T ~ A^-1: column j of G on
    S_j = {i >= j : A_ij != 0} solves A[S_j, S_j] g = e_1, scaled by
    1/sqrt(g_1)."""
    N = A.shape[0]
    L = sp.csc_matrix(sp.tril(A))
    Ad = A.tocsr()
    rows, cols, vals = [], [], []
    for j in range(N):
        S = np.sort(L.indices[L.indptr[j]:L.indptr[j + 1]])
        g = np.linalg.solve(Ad[S][:, S].toarray(), np.eye(len(S))[0])
        g /= np.sqrt(g[0])
        rows += list(S)
        cols += [j] * len(S)
        vals += list(g)
    return sp.csr_matrix((vals, (rows, cols)), shape=(N, N))


def _learned_iterations(A, S, b, d, params):
    g = GO.Graph(A.ptr, A.index, A.value)
    gdiag, goff = GO.factor(g, params)
    lr, lc = g.lr.numpy(), g.lc.numpy()
    Ghat = sp.csr_matrix((np.concatenate([gdiag, goff]).astype(np.float64),
                          (np.concatenate([np.arange(A.N), lr]),
                           np.concatenate([np.arange(A.N), lc]))), shape=(A.N, A.N))
    Gm = sp.diags(1.0 / np.sqrt(d)) @ Ghat
    GmT = Gm.T.tocsr()
    return pcg_iterations(S, b, lambda r: Gm @ (GmT @ r) + 1e-4 * r / d)


def _problem():
    A = G.diffusion3d(16, 7, sigma=1.0, corr_len=8.0, seed=1)
    S = sp.csr_matrix((A.value, A.index, A.ptr), shape=(A.N, A.N))
    b, _ = G.rhs_for(A, seed=1)
    return A, S, b, S.diagonal()


def test_untrained_factor_is_close_to_jacobi():
    A, S, b, d = _problem()
    it_jacobi = pcg_iterations(S, b, lambda r: r / d)
    it_untrained = _learned_iterations(A, S, b, d, GO.init_params(0))
    assert 0.8 * it_jacobi <= it_untrained <= it_jacobi + 2, (it_untrained, it_jacobi)


def test_shipped_weights_reach_fsai_quality():
    from cgxx_b200 import learned as LRN
    A, S, b, d = _problem()
    params, _ = LRN.load_weights(LRN.DEFAULT_WEIGHTS)
    it_jacobi = pcg_iterations(S, b, lambda r: r / d)
    it_trained = _learned_iterations(A, S, b, d, params)
    Gf = fsai_lower(S)
    GfT = Gf.T.tocsr()
    it_fsai = pcg_iterations(S, b, lambda r: Gf @ (GfT @ r))
    assert it_trained <= it_fsai + max(2, 0.05 * it_fsai), (it_trained, it_fsai)
    assert it_trained <= 0.6 * it_jacobi, (it_trained, it_jacobi)
