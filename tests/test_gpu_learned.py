"""The learned preconditioner on the GPU against its CPU oracle
(oracle/gnn_oracle.py; the reference has no counterpart, so parity is pinned
to that restatement).

Tolerances: the network runs with BF16 activations on the tensor cores; the
oracle rounds at the same points but accumulates in a different order, so a
value that lands near a BF16 rounding boundary can round the other way.
Factor values: max |G - G_oracle| <= 2e-2 max |G_oracle|. Gradient:
||g - g_oracle|| <= 3e-2 ||g_oracle||, loss within 1e-3 relative.
"""
import numpy as np
import pytest

import cgxx_b200 as cg
from cgxx_b200 import generators as G
from conftest import random_crs
from oracle import gnn_oracle as GO

pytestmark = pytest.mark.gpu


def _setup(A):
    h = cg.Handle(0)
    h.upload_crs(A.ptr, A.index, A.value)
    h.upload_jacobi(1.0 / A.diagonal())
    h.learned_setup()
    return h


def _oracle_factor_in_g_order(A, params, rows, cols):
    g = GO.Graph(A.ptr, A.index, A.value)
    gd, go = GO.factor(g, params)
    out = np.empty(len(rows), np.float32)
    k = 0
    for e, (r, c) in enumerate(zip(rows, cols)):
        if r == c:
            out[e] = gd[r]
        else:
            out[e] = go[k]
            k += 1
    assert k == len(go)
    return out


def _params(seed, scale=1.0):
    p = GO.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    # Move away from the near-zero head so every term contributes.
    return (p + scale * 0.05 * rng.standard_normal(p.size)).astype(np.float32)


MATRICES = [
    ("diffusion7_10", lambda: G.diffusion3d(10, 7, sigma=1.5, corr_len=4.0, seed=1)),
    ("diffusion27_6", lambda: G.diffusion3d(6, 27, sigma=1.0, corr_len=3.0, seed=2)),
    ("random_spd_500", lambda: random_crs(500, 0, 30, seed=7, spd=True)),
]


@pytest.mark.parametrize("name,make", MATRICES, ids=[m[0] for m in MATRICES])
def test_factor_matches_oracle(name, make):
    A = make()
    h = _setup(A)
    params = _params(3)
    net = cg.Gnn(0, params)
    h.learned_factor(net, 0.0)
    ghat, rows, cols = h.learned_get_factor()
    ref = _oracle_factor_in_g_order(A, params, rows, cols)
    assert np.all(rows >= cols)
    assert np.max(np.abs(ghat - ref)) <= 2e-2 * np.max(np.abs(ref))
    assert np.median(np.abs(ghat - ref)) <= 1e-3 * np.max(np.abs(ref))
    h.close()
    net.close()


@pytest.mark.parametrize("name,make", MATRICES + [
    ("diffusion7_13", lambda: G.diffusion3d(13, 7, sigma=1.0, corr_len=4.0, seed=5)),
    ("poisson2d_37", lambda: G.poisson2d(37)),
    # per-row SELL-U slices
    ("graph_4500", lambda: G.geometric_graph(4500, seed=5)),
], ids=[m[0] for m in MATRICES] + ["diffusion7_13", "poisson2d_37", "graph_4500"])
def test_apply_matches_factor(name, make):
    """z = G (G^T r) + eps C r from the device (BF16 factor values, the band
    copy of G for the 7- and 5-point stencils, SELL-U or FP32 CRS otherwise)
    against the same product in FP64 from the factor the device reports:
    within 1.6e-2 of (|G| |G|^T |r|)_i + eps C_i |r_i| per row (two BF16
    roundings of the factor values, 2^-9 each, and FP32 sums)."""
    A = make()
    h = _setup(A)
    net = cg.Gnn(0, _params(3))
    eps = 1e-3
    h.learned_factor(net, eps)
    ghat, rows, cols = h.learned_get_factor()
    dis = 1.0 / np.sqrt(A.diagonal())
    gv = dis[rows] * ghat.astype(np.float64)

    def g_times(v, x):  # G x
        return np.bincount(rows, weights=v * x[cols], minlength=A.N)

    def gt_times(v, x):  # G^T x
        return np.bincount(cols, weights=v * x[rows], minlength=A.N)

    C = 1.0 / A.diagonal()
    rng = np.random.default_rng(4)
    for _ in range(2):
        r = rng.standard_normal(A.N).astype(np.float32)
        z = h.learned_apply(r)
        rd = r.astype(np.float64)
        ref = g_times(gv, gt_times(gv, rd)) + eps * C * rd
        ga = np.abs(gv)
        bound = 1.6e-2 * g_times(ga, gt_times(ga, np.abs(rd))) + 1e-6 * eps * C * np.abs(rd)
        assert np.all(np.abs(z - ref) <= bound + 1e-30)
    h.close()
    net.close()


@pytest.mark.parametrize("name,make", MATRICES, ids=[m[0] for m in MATRICES])
def test_gradient_matches_oracle(name, make):
    A = make()
    h = _setup(A)
    params = _params(5)
    net = cg.Gnn(0, params)
    V = np.random.default_rng(9).choice([-1.0, 1.0], size=(A.N, 8)).astype(np.float32)
    loss, grad = net.loss_grad(h, probes=V)
    lo, go = GO.loss_and_grad(GO.Graph(A.ptr, A.index, A.value), params, V)
    assert abs(loss - lo) <= 1e-3 * abs(lo)
    assert np.linalg.norm(grad - go) <= 3e-2 * np.linalg.norm(go)
    # Each parameter block separately, so one block cannot hide in another.
    o = 0
    for pname, shp in GO.param_shapes():
        n = int(np.prod(shp))
        gb, rb = grad[o:o + n], go[o:o + n]
        if np.linalg.norm(rb) > 1e-6 * np.linalg.norm(go):
            assert np.linalg.norm(gb - rb) <= 5e-2 * np.linalg.norm(rb), pname
        o += n
    h.close()
    net.close()


def test_gradient_is_deterministic():
    A = G.diffusion3d(12, 7, seed=4)
    h = _setup(A)
    net = cg.Gnn(0, _params(1))
    l1, g1 = net.loss_grad(h, seed=77)
    l2, g2 = net.loss_grad(h, seed=77)
    assert l1 == l2 and np.array_equal(g1, g2)
    h.close()
    net.close()


def test_probe_recipe_matches_oracle():
    """Probes made on the device (Rademacher hash, then smoothed columns)
    equal the oracle's restatement: the loss and gradient from the device's
    own probes match those from the oracle's probes passed in explicitly."""
    A = G.diffusion3d(12, 7, seed=4)
    h = _setup(A)
    net = cg.Gnn(0, _params(2))
    gr = GO.Graph(A.ptr, A.index, A.value)
    seed = 12345
    l0, g0 = net.loss_grad(h, seed=seed)
    l1, g1 = net.loss_grad(h, probes=GO.rademacher(A.N, seed))
    assert l0 == l1 and np.array_equal(g0, g1)
    net.set_probes(3, 4, 3.0)
    l2, g2 = net.loss_grad(h, seed=seed)
    V = GO.smooth_probes(gr, GO.rademacher(A.N, seed), 3, 4, 3.0)
    l3, g3 = net.loss_grad(h, probes=V)
    assert abs(l2 - l3) <= 1e-4 * abs(l3)
    assert np.linalg.norm(g2 - g3) <= 1e-3 * np.linalg.norm(g3)
    assert abs(l2 - l0) > 1e-3 * abs(l0)  # the recipe changed the probes
    h.close()
    net.close()


def test_residual_probes_match_oracle():
    """Residual snapshots of the solver's own iterates as probe columns: the
    device's capture (D^-1/2 (k - A x), unit RMS) equals the oracle's, so the
    loss from the recipe matches the loss from explicit probes."""
    A = G.diffusion3d(12, 7, seed=6)
    h = _setup(A)
    b, _ = G.rhs_for(A, seed=3)
    h.upload_jacobi(1.0 / A.diagonal())
    h.set_vector("K", b)
    h.fill_vector("X", 0.0)
    gr = GO.Graph(A.ptr, A.index, A.value)
    cols = []
    for c, its in ((6, 3), (7, 7)):
        h.solve(max_iterations=its, tolerance=1e-30)
        h.learned_capture_residual(c)
        x = h.get_vector("X")
        cols.append(GO.residual_probe(gr, b - A.matvec(x)))
    net = cg.Gnn(0, _params(3))
    net.set_probes(residual_cols=2)
    seed = 99
    l_dev, g_dev = net.loss_grad(h, seed=seed)
    V = GO.rademacher(A.N, seed)
    V[:, 6], V[:, 7] = cols[0], cols[1]
    l_ref, g_ref = net.loss_grad(h, probes=V)
    assert abs(l_dev - l_ref) <= 1e-5 * abs(l_ref)
    assert np.linalg.norm(g_dev - g_ref) <= 1e-4 * np.linalg.norm(g_ref)
    # New values drop the snapshots: the recipe then refuses to run.
    h.update_crs_values(A.value * 2.0)
    h.learned_setup()
    with pytest.raises(cg.CgxError):
        net.loss_grad(h, seed=seed)
    h.close()
    net.close()


def test_training_lowers_the_loss():
    fam = G.Diffusion7Family(12)
    rng = np.random.default_rng(0)
    mats = [fam.values(G.diffusion_field(12, rng.uniform(0.5, 2), rng.uniform(4, 16), 50 + k))
            for k in range(4)]
    h = cg.Handle(0)
    h.upload_crs(fam.ptr, fam.index, mats[0])
    h.learned_setup()
    net = cg.Gnn(0, GO.init_params(0))

    def mean_loss():
        tot = 0.0
        for v in mats:
            h.update_crs_values(v)
            h.learned_setup()
            tot += net.loss_grad(h, seed=12345)[0]
        return tot / len(mats)

    before = mean_loss()
    for step in range(60):
        h.update_crs_values(mats[step % len(mats)])
        h.learned_setup()
        net.train_step(h, seed=1000 + step, lr=3e-3)
    after = mean_loss()
    assert after < before
    h.close()
    net.close()


def _solve(h, precond, b):
    h.set_vector("K", b)
    h.fill_vector("X", 0.0)
    return h.solve(max_iterations=20000, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                   preconditioner=precond)


def _shipped(name):
    from cgxx_b200 import learned as LRN
    import os
    params, _ = LRN.load_weights(os.path.join(os.path.dirname(LRN.DEFAULT_WEIGHTS), name))
    return params


@pytest.mark.parametrize("loop", [cg.LOOP_GRAPH, cg.LOOP_CHUNKED, cg.LOOP_KERNELS])
def test_learned_solve_converges_with_fewer_iterations(loop):
    """The shipped weights on a field they were not trained on: about half
    the inner iterations of Jacobi, in every loop mode (graph and chunked
    run the fused band iteration two iterations per body or launch)."""
    A = G.diffusion3d(24, 7, sigma=1.0, corr_len=8.0, seed=11)
    b, xs = G.rhs_for(A, seed=3)
    h = _setup(A)
    net = cg.Gnn(0, _shipped("diffusion7.gnn"))
    h.learned_factor(net, 1e-4)
    h.set_vector("K", b)
    rj = h.solve(max_iterations=20000, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                 preconditioner=cg.PRECOND_JACOBI, loop=loop)
    h.fill_vector("X", 0.0)
    rl = h.solve(max_iterations=20000, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                 preconditioner=cg.PRECOND_LEARNED, loop=loop)
    x = h.get_vector("X")
    assert rl["converged"] == 1 and rl["fell_back"] == 0
    assert np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b) <= 1e-9
    assert rl["iterations"] < 0.75 * rj["iterations"], (rl["iterations"], rj["iterations"])
    h.close()
    net.close()


def test_learned_solve_on_geometric_graph():
    """The irregular family: a random geometric graph Laplacian (mean degree
    12, exp(-d/r) weights, 1e-3 I shift). Its slices are not uniform, so the
    FP32 SpMV runs on FP32 CRS and the factor applies take SELL-U's per-row
    offsets; the learned factor still halves the inner iterations of Jacobi."""
    A = G.geometric_graph(20000, seed=3)
    b, _ = G.rhs_for(A, seed=4)
    h = _setup(A)
    net = cg.Gnn(0, _shipped("graph12.gnn"))
    h.learned_factor(net, 1e-4)
    h.set_vector("K", b)
    h.fill_vector("X", 0.0)
    rj = h.solve(max_iterations=20000, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                 preconditioner=cg.PRECOND_JACOBI)
    xj = h.get_vector("X")
    slots, uniform, slices = h.inner_layout()
    assert slots == 0
    h.fill_vector("X", 0.0)
    rl = h.solve(max_iterations=20000, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                 preconditioner=cg.PRECOND_LEARNED)
    x = h.get_vector("X")
    for r, xv in ((rj, xj), (rl, x)):
        assert r["converged"] == 1
        assert np.linalg.norm(b - A.matvec(xv)) / np.linalg.norm(b) <= 1e-9
    assert rl["fell_back"] == 0
    assert rl["iterations"] < 0.75 * rj["iterations"], (rl["iterations"], rj["iterations"])
    h.close()
    net.close()


def test_learned_setup_rejects_unsymmetric_pattern():
    N = 50
    rows = np.concatenate([np.arange(N), np.arange(1, N)])
    cols = np.concatenate([np.arange(N), np.arange(0, N - 1)])  # lower only
    A = G.crs_from_unsorted(N, rows, cols, np.concatenate([np.full(N, 2.0), -np.ones(N - 1)]))
    h = cg.Handle(0)
    h.upload_crs(A.ptr, A.index, A.value)
    with pytest.raises(cg.CgxError) as e:
        h.learned_setup()
    assert "symmetric" in e.value.message
    h.close()


def test_eps_change_reaches_the_solve():
    """eps is an argument of the kernels that the cached inner-solve graph
    holds; a new eps must reach the next solve. The solve after
    learned_factor(eps2) equals a fresh handle's solve with eps2, and differs
    from the one with eps1 (eps2 large enough to change the iterates)."""
    A = G.diffusion3d(14, 7, sigma=1.0, corr_len=4.0, seed=9)
    b, _ = G.rhs_for(A, seed=10)
    net = cg.Gnn(0, GO.init_params(0))

    def solve(h, eps):
        h.learned_factor(net, eps)
        h.set_vector("K", b)
        h.fill_vector("X", 0.0)
        r = h.solve(max_iterations=5000, tolerance=1e-9, precision=cg.PRECISION_MIXED,
                    preconditioner=cg.PRECOND_LEARNED)
        return r["iterations"], h.get_vector("X")

    h = _setup(A)
    it1, x1 = solve(h, 1e-4)
    it2, x2 = solve(h, 1.0)
    h.close()
    fresh = _setup(A)
    it2f, x2f = solve(fresh, 1.0)
    fresh.close()
    net.close()
    assert it2 == it2f and np.array_equal(x2, x2f)
    assert it1 != it2 or not np.array_equal(x1, x2)


def test_training_gains_over_the_untrained_network():
    """What training adds: on 8 held-out 96^3 fields of the training family
    (sigma ~ U[0.5, 2], correlation length ~ U[4, 16], seeds outside the
    training set), the shipped weights need at least 10 % fewer inner
    iterations than the same network untrained (init_params(0)), whose
    factor is close to Jacobi. Both solves reach the FP64 1e-9 residual."""
    from cgxx_b200 import learned as LRN
    fam = G.Diffusion7Family(96)
    specs = LRN.family_specs(8, 900000, 2000)  # the held-out family seeds
    trained = cg.Gnn(0, _shipped("diffusion7.gnn"))
    untrained = cg.Gnn(0, GO.init_params(0))
    h = cg.Handle(0)
    h.upload_crs(fam.ptr, fam.index, fam.values(np.ones(fam.N)))
    its = {"trained": [], "untrained": []}
    for k, (sigma, ell, seed) in enumerate(specs):
        v = fam.values(G.diffusion_field(96, sigma, ell, seed))
        A = G.Crs(fam.N, fam.ptr, fam.index, v)
        b, _ = G.rhs_for(A, seed=k)
        h.update_crs_values(v)
        h.upload_jacobi(1.0 / A.diagonal())
        h.set_vector("K", b)
        h.learned_setup()
        for name, net in (("trained", trained), ("untrained", untrained)):
            h.learned_factor(net, 1e-4)
            h.fill_vector("X", 0.0)
            r = h.solve(max_iterations=20000, tolerance=1e-9,
                        precision=cg.PRECISION_MIXED, preconditioner=cg.PRECOND_LEARNED)
            assert r["converged"] == 1 and r["fell_back"] == 0, (name, r)
            its[name].append(r["iterations"])
    h.close()
    trained.close()
    untrained.close()
    t, u = np.median(its["trained"]), np.median(its["untrained"])
    assert t <= 0.9 * u, its
    assert all(a < b for a, b in zip(its["trained"], its["untrained"])), its


def test_learned_twice_as_fast_as_plain_on_heldout_fields():
    """The learned-preconditioner mixed solve against plain FP64 Jacobi-CG on
    8 held-out 96^3 fields of the training family (the default loop mode,
    shipped weights): the median over fields of plain time / (learned solve
    + set-up and inference of the factor) is at least 2, and every solve
    reaches the FP64 1e-9 residual without falling back."""
    from cgxx_b200 import learned as LRN
    fam = G.Diffusion7Family(96)
    specs = LRN.family_specs(8, 900000, 2000)
    net = cg.Gnn(0, _shipped("diffusion7.gnn"))
    h = cg.Handle(0)
    h.upload_crs(fam.ptr, fam.index, fam.values(np.ones(fam.N)))
    ratios = []
    for k, (sigma, ell, seed) in enumerate(specs):
        v = fam.values(G.diffusion_field(96, sigma, ell, seed))
        A = G.Crs(fam.N, fam.ptr, fam.index, v)
        b, _ = G.rhs_for(A, seed=k)
        h.update_crs_values(v)
        h.upload_jacobi(1.0 / A.diagonal())
        LRN.solve_pair(h, fam.ptr, fam.index, v, b, True, net, 1e-4)  # warm-up
        r = LRN.solve_pair(h, fam.ptr, fam.index, v, b, True, net, 1e-4)
        for key in ("learned_mixed", "plain_fp64"):
            assert r[key]["converged"] and not r[key]["fell_back"], (k, key, r[key])
        ratios.append(r["plain_fp64"]["ms"] / (r["learned_mixed"]["ms"] + r["factor_ms"]))
    h.close()
    net.close()
    assert np.median(ratios) >= 2.0, ratios
