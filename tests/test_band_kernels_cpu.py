"""The fused band row loops (cgxx_b200/csrc/fused.cuh) and the persistent
inner solve built on them (cgxx_b200/csrc/persist.cuh), restated in numpy
(no GPU).

One thread owns one row, grid-stride; row i's band values are the
row-major U[i] (diagonal and upper entries at offsets 0 < d1 < d2 < d3) and
its lower entries are read from the rows above, U[i - d_k][k]. The learned
factor's band copy holds Gb[i][k] = G(i, i - d_k). Neighbour indices are
clamped into [0, N - 1] before the load and the value masked afterwards.
This file restates that arithmetic row by row and checks, before the
kernels run on a device:

  - every load stays inside the buffer it addresses (U, Gb and the vectors
    hold N rows) on 3-D and 2-D grids, grids with fewer than four offsets,
    and a band that is not a grid's;
  - the products equal A p, G y and G^T r;
  - the fused persistent loop (ping-pong p and r, d one update behind and
    applied at the end, the learned and Jacobi phase orders) and the split
    one (the graph iteration's kernels as phases) give what the unfused PCG
    gives;
  - the partial-sum slots of the persistent phases are never rewritten
    before every CTA has read them.
"""
import numpy as np
import pytest

from cgxx_b200 import generators as G

f32 = np.float32


class Buf:
    """A device buffer with bounds-checked loads."""

    def __init__(self, values, size=None):
        values = np.asarray(values, np.float32)
        self.size = len(values) if size is None else size
        self.v = np.zeros((self.size,) + values.shape[1:], np.float32)
        self.v[:len(values)] = values

    def __getitem__(self, idx):
        idx = np.asarray(idx)
        if idx.size:
            assert idx.min() >= 0 and idx.max() < self.size, (idx.min(), idx.max(), self.size)
        return self.v[idx]


def fma(a, b, c):
    return (np.float64(a) * np.asarray(b, np.float64) + np.asarray(c, np.float64)).astype(f32)


def band_dir(offs, U, z, pold, d, al, be, N):
    """band_dir_rows: p = z + be p_old (own row and every neighbour the
    product reads), d += al p_old, q = A p."""
    i = np.arange(N)
    nmax = N - 1
    u = U[i]
    po0 = pold[i]
    p0 = fma(be, po0, z[i])
    s = fma(u[:, 0], p0, np.zeros(N, f32))
    for k in range(1, 4):
        ju = np.minimum(i + offs[k], nmax)
        s = fma(u[:, k], fma(be, pold[ju], z[ju]), s)
    for k in range(1, 4):
        j = i - offs[k]
        jc = np.maximum(j, 0)
        lv = np.where(j < 0, f32(0), U[jc][:, k])
        s = fma(lv, fma(be, pold[jc], z[jc]), s)
    dn = fma(al, po0, d[i])
    return p0, dn, s


def gband_res(offs, Gb, rold, q, na, N):
    """gband_res_rows: r = r_old + na q (own row and the rows below it that
    G^T reads), y = G^T r."""
    i = np.arange(N)
    r0 = fma(na, q[i], rold[i])
    s = fma(Gb[i][:, 0], r0, np.zeros(N, f32))
    for k in range(1, 4):
        j = i + offs[k]
        jc = np.minimum(j, N - 1)
        v = np.where(j < N, Gb[jc][:, k], f32(0))
        s = fma(v, fma(na, q[jc], rold[jc]), s)
    return r0, s


def gband_z(offs, Gb, y, r, C, eps, N):
    """gband_z_rows: z = G y + eps C r (the factor's band holds 0 where
    i - d_k < 0)."""
    i = np.arange(N)
    g = Gb[i]
    s = np.zeros(N, f32)
    for k in range(4):
        s = fma(g[:, k], y[np.maximum(i - offs[k], 0)], s)
    ri = r[i]
    return fma((f32(eps) * C[i]).astype(f32), ri, s)


def grid_matrix(nx, ny, nz, seed):
    """SPD 7-point (5-point when nz = 1) matrix on an nx x ny x nz grid."""
    rng = np.random.default_rng(seed)
    N = nx * ny * nz
    idx = np.arange(N).reshape(nz, ny, nx)
    rows, cols, vals = [np.arange(N)], [np.arange(N)], [np.full(N, 7.0)]
    for axis in (2, 1, 0):
        a = idx.take(range(idx.shape[axis] - 1), axis=axis).ravel()
        b = idx.take(range(1, idx.shape[axis]), axis=axis).ravel()
        if len(a) == 0:
            continue
        wv = rng.uniform(0.2, 1.0, len(a))
        rows += [a, b]
        cols += [b, a]
        vals += [-wv, -wv]
    return G.crs_from_unsorted(N, np.concatenate(rows), np.concatenate(cols),
                               np.concatenate(vals))


def odd_band_matrix(N, offs, seed):
    """SPD matrix whose offsets are `offs` (not a grid's)."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [np.arange(N)], [np.arange(N)], [np.full(N, 2.0 * len(offs) + 1)]
    for dk in offs[1:]:
        a = np.arange(N - dk)
        wv = rng.uniform(0.2, 1.0, len(a))
        rows += [a, a + dk]
        cols += [a + dk, a]
        vals += [-wv, -wv]
    return G.crs_from_unsorted(N, np.concatenate(rows), np.concatenate(cols),
                               np.concatenate(vals))


def band_rows(A, offs):
    """Row-major U (N x 4) and the factor's band Gb (N x 4) of G = the
    scaled |tril(A)| with unit diagonal; offsets past the stored ones are 0
    with zero values, as the device views pad them."""
    rows = np.repeat(np.arange(A.N), np.diff(A.ptr))
    U = np.zeros((A.N, 4), np.float32)
    Gb = np.zeros((A.N, 4), np.float32)
    top = np.abs(A.value).max()
    for r, c, v in zip(rows, A.index, A.value):
        if c >= r:
            U[r, offs.index(int(c - r))] = v
        else:
            Gb[r, offs.index(int(r - c))] = abs(v) / top
    Gb[np.arange(A.N), 0] = 1.0
    return U, Gb, list(offs) + [0] * (4 - len(offs))


def lower_csr(Gb, offs):
    """G and G^T as CRS from the factor's band (the padded offsets, 0 with
    zero values, add nothing)."""
    N = len(Gb)
    rows, cols, vals = [], [], []
    for k, dk in enumerate(offs):
        if k > 0 and dk == 0:
            continue
        r = np.arange(N)
        keep = (Gb[:, k] != 0) & (r - dk >= 0)
        rows.append(r[keep])
        cols.append(r[keep] - dk)
        vals.append(Gb[keep, k].astype(np.float64))
    rows, cols, vals = map(np.concatenate, (rows, cols, vals))
    return (G.crs_from_unsorted(N, rows, cols, vals), G.crs_from_unsorted(N, cols, rows, vals))


CASES = {"grid3d": (23, 11, 7), "grid2d": (45, 20, 1), "thin": (33, 3, 2),
         "line": (1, 1, 17), "odd": None}


def _setup(case):
    if case == "odd":
        offs = [0, 1, 5, 19]
        A = odd_band_matrix(301, offs, seed=3)
    else:
        nx, ny, nz = CASES[case]
        A = grid_matrix(nx, ny, nz, seed=nx + ny + nz)
        offs = [0]
        # the offsets a neighbour pair really has: x (nx > 1), y (ny > 1), z (nz > 1)
        for dk, present in ((1, nx > 1), (nx, ny > 1), (nx * ny, nz > 1)):
            if present and dk not in offs:
                offs.append(dk)
        offs.sort()
    U, Gb, d4 = band_rows(A, offs)
    return A, U, Gb, d4


@pytest.mark.parametrize("case", sorted(CASES))
def test_fused_products_stay_in_bounds_and_match(case):
    A, U, Gb, d4 = _setup(case)
    N = A.N
    rng = np.random.default_rng(1)
    x = Buf(rng.standard_normal(N))
    zero = Buf(np.zeros(N))
    pn, dn, q = band_dir(d4, Buf(U), x, zero, zero, 0.0, 0.0, N)
    A32 = G.Crs(N, A.ptr, A.index, A.value.astype(np.float32).astype(np.float64))
    xd = x.v.astype(np.float64)
    assert np.allclose(q, A32.matvec(xd), rtol=1e-5, atol=1e-5)
    assert np.array_equal(pn, x.v) and np.all(dn == 0)
    Gl, Gt = lower_csr(Gb, d4)
    C = Buf(rng.uniform(0.5, 1.5, N))
    zg = gband_z(d4, Buf(Gb), x, zero, C, 0.0, N)
    assert np.allclose(zg, Gl.matvec(xd), rtol=1e-5, atol=1e-5)
    rn, y = gband_res(d4, Buf(Gb), x, zero, 0.0, N)
    assert np.array_equal(rn, x.v)
    assert np.allclose(y, Gt.matvec(xd), rtol=1e-5, atol=1e-5)


def _pcg(A32, apply, b, iters):
    xr, r = np.zeros(len(b)), b.copy()
    zz = apply(r)
    p, rho = zz.copy(), r @ zz
    for _ in range(iters):
        q = A32.matvec(p)
        a = rho / (p @ q)
        xr += a * p
        r -= a * q
        zz = apply(r)
        rn = r @ zz
        p = zz + (rn / rho) * p
        rho = rn
    return xr


@pytest.mark.parametrize("learned", [True, False])
@pytest.mark.parametrize("case", ["grid3d", "grid2d", "odd"])
def test_persistent_iteration_matches_pcg(case, learned):
    """k_inner_persist's phases in its order (ping-pong p and r, d one
    update behind, applied at the end as k_outer_update_pending does)
    against a plain PCG with M^-1 = G G^T + eps C or C."""
    A, U, Gb, d4 = _setup(case)
    N = A.N
    Gl, Gt = lower_csr(Gb, d4)
    A32 = G.Crs(N, A.ptr, A.index, A.value.astype(np.float32).astype(np.float64))
    rng = np.random.default_rng(6)
    b = rng.standard_normal(N)
    Cv = rng.uniform(0.5, 1.5, N).astype(np.float32)
    eps = 0.25 if learned else 0.0
    iters = 12
    if learned:
        apply = lambda r: Gl.matvec(Gt.matvec(r)) + eps * Cv * r
    else:
        apply = lambda r: Cv * r
    xr = _pcg(A32, apply, b, iters)

    Ub, Gbb, C = Buf(U), Buf(Gb), Buf(Cv)
    r = [Buf(b), Buf(np.zeros(N))]
    z = Buf(apply(r[0].v.astype(np.float64)))
    p = [Buf(z.v), Buf(np.zeros(N))]
    d = Buf(np.zeros(N))
    rho = float(r[0].v.astype(np.float64) @ z.v)
    al = be = 0.0
    par = 0
    for _ in range(iters):
        pn, dn, q = band_dir(d4, Ub, z, p[par], d, al, be, N)
        p[1 - par], d, qb = Buf(pn), Buf(dn), Buf(q)
        al = rho / float(pn.astype(np.float64) @ q)
        if learned:
            rn_, y = gband_res(d4, Gbb, r[par], qb, -al, N)
            r[1 - par] = Buf(rn_)
        else:
            r0 = fma(-al, q, r[0].v)
            r[0] = Buf(r0)
            z = Buf(Cv * r0)
        par = 1 - par
        if learned:
            rcur = r[par]
            z = Buf(gband_z(d4, Gbb, Buf(y), rcur, C, eps, N))
        else:
            rcur = r[0]
        rn = float(rcur.v.astype(np.float64) @ z.v)
        be, rho = rn / rho, rn
    xf = d.v + al * p[par].v
    assert np.allclose(xf, xr, rtol=2e-3, atol=2e-3 * np.abs(xr).max())


@pytest.mark.parametrize("defer", [False, True])
@pytest.mark.parametrize("learned", [True, False])
@pytest.mark.parametrize("case", ["grid3d", "odd"])
def test_split_iteration_matches_pcg(case, learned, defer):
    """k_inner_persist_split's phases in its order (q = A p | r -= a q
    [, d += a p] | y = G^T r | z = G y + eps C r | [d += a p,] p = z + b p;
    Jacobi without the two factor phases and with p = C r + b p) against a
    plain PCG. The loop stops after its residual phase; with the d update
    deferred to the direction phase, the last one is pending and applied at
    the end, as k_outer_update_pending does."""
    A, U, Gb, d4 = _setup(case)
    N = A.N
    Gl, Gt = lower_csr(Gb, d4)
    A32 = G.Crs(N, A.ptr, A.index, A.value.astype(np.float32).astype(np.float64))
    rng = np.random.default_rng(8)
    b = rng.standard_normal(N)
    Cv = rng.uniform(0.5, 1.5, N).astype(np.float32)
    eps = 0.25 if learned else 0.0
    iters = 12
    if learned:
        apply = lambda r: Gl.matvec(Gt.matvec(r)) + eps * Cv * r
    else:
        apply = lambda r: Cv * r
    xr = _pcg(A32, apply, b, iters)

    Ub, Gbb, C = Buf(U), Buf(Gb), Buf(Cv)
    r = b.astype(np.float32)
    z = apply(r.astype(np.float64)).astype(np.float32)
    p = z.copy()
    d = np.zeros(N, np.float32)
    rho = float(r.astype(np.float64) @ z)
    zero = Buf(np.zeros(N))
    for k in range(iters):
        _, _, q = band_dir(d4, Ub, zero, Buf(p), zero, 0.0, 1.0, N)  # q = A p
        al = rho / float(p.astype(np.float64) @ q)
        r = fma(-al, q, r)
        if not defer:
            d = fma(al, p, d)
        if k == iters - 1:
            break  # the residual test stops the loop here
        if learned:
            _, y = gband_res(d4, Gbb, Buf(r), zero, 0.0, N)  # y = G^T r
            z = gband_z(d4, Gbb, Buf(y), Buf(r), C, eps, N)
        else:
            z = (Cv * r).astype(np.float32)
        rn = float(r.astype(np.float64) @ z)
        be, rho = rn / rho, rn
        if defer:
            d = fma(al, p, d)
        p = fma(be, p, z)
    xf = fma(al, p, d) if defer else d  # the pending update
    assert np.allclose(xf, xr, rtol=2e-3, atol=2e-3 * np.abs(xr).max())


@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("learned", [True, False])
def test_persistent_slots_are_read_before_reuse(learned, split):
    """Phase k writes slot k before a barrier and every CTA reads it after
    that barrier (the Jacobi phase B writes slots 1 and 2, read after its
    barrier); the split form adds barriers after y = G^T r and after the
    direction update. A CTA may write a slot again only once it has passed a later
    barrier than the one after which the slot was last read: then every CTA
    has finished reading it."""
    bar = 0
    last_read = {}  # slot -> barrier after which it was read
    for it in range(5):
        events = [("w", 0), ("b",), ("r", 0)]
        if learned:
            events += [("w", 1), ("b",), ("r", 1)]
            events += [("b",)] if split else []  # y = G^T r
            events += [("w", 2), ("b",), ("r", 2)]
        else:
            events += [("w", 1), ("w", 2), ("b",), ("r", 1), ("r", 2)]
        events += [("b",)] if split else []  # p = z + b p
        for e in events:
            if e[0] == "b":
                bar += 1
            elif e[0] == "r":
                last_read[e[1]] = bar
            else:
                assert e[1] not in last_read or bar > last_read[e[1]], (it, e, bar, last_read)


@pytest.mark.parametrize("tpb", [256, 512, 1024])
def test_persistent_grid_fits_the_slots(tpb):
    """The persistent grid (SMs x resident CTAs of tpb threads, at most one
    CTA per tpb-row tile) never exceeds the kMaxGrid partial-sum slots, and
    the grid-stride loops cover every row once, one row per thread and four
    per thread (with the N mod 4 tail)."""
    kMaxGrid = 148 * 8
    for per_sm in (1, 2048 // tpb):
        for N in (1, 255, 256, 257, 4099, 884736):
            tiles = -(-N // tpb)
            grid = max(1, min(148 * per_sm, kMaxGrid, tiles))
            assert grid <= kMaxGrid
            seen = np.zeros(N, np.int32)
            for blk in range(grid):
                for start in range(blk * tpb, N, grid * tpb):
                    seen[start:min(N, start + tpb)] += 1
            assert np.all(seen == 1)
            seen[:] = 0
            n4 = N // 4
            for blk in range(grid):
                for start in range(blk * tpb, n4, grid * tpb):
                    seen[4 * start:4 * min(n4, start + tpb)] += 1
                for start in range(4 * n4 + blk * tpb, N, grid * tpb):
                    seen[start:min(N, start + tpb)] += 1
            assert np.all(seen == 1)
