"""The band kernels' warp arithmetic restated in numpy (no GPU).

cgxx_b200/csrc/band.cuh runs one row per lane, 32 consecutive rows per warp
(the last warp may run past row N - 1, its rows clamped), takes the rows
i +- 1 from the adjacent lanes when d_1 = 1 and loads the rest at clamped
offsets from slot-major arrays. This file restates that arithmetic lane by
lane and checks two things before the kernels ever run on a device:

  - every load and store stays inside the buffer it addresses (the slot
    arrays hold 4 * band_ld(N) values, the vectors N + 8);
  - the products and the fused inner iteration (p and r formed again at
    neighbouring rows, ping-pong buffers, the lagged update of d) give what
    the unfused PCG gives, to FP32 rounding.
"""
import numpy as np
import pytest

from cgxx_b200 import generators as G

PAD = 8  # elements of padding after every device vector


def band_ld(N):
    return (N + 63) // 64 * 64


class Buf:
    """A device buffer with bounds-checked gathers."""

    def __init__(self, values, size):
        self.size = size
        self.v = np.zeros(size, np.float32)
        self.v[:len(values)] = values

    def __getitem__(self, idx):
        idx = np.asarray(idx)
        assert idx.min() >= 0 and idx.max() < self.size, (idx.min(), idx.max(), self.size)
        return self.v[idx]


def lanes(N):
    i = np.arange((N + 31) // 32 * 32)
    return i, i - i % 32, i % 32, np.minimum(i, N - 1)


def lane_next(v, edge, lane):
    return np.where(lane == 31, edge, np.roll(v, -1))


def lane_prev(v, edge, lane):
    return np.where(lane == 0, edge, np.roll(v, 1))


def warp_hi(base, N):
    return np.minimum(base + 32, N - 1)


def warp_lo(base):
    return np.maximum(base - 1, 0)


def f32(a):
    return np.asarray(a, np.float32)


def band_of(A):
    """Slot-major U (4 slots of band_ld(N)) and the padded offsets d."""
    rows = np.repeat(np.arange(A.N), np.diff(A.ptr))
    D = sorted(set(int(d) for d in np.unique(A.index - rows) if d > 0))
    up = [0] + D
    assert len(up) <= 4
    ld = band_ld(A.N)
    U = np.zeros(4 * ld, np.float32)
    for r, c, v in zip(rows, A.index, A.value):
        if c >= r:
            U[up.index(int(c - r)) * ld + r] = v
    return Buf(U, 4 * ld), ld, up + [0] * (4 - len(up))


def k_band(U, ld, d, x, N):
    """k_band<D1>: y = A x (valid rows)."""
    i, base, lane, ic = lanes(N)
    D1 = d[1] == 1
    u = [U[k * ld + ic] for k in range(4)]
    x0 = x[ic]
    if D1:
        hi, lo = warp_hi(base, N), warp_lo(base)
        xu1 = lane_next(x0, x[hi], lane)
        xl1 = lane_prev(x0, x[lo], lane)
        lv1 = lane_prev(u[1], U[ld + lo], lane)
        lv1 = np.where(i < 1, 0, lv1)
    else:
        xu1 = x[np.minimum(ic + d[1], N - 1)]
        j = ic - d[1]
        jc = np.maximum(j, 0)
        lv1 = np.where(j < 0, 0, U[ld + jc])
        xl1 = x[jc]
    xu = [x0, xu1] + [x[np.minimum(ic + d[k], N - 1)] for k in (2, 3)]
    lv, xl = [None, lv1], [None, xl1]
    for k in (2, 3):
        j = ic - d[k]
        jc = np.maximum(j, 0)
        lv.append(np.where(j < 0, 0, U[k * ld + jc]))
        xl.append(x[jc])
    s = u[0] * xu[0]
    for k in (1, 2, 3):
        s = s + u[k] * xu[k]
    for k in (1, 2, 3):
        s = s + lv[k] * xl[k]
    return s[:N]


def k_band_dir(U, ld, d, z, pold, dvec, al, be, N):
    """k_band_dir<D1>: returns (p_new, d_new, q)."""
    i, base, lane, ic = lanes(N)
    D1 = d[1] == 1
    pn = lambda j: be * pold[j] + z[j]  # noqa: E731
    po = pold[ic]
    p0 = be * po + z[ic]
    u = [U[k * ld + ic] for k in range(4)]
    if D1:
        hi, lo = warp_hi(base, N), warp_lo(base)
        pu1 = lane_next(p0, pn(hi), lane)
        pl1 = lane_prev(p0, pn(lo), lane)
        lv1 = np.where(i < 1, 0, lane_prev(u[1], U[ld + lo], lane))
    else:
        pu1 = pn(np.minimum(ic + d[1], N - 1))
        j = ic - d[1]
        jc = np.maximum(j, 0)
        lv1 = np.where(j < 0, 0, U[ld + jc])
        pl1 = pn(jc)
    pu = [p0, pu1] + [pn(np.minimum(ic + d[k], N - 1)) for k in (2, 3)]
    lv, pl = [None, lv1], [None, pl1]
    for k in (2, 3):
        j = ic - d[k]
        jc = np.maximum(j, 0)
        lv.append(np.where(j < 0, 0, U[k * ld + jc]))
        pl.append(pn(jc))
    s = u[0] * pu[0]
    for k in (1, 2, 3):
        s = s + u[k] * pu[k]
    for k in (1, 2, 3):
        s = s + lv[k] * pl[k]
    dn = dvec[ic] + al * po
    return p0[:N], dn[:N], s[:N]


def gband_of(Gl, N, d):
    """Slot-major Gb_k[i] = G(i, i - d_k) of a lower-triangular CRS G."""
    ld = band_ld(N)
    V = np.zeros(4 * ld, np.float32)
    rows = np.repeat(np.arange(N), np.diff(Gl.ptr))
    for r, c, v in zip(rows, Gl.index, Gl.value):
        V[d.index(int(r - c)) * ld + r] = v
    return Buf(V, 4 * ld), ld


def k_gband(Gb, ld, d, x, N, trans):
    i, base, lane, ic = lanes(N)
    D1 = d[1] == 1
    x0 = x[ic]
    if not trans:
        v = [Gb[k * ld + ic] for k in range(4)]
        x1 = lane_prev(x0, x[warp_lo(base)], lane) if D1 else x[np.maximum(ic - d[1], 0)]
        xs = [x0, x1, x[np.maximum(ic - d[2], 0)], x[np.maximum(ic - d[3], 0)]]
    else:
        v = [Gb[ic]]
        if D1:
            hi = warp_hi(base, N)
            v1 = lane_next(Gb[ld + ic], Gb[ld + hi], lane)
            x1 = lane_next(x0, x[hi], lane)
            v.append(np.where(i + 1 < N, v1, 0))
        else:
            j = ic + d[1]
            jc = np.minimum(j, N - 1)
            v.append(np.where(j < N, Gb[ld + jc], 0))
            x1 = x[jc]
        xs = [x0, x1]
        for k in (2, 3):
            j = ic + d[k]
            jc = np.minimum(j, N - 1)
            v.append(np.where(j < N, Gb[k * ld + jc], 0))
            xs.append(x[jc])
    s = v[0] * xs[0]
    for k in (1, 2, 3):
        s = s + v[k] * xs[k]
    return s[:N]


def k_gband_res(Gb, ld, d, rold, q, al, N):
    """k_gband_res<D1>: returns (r_new, y = G^T r_new)."""
    i, base, lane, ic = lanes(N)
    D1 = d[1] == 1
    rn = lambda j: rold[j] - al * q[j]  # noqa: E731
    r0 = rn(ic)
    v = [Gb[ic]]
    if D1:
        hi = warp_hi(base, N)
        v1 = lane_next(Gb[ld + ic], Gb[ld + hi], lane)
        xs = [r0, lane_next(r0, rn(hi), lane)]
        v.append(np.where(i + 1 < N, v1, 0))
    else:
        j = ic + d[1]
        jc = np.minimum(j, N - 1)
        v.append(np.where(j < N, Gb[ld + jc], 0))
        xs = [r0, rn(jc)]
    for k in (2, 3):
        j = ic + d[k]
        jc = np.minimum(j, N - 1)
        v.append(np.where(j < N, Gb[k * ld + jc], 0))
        xs.append(rn(jc))
    s = v[0] * xs[0]
    for k in (1, 2, 3):
        s = s + v[k] * xs[k]
    return r0[:N], s[:N]


def _strided(N, seed):
    """SPD matrix with offsets 0, +-2, +-9 (d_1 = 2: no lane shuffles)."""
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


CASES = {
    "7pt_5": lambda: G.diffusion3d(5, 7, seed=1),        # N 125, d 0 1 5 25
    "7pt_4": lambda: G.diffusion3d(4, 7, seed=2),        # N 64, whole warps
    "5pt_7": lambda: G.poisson2d(7),                     # N 49, K = 3
    "5pt_2": lambda: G.poisson2d(2),                     # N 4 < one warp
    "strided_77": lambda: _strided(77, 3),               # d_1 = 2
}


def _lower(A):
    rows = np.repeat(np.arange(A.N), np.diff(A.ptr))
    keep = A.index <= rows
    return G.crs_from_unsorted(A.N, rows[keep], A.index[keep],
                               np.abs(A.value[keep]) / np.abs(A.value).max())


@pytest.mark.parametrize("case", sorted(CASES))
def test_products_stay_in_bounds_and_match(case):
    A = CASES[case]()
    N = A.N
    U, ld, d = band_of(A)
    rng = np.random.default_rng(4)
    x = Buf(f32(rng.standard_normal(N)), N + PAD)
    y = k_band(U, ld, d, x, N)
    Af = G.Crs(N, A.ptr, A.index, A.value.astype(np.float32).astype(np.float64))
    assert np.allclose(y, Af.matvec(x.v[:N].astype(np.float64)), rtol=1e-5, atol=1e-5)
    Gl = _lower(A)
    Gb, gld = gband_of(Gl, N, d)
    Gd = G.Crs(N, Gl.ptr, Gl.index, Gl.value.astype(np.float32).astype(np.float64))
    z = k_gband(Gb, gld, d, x, N, trans=False)
    assert np.allclose(z, Gd.matvec(x.v[:N].astype(np.float64)), rtol=1e-5, atol=1e-5)
    GT = G.crs_from_unsorted(N, Gd.index, np.repeat(np.arange(N), np.diff(Gd.ptr)), Gd.value)
    yt = k_gband(Gb, gld, d, x, N, trans=True)
    assert np.allclose(yt, GT.matvec(x.v[:N].astype(np.float64)), rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("case", sorted(CASES))
def test_fused_learned_iteration_matches_pcg(case):
    """Inner PCG with M^-1 = G G^T: the fused kernels (ping-pong p and r,
    d one update behind, applied at the end) against a plain PCG."""
    A = CASES[case]()
    N = A.N
    U, ld, d = band_of(A)
    Gl = _lower(A)
    Gb, gld = gband_of(Gl, N, d)
    rows = np.repeat(np.arange(N), np.diff(Gl.ptr))
    gv = Gb.v[np.array([d.index(int(r - c)) * gld + r for r, c in zip(rows, Gl.index)], int)]
    Gd = G.Crs(N, Gl.ptr, Gl.index, gv.astype(np.float64))
    GT = G.crs_from_unsorted(N, Gl.index, rows, gv.astype(np.float64))
    A32 = G.Crs(N, A.ptr, A.index, A.value.astype(np.float32).astype(np.float64))
    b = np.random.default_rng(6).standard_normal(N)
    iters = min(12, N)

    # Plain PCG (float64 on the FP32 operator).
    xr = np.zeros(N)
    r = b.copy()
    zz = Gd.matvec(GT.matvec(r))
    p = zz.copy()
    rho = r @ zz
    for _ in range(iters):
        q = A32.matvec(p)
        a = rho / (p @ q)
        xr += a * p
        r -= a * q
        zz = Gd.matvec(GT.matvec(r))
        rn = r @ zz
        p = zz + (rn / rho) * p
        rho = rn

    # Fused: start (r, z = G G^T r, p = z, a = b = 0), then the three kernels.
    size = N + PAD
    rbuf = [Buf(f32(b), size), Buf(np.zeros(N, np.float32), size)]
    y = Buf(k_gband(Gb, gld, d, rbuf[0], N, trans=True), size)
    zb = Buf(k_gband(Gb, gld, d, y, N, trans=False), size)
    pbuf = [Buf(zb.v[:N], size), Buf(np.zeros(N, np.float32), size)]
    dv = Buf(np.zeros(N, np.float32), size)
    rho = float(rbuf[0].v[:N].astype(np.float64) @ zb.v[:N])
    al = be = np.float32(0)
    for it in range(iters):
        par = it & 1
        pn, dn, q = k_band_dir(U, ld, d, zb, pbuf[par], dv, al, be, N)
        pbuf[1 - par] = Buf(f32(pn), size)
        dv = Buf(f32(dn), size)
        qb = Buf(f32(q), size)
        al = np.float32(rho / float(pn.astype(np.float64) @ q.astype(np.float64)))
        rnew, yv = k_gband_res(Gb, gld, d, rbuf[par], qb, al, N)
        rbuf[1 - par] = Buf(f32(rnew), size)
        zv = k_gband(Gb, gld, d, Buf(f32(yv), size), N, trans=False)
        zb = Buf(f32(zv), size)
        rn = float(rnew.astype(np.float64) @ zv.astype(np.float64))
        be = np.float32(rn / rho)
        rho = rn
    xf = dv.v[:N] + al * pbuf[iters & 1].v[:N]   # the pending update
    assert np.allclose(xf, xr, rtol=2e-3, atol=2e-3 * np.abs(xr).max())
