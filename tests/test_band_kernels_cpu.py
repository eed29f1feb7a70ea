"""The z-marching stencil kernels (cgxx_b200/csrc/stencil.cuh) restated in
numpy (no GPU).

A CTA owns a 32 x 8 tile of the x-y plane (lane = x, warp = y) and marches
through a chunk of planes; x and y neighbours come from a shared-memory tile
with a one-cell halo, z neighbours from the previous and next plane of the
thread's own column. Tiles may run past the grid's edge (their cells clamped
to it). This file restates that arithmetic cell by cell and checks, before
the kernels run on a device:

  - every load stays inside the buffer it addresses (U and the factor hold
    N rows, the vectors N + 8 entries) and every store hits a valid cell;
  - the products equal A p, G y and G^T r (the symmetric band form's
    values), on full and partial tiles, 2-D grids and uneven plane chunks;
  - the fused inner iteration (p and r formed again at neighbouring cells,
    ping-pong buffers, the lagged update of d applied at the end) gives
    what the unfused PCG gives.
"""
import numpy as np
import pytest

from cgxx_b200 import generators as G

PAD = 8
SX, SY = 32, 8


class Buf:
    """A device buffer with bounds-checked loads."""

    def __init__(self, values, size):
        self.size = size
        self.v = np.zeros((size,) + np.shape(values)[1:], np.float32)
        self.v[:len(values)] = values

    def __getitem__(self, idx):
        idx = np.asarray(idx)
        assert idx.min() >= 0 and idx.max() < self.size, (idx.min(), idx.max(), self.size)
        return self.v[idx]


def geom(nx, ny, nz, sms=148):
    tiles_x, tiles_y = -(-nx // SX), -(-ny // SY)
    tiles = tiles_x * tiles_y
    want = min(6 * sms, 1184)
    chunks = max(1, min(nz, -(-want // tiles), 1184 // tiles))
    lz = -(-nz // chunks)
    return dict(nx=nx, ny=ny, nz=nz, tx=tiles_x, ty=tiles_y, lz=lz,
                grid=tiles * -(-nz // lz))


def tiles_of(g):
    """(tx, ty, z0, z1) per CTA, and the tile's clamped cell columns."""
    lane, w = np.meshgrid(np.arange(SX), np.arange(SY))
    lane, w = lane.ravel(), w.ravel()
    for b in range(g["grid"]):
        tx, rest = b % g["tx"], b // g["tx"]
        ty, chunk = rest % g["ty"], rest // g["ty"]
        x, y = tx * SX + lane, ty * SY + w
        valid = (x < g["nx"]) & (y < g["ny"])
        col = np.minimum(y, g["ny"] - 1) * g["nx"] + np.minimum(x, g["nx"] - 1)
        z0 = chunk * g["lz"]
        z1 = min(g["nz"], z0 + g["lz"])
        yield lane, w, valid, col, z0, z1, x == g["nx"] - 1, y == g["ny"] - 1


def st_dir(g, U, z, pold, d, al, be, N):
    """k_st_dir: returns (p_new, d_new, q) on the valid cells."""
    plane = g["nx"] * g["ny"]
    nx = g["nx"]
    pn_out, d_out, q_out = np.full(N, np.nan), np.full(N, np.nan), np.full(N, np.nan)
    pn = lambda j: be * pold[j] + z[j]  # noqa: E731
    for lane, w, valid, col, z0, z1, _, _ in tiles_of(g):
        if z0 >= z1:
            continue
        i = z0 * plane + col
        p_m = pn(i - plane) if z0 > 0 else np.zeros(len(i))
        lw = U[i - plane][:, 3] if z0 > 0 else np.zeros(len(i))
        po_c = pold[i]
        p_c = be * po_c + z[i]
        for zz in range(z0, z1):
            u = U[i]
            inn = np.minimum(i + plane, N - 1)
            po_n = pold[inn]
            p_n = be * po_n + z[inn]
            sp = np.zeros((SY + 2, SX + 2))
            suy = np.zeros((SY, SX + 1))
            suz = np.zeros((SY + 1, SX))
            sp[w + 1, lane + 1] = p_c
            suy[w, lane + 1] = u[:, 1]
            suz[w + 1, lane] = u[:, 2]
            m = lane == 0
            sp[w[m] + 1, 0] = pn(np.maximum(i[m] - 1, 0))
            suy[w[m], 0] = U[np.maximum(i[m] - 1, 0)][:, 1]
            m = lane == SX - 1
            sp[w[m] + 1, SX + 1] = pn(np.minimum(i[m] + 1, N - 1))
            m = w == 0
            sp[0, lane[m] + 1] = pn(np.maximum(i[m] - nx, 0))
            suz[0, lane[m]] = U[np.maximum(i[m] - nx, 0)][:, 2]
            m = w == SY - 1
            sp[SY + 1, lane[m] + 1] = pn(np.minimum(i[m] + nx, N - 1))
            lv1 = np.where(i < 1, 0, suy[w, lane])
            lv2 = np.where(i < nx, 0, suz[w, lane])
            lv3 = np.where(i < plane, 0, lw)
            s = (u[:, 0] * p_c + u[:, 1] * sp[w + 1, lane + 2] + u[:, 2] * sp[w + 2, lane + 1]
                 + u[:, 3] * p_n + lv1 * sp[w + 1, lane] + lv2 * sp[w, lane + 1] + lv3 * p_m)
            iv = i[valid]
            assert np.all(np.isnan(q_out[iv]))  # each cell written once
            q_out[iv], pn_out[iv] = s[valid], p_c[valid]
            d_out[iv] = d[iv] + al * po_c[valid]
            p_m, p_c, po_c, lw = p_c, p_n, po_n, u[:, 3]
            i = i + plane
    return pn_out, d_out, q_out


def st_res(g, Gb, rold, q, al, N):
    """k_st_res: returns (r_new, y = G^T r_new)."""
    plane, nx = g["nx"] * g["ny"], g["nx"]
    r_out, y_out = np.full(N, np.nan), np.full(N, np.nan)
    rn = lambda j: rold[j] - al * q[j]  # noqa: E731
    for lane, w, valid, col, z0, z1, xlast, ylast in tiles_of(g):
        if z0 >= z1:
            continue
        i = z0 * plane + col
        r_c, gc = rn(i), Gb[i]
        for zz in range(z0, z1):
            inn = np.minimum(i + plane, N - 1)
            r_n, gn = rn(inn), Gb[inn]
            sr = np.zeros((SY + 1, SX + 1))
            sg1 = np.zeros((SY, SX + 1))
            sg2 = np.zeros((SY + 1, SX))
            sr[w, lane], sg1[w, lane], sg2[w, lane] = r_c, gc[:, 1], gc[:, 2]
            m = lane == SX - 1
            j = np.minimum(i[m] + 1, N - 1)
            sr[w[m], SX], sg1[w[m], SX] = rn(j), Gb[j][:, 1]
            m = w == SY - 1
            j = np.minimum(i[m] + nx, N - 1)
            sr[SY, lane[m]], sg2[SY, lane[m]] = rn(j), Gb[j][:, 2]
            v1 = np.where((i + 1 < N) & ~xlast, sg1[w, lane + 1], 0)
            v2 = np.where((i + nx < N) & ~ylast, sg2[w + 1, lane], 0)
            v3 = np.where(i + plane < N, gn[:, 3], 0)
            s = gc[:, 0] * r_c + v1 * sr[w, lane + 1] + v2 * sr[w + 1, lane] + v3 * r_n
            iv = i[valid]
            assert np.all(np.isnan(y_out[iv]))
            r_out[iv], y_out[iv] = r_c[valid], s[valid]
            r_c, gc = r_n, gn
            i = i + plane
    return r_out, y_out


def st_gz(g, Gb, y, N):
    """k_st_gz: z = G y."""
    plane, nx = g["nx"] * g["ny"], g["nx"]
    out = np.full(N, np.nan)
    for lane, w, valid, col, z0, z1, _, _ in tiles_of(g):
        if z0 >= z1:
            continue
        i = z0 * plane + col
        y_m = y[i - plane] if z0 > 0 else y[np.zeros(len(i), int)]
        y_c = y[i]
        for zz in range(z0, z1):
            gv = Gb[i]
            sy = np.zeros((SY + 1, SX + 1))
            sy[w + 1, lane + 1] = y_c
            m = lane == 0
            sy[w[m] + 1, 0] = y[np.maximum(i[m] - 1, 0)]
            m = w == 0
            sy[0, lane[m] + 1] = y[np.maximum(i[m] - nx, 0)]
            y_n = y[np.minimum(i + plane, N - 1)]
            s = (gv[:, 0] * y_c + gv[:, 1] * sy[w + 1, lane] + gv[:, 2] * sy[w, lane + 1]
                 + gv[:, 3] * y_m)
            iv = i[valid]
            assert np.all(np.isnan(out[iv]))
            out[iv] = s[valid]
            y_m, y_c = y_c, y_n
            i = i + plane
    return out


def band_rows(A, nx, plane):
    """Row-major U (N x 4) for offsets 0, 1, nx, plane and the lower factor
    values Gb[i][k] = G(i, i - d_k) of G = |tril(A)| scaled."""
    d = [0, 1, nx, plane]
    rows = np.repeat(np.arange(A.N), np.diff(A.ptr))
    U = np.zeros((A.N, 4), np.float32)
    Gb = np.zeros((A.N, 4), np.float32)
    top = np.abs(A.value).max()
    for r, c, v in zip(rows, A.index, A.value):
        if c >= r:
            U[r, d.index(int(c - r))] = v
        else:
            Gb[r, d.index(int(r - c))] = abs(v) / top
    Gb[np.arange(A.N), 0] = 1.0
    return U, Gb


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


CASES = {"full": (64, 16, 5), "partial": (37, 11, 7), "chunked": (9, 9, 41),
         "flat": (45, 20, 1), "thin": (33, 3, 2)}


def _setup(case):
    nx, ny, nz = CASES[case]
    A = grid_matrix(nx, ny, nz, seed=nx + ny + nz)
    U, Gb = band_rows(A, nx, nx * ny)
    g = geom(nx, ny, nz)
    return A, U, Gb, g


def _lower_csr(Gb, nx, plane):
    N = len(Gb)
    rows, cols, vals = [], [], []
    for k, dk in enumerate((0, 1, nx, plane)):
        r = np.arange(N)
        keep = (Gb[:, k] != 0) & (r - dk >= 0)
        rows.append(r[keep])
        cols.append(r[keep] - dk)
        vals.append(Gb[keep, k].astype(np.float64))
    rows, cols, vals = map(np.concatenate, (rows, cols, vals))
    return (G.crs_from_unsorted(N, rows, cols, vals), G.crs_from_unsorted(N, cols, rows, vals))


@pytest.mark.parametrize("case", sorted(CASES))
def test_stencil_products_stay_in_bounds_and_match(case):
    A, U, Gb, g = _setup(case)
    N = A.N
    rng = np.random.default_rng(1)
    size = N + PAD
    x = Buf(rng.standard_normal(N).astype(np.float32), size)
    zero = Buf(np.zeros(N, np.float32), size)
    pn, dn, q = st_dir(g, Buf(U, N), x, zero, zero, 0.0, 0.0, N)
    A32 = G.Crs(N, A.ptr, A.index, A.value.astype(np.float32).astype(np.float64))
    xd = x.v[:N].astype(np.float64)
    assert np.allclose(q, A32.matvec(xd), rtol=1e-5, atol=1e-5)
    assert np.array_equal(pn, x.v[:N]) and np.all(dn == 0)
    Gl, Gt = _lower_csr(Gb, g["nx"], g["nx"] * g["ny"])
    assert np.allclose(st_gz(g, Buf(Gb, N), x, N), Gl.matvec(xd), rtol=1e-5, atol=1e-5)
    rn, y = st_res(g, Buf(Gb, N), x, zero, 0.0, N)
    assert np.array_equal(rn, x.v[:N])
    assert np.allclose(y, Gt.matvec(xd), rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("case", ["partial", "chunked", "flat"])
def test_fused_learned_iteration_matches_pcg(case):
    """Inner PCG with M^-1 = G G^T: the fused stencil kernels (ping-pong p
    and r, d one update behind, applied at the end) against a plain PCG."""
    A, U, Gb, g = _setup(case)
    N = A.N
    Gl, Gt = _lower_csr(Gb, g["nx"], g["nx"] * g["ny"])
    A32 = G.Crs(N, A.ptr, A.index, A.value.astype(np.float32).astype(np.float64))
    b = np.random.default_rng(6).standard_normal(N)
    iters = 12

    xr, r = np.zeros(N), b.copy()
    zz = Gl.matvec(Gt.matvec(r))
    p, rho = zz.copy(), r @ zz
    for _ in range(iters):
        q = A32.matvec(p)
        a = rho / (p @ q)
        xr += a * p
        r -= a * q
        zz = Gl.matvec(Gt.matvec(r))
        rn = r @ zz
        p = zz + (rn / rho) * p
        rho = rn

    size = N + PAD
    Ub, Gbb = Buf(U, N), Buf(Gb, N)
    rbuf = [Buf(b.astype(np.float32), size), Buf(np.zeros(N, np.float32), size)]
    zv = Buf(Gl.matvec(Gt.matvec(rbuf[0].v[:N].astype(np.float64))).astype(np.float32), size)
    pbuf = [Buf(zv.v[:N], size), Buf(np.zeros(N, np.float32), size)]
    dv = Buf(np.zeros(N, np.float32), size)
    rho = float(rbuf[0].v[:N].astype(np.float64) @ zv.v[:N])
    al = be = 0.0
    for it in range(iters):
        par = it & 1
        pn, dn, q = st_dir(g, Ub, zv, pbuf[par], dv, al, be, N)
        pbuf[1 - par], dv, qb = Buf(pn, size), Buf(dn, size), Buf(q, size)
        al = rho / float(pn @ q)
        rnew, y = st_res(g, Gbb, rbuf[par], qb, al, N)
        rbuf[1 - par] = Buf(rnew, size)
        zvv = st_gz(g, Gbb, Buf(y, size), N)
        zv = Buf(zvv, size)
        rn = float(rnew.astype(np.float64) @ zvv)
        be, rho = rn / rho, rn
    xf = dv.v[:N] + al * pbuf[iters & 1].v[:N]
    assert np.allclose(xf, xr, rtol=2e-3, atol=2e-3 * np.abs(xr).max())
