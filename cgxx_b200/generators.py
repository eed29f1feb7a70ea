"""Seeded synthetic SPD systems (numpy).

The reference ships no matrices; every workload here is generated from a
seed. All matrices come out in CRS with the column indices of each row in
ascending order -- the order the reference's reader produces for a symmetric
MatrixMarket file written row by row (Matrix.cpp:80-103 mirrors each
off-diagonal entry right after it, and CRS conversion keeps that order,
Matrix.cpp:203-228).

Families
  poisson2d(n)                5-point Laplacian, Dirichlet, diag 4 / off -1
  diffusion3d(n, stencil=7|27, sigma, corr_len, seed)
      cell-centred variable-coefficient diffusion with coefficient exp(g), g a
      Gaussian random field (FFT spectral synthesis, Gaussian covariance,
      correlation length `corr_len` cells, standard deviation `sigma`).
      Coupling of neighbours i, j: w_d * 2 k_i k_j / (k_i + k_j) (harmonic
      mean) with w_d = 1 / (|dx|+|dy|+|dz|) (faces 1, edges 1/2, corners 1/3);
      a neighbour outside the grid is a Dirichlet ghost cell with coupling
      w_d * k_i that goes into the diagonal only.
  geometric_graph(npts, mean_degree, seed)
      Laplacian of a random geometric graph in the unit cube, edge weights
      exp(-d / r), plus shift * I.
"""
from dataclasses import dataclass

import numpy as np


@dataclass
class Crs:
    N: int
    ptr: np.ndarray    # int32[N+1]
    index: np.ndarray  # int32[nz]
    value: np.ndarray  # float64[nz]

    @property
    def nz(self):
        return int(self.ptr[-1])

    def diagonal(self):
        d = np.zeros(self.N)
        rows = np.repeat(np.arange(self.N, dtype=np.int64), np.diff(self.ptr))
        m = rows == self.index
        d[rows[m]] = self.value[m]
        return d

    def matvec(self, x):
        rows = np.repeat(np.arange(self.N, dtype=np.int64), np.diff(self.ptr))
        return np.bincount(rows, weights=self.value * x[self.index], minlength=self.N)

    def rows(self):
        return np.repeat(np.arange(self.N, dtype=np.int32), np.diff(self.ptr))


def crs_from_sorted(N, rows, cols, vals):
    """CRS from entries already ordered by (row, col)."""
    ptr = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=N), out=ptr[1:])
    return Crs(N, ptr.astype(np.int32), cols.astype(np.int32), vals.astype(np.float64))


def crs_from_unsorted(N, rows, cols, vals):
    order = np.lexsort((cols, rows))
    return crs_from_sorted(N, rows[order], cols[order], vals[order])


# ---------------------------------------------------------------------------
# Structured grids

def _stencil_crs(shape, offsets, coupling, diag):
    """Builds a CRS matrix on a structured grid.

    offsets: list of (dz, dy, dx) sorted so that the linear index offset
    increases; coupling(k) -> float64 array over cells (value of the entry to
    the neighbour at offsets[k], NaN-free, defined where the neighbour is
    inside); diag: float64 array of diagonal values.
    """
    nz_, ny, nx = shape
    N = nz_ * ny * nx
    z, y, x = np.meshgrid(np.arange(nz_), np.arange(ny), np.arange(nx), indexing="ij")
    z, y, x = z.ravel(), y.ravel(), x.ravel()
    lin = np.arange(N, dtype=np.int64)
    masks, targets = [], []
    for (dz, dy, dx) in offsets:
        if (dz, dy, dx) == (0, 0, 0):
            masks.append(np.ones(N, dtype=bool))
            targets.append(lin)
            continue
        zz, yy, xx = z + dz, y + dy, x + dx
        m = (zz >= 0) & (zz < nz_) & (yy >= 0) & (yy < ny) & (xx >= 0) & (xx < nx)
        masks.append(m)
        targets.append(lin + (dz * ny + dy) * nx + dx)
    counts = np.zeros(N, dtype=np.int64)
    for m in masks:
        counts += m
    ptr = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr[1:])
    nnz = int(ptr[-1])
    index = np.empty(nnz, dtype=np.int32)
    value = np.empty(nnz, dtype=np.float64)
    pos = ptr[:-1].copy()
    for k, (off, m) in enumerate(zip(offsets, masks)):
        rows = np.nonzero(m)[0]
        p = pos[rows]
        index[p] = targets[k][rows]
        value[p] = diag[rows] if off == (0, 0, 0) else coupling(k)[rows]
        pos[rows] += 1
    return Crs(N, ptr.astype(np.int32), index, value)


def poisson2d(n):
    """2-D 5-point Poisson on an n x n grid, Dirichlet: diag 4, neighbours -1."""
    offsets = [(0, -1, 0), (0, 0, -1), (0, 0, 0), (0, 0, 1), (0, 1, 0)]
    N = n * n
    return _stencil_crs((1, n, n), offsets, lambda k: np.full(N, -1.0), np.full(N, 4.0))


def gaussian_random_field(shape, sigma, corr_len, rng):
    """Stationary Gaussian field with covariance sigma^2 exp(-r^2 / (2 l^2))
    by spectral synthesis on the periodic grid, normalised to mean 0 and
    standard deviation sigma."""
    white = rng.standard_normal(shape)
    k2 = np.zeros(shape)
    for ax, n in enumerate(shape):
        k = 2 * np.pi * np.fft.fftfreq(n)
        sh = [1] * len(shape)
        sh[ax] = n
        k2 = k2 + (k.reshape(sh)) ** 2
    amp = np.exp(-0.25 * corr_len ** 2 * k2)  # sqrt of exp(-l^2 k^2 / 2)
    g = np.real(np.fft.ifftn(np.fft.fftn(white) * amp))
    g -= g.mean()
    s = g.std()
    if s > 0:
        g *= sigma / s
    return g


def diffusion_field(n, sigma, corr_len, seed):
    """exp(g) on an n^3 grid, g the Gaussian random field of diffusion3d."""
    rng = np.random.default_rng(seed)
    return np.exp(gaussian_random_field((n, n, n), sigma, corr_len, rng))


class Diffusion7Family:
    """Many 7-point matrices on one n^3 grid: the pattern (ptr, index) is
    built once and `values(coeff)` returns the value array of diffusion3d for
    a new coefficient field, in the same order."""

    def __init__(self, n):
        self.n = n
        A = diffusion3d(n, stencil=7, coeff=np.ones((n, n, n)))
        self.ptr, self.index, self.N = A.ptr, A.index, A.N
        rows = A.rows().astype(np.int64)
        self._rows, self._cols = rows, A.index.astype(np.int64)
        self._diag = rows == self._cols
        # Dirichlet ghost faces per row: 6 minus the number of neighbours.
        self._ghost = 6 - (np.diff(A.ptr) - 1)

    def values(self, coeff):
        k = coeff.ravel().astype(np.float64)
        ki, kj = k[self._rows], k[self._cols]
        off = -2.0 * ki * kj / (ki + kj)
        val = np.where(self._diag, 0.0, off)
        diag = -np.bincount(self._rows, weights=val, minlength=self.N) + self._ghost * k
        val[self._diag] = diag
        return val

    def matrix(self, coeff):
        return Crs(self.N, self.ptr, self.index, self.values(coeff))


def diffusion3d(n, stencil=7, sigma=1.0, corr_len=8.0, seed=0, coeff=None):
    """Variable-coefficient diffusion on an n^3 grid (see module docstring)."""
    shape = (n, n, n)
    if coeff is None:
        rng = np.random.default_rng(seed)
        coeff = np.exp(gaussian_random_field(shape, sigma, corr_len, rng))
    kap = coeff.ravel().astype(np.float64)
    if stencil == 7:
        offs = [(-1, 0, 0), (0, -1, 0), (0, 0, -1), (0, 0, 0), (0, 0, 1), (0, 1, 0), (1, 0, 0)]
    elif stencil == 27:
        offs = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    else:
        raise ValueError("stencil must be 7 or 27")
    N = n ** 3
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    z, y, x = z.ravel(), y.ravel(), x.ravel()
    lin = np.arange(N, dtype=np.int64)
    couplings = []
    diag = np.zeros(N)
    for (dz, dy, dx) in offs:
        if (dz, dy, dx) == (0, 0, 0):
            couplings.append(None)
            continue
        w = 1.0 / (abs(dz) + abs(dy) + abs(dx))
        zz, yy, xx = z + dz, y + dy, x + dx
        m = (zz >= 0) & (zz < n) & (yy >= 0) & (yy < n) & (xx >= 0) & (xx < n)
        nb = np.where(m, lin + (dz * n + dy) * n + dx, lin)
        kj = kap[nb]
        hm = 2.0 * kap * kj / (kap + kj)
        c = np.where(m, w * hm, w * kap)
        diag += c
        couplings.append(-w * hm)
    return _stencil_crs(shape, offs, lambda k: couplings[k], diag)


# ---------------------------------------------------------------------------
# Random geometric graph Laplacian

def _morton_order(pts, bits=10):
    """Permutation that sorts points in [0,1)^3 along a Z-order (Morton)
    curve of 2^bits cells per axis."""
    q = np.minimum((pts * (1 << bits)).astype(np.uint64), (1 << bits) - 1)
    code = np.zeros(len(pts), np.uint64)
    for b in range(bits):
        for a in range(3):
            code |= ((q[:, a] >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + a)
    return np.argsort(code, kind="stable")


def geometric_graph(npts, mean_degree=12.0, seed=0, shift=1e-3):
    """Random geometric graph Laplacian: npts uniform points in the unit
    cube, numbered along a Morton curve (neighbouring points get nearby
    numbers), edges between points closer than r with r set for the mean
    degree, weights exp(-d/r), plus shift * I."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    pts = rng.random((npts, 3))
    pts = pts[_morton_order(pts)]
    r = (3.0 * mean_degree / (4.0 * np.pi * npts)) ** (1.0 / 3.0)
    pairs = cKDTree(pts).query_pairs(r, output_type="ndarray").astype(np.int64)
    i, j = pairs[:, 0], pairs[:, 1]
    d = np.linalg.norm(pts[i] - pts[j], axis=1)
    w = np.exp(-d / r)
    deg = np.bincount(i, weights=w, minlength=npts) + np.bincount(j, weights=w, minlength=npts)
    diag_idx = np.arange(npts, dtype=np.int64)
    rows = np.concatenate([i, j, diag_idx])
    cols = np.concatenate([j, i, diag_idx])
    vals = np.concatenate([-w, -w, deg + shift])
    return crs_from_unsorted(npts, rows, cols, vals)


# ---------------------------------------------------------------------------
# Format conversions with the reference's layouts and orders

def to_ell(A: Crs):
    """Column-major ELL (Matrix.cpp:339-361): element (i, j) at j*N + i, row i
    keeps its CRS order. Padding slots hold index 0 / value 0."""
    lengths = np.diff(A.ptr).astype(np.int32)
    max_nz = int(lengths.max()) if A.N else 0
    index = np.zeros(max_nz * A.N, dtype=np.int32)
    data = np.zeros(max_nz * A.N, dtype=np.float64)
    rows = A.rows().astype(np.int64)
    slot = np.arange(A.nz, dtype=np.int64) - A.ptr[:-1].astype(np.int64)[rows]
    k = slot * A.N + rows
    index[k] = A.index
    data[k] = A.value
    return max_nz, lengths, index, data


def symmetric_file_coo(A: Crs):
    """The COO arrays the reference's reader (Matrix.cpp:80-103) produces from
    the symmetric MatrixMarket file of A's lower triangle written row by row:
    entry (i, j, v) with j <= i, followed by its mirror (j, i, v) if j < i."""
    rows = A.rows()
    low = A.index <= rows
    r, c, v = rows[low], A.index[low], A.value[low]
    off = r != c
    reps = 1 + off.astype(np.int64)
    n = int(reps.sum())
    I = np.empty(n, dtype=np.int32)
    J = np.empty(n, dtype=np.int32)
    V = np.empty(n, dtype=np.float64)
    start = np.zeros(len(r), dtype=np.int64)
    np.cumsum(reps[:-1], out=start[1:])
    I[start], J[start], V[start] = r, c, v
    s2 = start[off] + 1
    I[s2], J[s2], V[s2] = c[off], r[off], v[off]
    return I, J, V


def write_mtx_symmetric(path, A: Crs):
    """Writes A's lower triangle as `matrix coordinate real symmetric` with 17
    significant digits (exact round trip), through libcgb200's parallel
    writer."""
    from ._lib import mtx_write_symmetric_crs
    mtx_write_symmetric_crs(path, A.ptr, A.index, A.value)


def write_mtx_symmetric_py(path, A: Crs):
    """Pure-Python writer (small matrices; no native library needed)."""
    rows = A.rows()
    low = A.index <= rows
    r, c, v = rows[low] + 1, A.index[low] + 1, A.value[low]
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n")
        f.write(f"{A.N} {A.N} {len(r)}\n")
        f.writelines(f"{a} {b} {x!r}\n" if False else "%d %d %.17g\n" % (a, b, x)
                     for a, b, x in zip(r.tolist(), c.tolist(), v.tolist()))


def rhs_for(A: Crs, seed=0):
    """b = A x* with x* ~ U[-1, 1] from `seed`; returns (b, x*)."""
    xs = np.random.default_rng(seed).uniform(-1.0, 1.0, A.N)
    return A.matvec(xs), xs


def rhs_ones(A: Crs):
    """k = A * 1 summed in CRS order, as CG::init does in COO order
    (CG.cpp:256-261)."""
    return A.matvec(np.ones(A.N))
