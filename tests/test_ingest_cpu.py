"""The device COO conversion (cgxx_b200/csrc/ingest.cuh) restated in numpy.

The device sorts (row, entry) pairs by row with an LSD radix sort: per
4096-entry tile a digit histogram, an exclusive scan over (digit, tile),
then a scatter in 16 rounds of 256 entries in which lanes with the same
digit are ranked within their warp and warps are taken in order. This file
restates those steps index by index and checks, without a GPU, that every
write lands inside its buffer and that the result is the stable order by
row (numpy's stable argsort) -- the order the reference's CRS and ELL
conversion (Matrix.cpp:203-228, 339-361) produce -- and that the row
pointers built from the sorted rows are the reference's.
"""
import numpy as np
import pytest

TILE, RADIX, THREADS, WARP = 4096, 256, 256, 32


def sort_hist(keys, shift, ntiles):
    hist = np.zeros(RADIX * ntiles, np.int64)
    for t in range(ntiles):
        d = (keys[t * TILE:(t + 1) * TILE] >> shift) & (RADIX - 1)
        c = np.bincount(d, minlength=RADIX)
        hist[np.arange(RADIX) * ntiles + t] = c
    return hist


def sort_scatter(keys, vals, shift, ntiles, offs):
    n = len(keys)
    kout = np.full(n, -1, np.int64)
    vout = np.full(n, -1, np.int64)
    for t in range(ntiles):
        run = offs[np.arange(RADIX) * ntiles + t].copy()
        for rnd in range(TILE // THREADS):
            i = t * TILE + rnd * THREADS + np.arange(THREADS)
            valid = i < n
            key = np.where(valid, keys[np.minimum(i, n - 1)], 0)
            d = np.where(valid, (key >> shift) & (RADIX - 1), RADIX)
            wcnt = np.zeros((THREADS // WARP, RADIX + 1), np.int64)
            rank = np.zeros(THREADS, np.int64)
            for w in range(THREADS // WARP):
                dw = d[w * WARP:(w + 1) * WARP]
                for lane in range(WARP):  # __match_any_sync + popc(peers & lanes below)
                    rank[w * WARP + lane] = np.sum(dw[:lane] == dw[lane])
                for v in np.unique(dw):
                    wcnt[w, v] = np.sum(dw == v)
            for tid in np.nonzero(valid)[0]:
                w = tid // WARP
                pos = run[d[tid]] + rank[tid] + wcnt[:w, d[tid]].sum()
                assert 0 <= pos < n and kout[pos] == -1  # in bounds, written once
                kout[pos] = key[tid]
                vout[pos] = vals[i[tid]] if vals is not None else i[tid]
            run += wcnt[:, :RADIX].sum(0)
    return kout, vout


def rows_ptr(N, rows):
    nz = len(rows)
    ptr = np.full(N + 1, -1, np.int64)
    for k in range(nz + 1):
        prev = rows[k - 1] if k > 0 else -1
        cur = rows[k] if k < nz else N
        for r in range(prev + 1, cur + 1):
            assert ptr[r] == -1
            ptr[r] = k
    return ptr


def device_sort(N, I):
    nz = len(I)
    ntiles = max(1, (nz + TILE - 1) // TILE)
    bits = 0
    while bits < 31 and ((N - 1) >> bits) != 0:
        bits += 1
    keys, vals = I.astype(np.int64), None
    for p in range(max(1, (bits + 7) // 8)):
        hist = sort_hist(keys, 8 * p, ntiles)
        offs = np.concatenate([[0], np.cumsum(hist)])
        keys, vals = sort_scatter(keys, vals, 8 * p, ntiles, offs)
    return keys, vals


@pytest.mark.parametrize("N,nz,seed", [(1, 5, 0), (7, 300, 1), (300, 5000, 2),
                                       (70000, 9000, 3), (1000, 8193, 4)])
def test_radix_sort_is_the_stable_row_order(N, nz, seed):
    rng = np.random.default_rng(seed)
    # Many repeats per row, rows out of order: stability is visible.
    I = rng.integers(0, N, nz)
    keys, order = device_sort(N, I)
    ref = np.argsort(I, kind="stable")
    assert np.array_equal(order, ref)
    assert np.array_equal(keys, I[ref])
    counts = np.bincount(I, minlength=N)
    assert np.array_equal(rows_ptr(N, keys), np.concatenate([[0], np.cumsum(counts)]))


def test_row_pointers_with_empty_rows():
    rows = np.array([2, 2, 5, 5, 5, 9])
    assert list(rows_ptr(12, rows)) == [0, 0, 0, 2, 2, 2, 5, 5, 5, 5, 6, 6, 6]
    assert list(rows_ptr(4, np.array([], np.int64))) == [0, 0, 0, 0, 0]
