import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available():
    try:
        import cgxx_b200
        return cgxx_b200.device_count() > 0
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    # Tests marked gpu fail loudly (no silent skip) when selected with -m gpu
    # on a machine whose library cannot see a device; under -m "not gpu" they
    # are deselected by the marker expression.
    pass


@pytest.fixture(scope="session")
def handle():
    import cgxx_b200
    h = cgxx_b200.Handle(0)
    yield h
    h.close()


def random_crs(N, min_len=0, max_len=40, seed=0, spd=False):
    """Random sparse matrix with ragged rows (lengths in [min_len, max_len]).
    spd=True: symmetric, strictly diagonally dominant with positive
    diagonal (hence SPD), every row non-empty."""
    from cgxx_b200 import generators as G
    rng = np.random.default_rng(seed)
    if not spd:
        lens = rng.integers(min_len, max_len + 1, N)
        rows = np.repeat(np.arange(N), lens)
        cols = rng.integers(0, N, lens.sum())
        vals = rng.standard_normal(lens.sum())
        return G.crs_from_unsorted(N, rows, cols, vals)
    half = rng.integers(0, max(1, max_len // 2) + 1, N)
    r = np.repeat(np.arange(N), half)
    c = rng.integers(0, N, half.sum())
    keep = r != c
    r, c = r[keep], c[keep]
    w = rng.uniform(0.1, 1.0, len(r))
    rows = np.concatenate([r, c])
    cols = np.concatenate([c, r])
    vals = np.concatenate([-w, -w])
    # merge duplicates
    key = rows.astype(np.int64) * N + cols
    uk, inv = np.unique(key, return_inverse=True)
    v = np.bincount(inv, weights=vals)
    rows, cols = (uk // N).astype(np.int64), (uk % N).astype(np.int64)
    diag = np.bincount(rows, weights=np.abs(v), minlength=N) + rng.uniform(0.5, 2.0, N)
    rows = np.concatenate([rows, np.arange(N)])
    cols = np.concatenate([cols, np.arange(N)])
    vals = np.concatenate([v, diag])
    return G.crs_from_unsorted(N, rows, cols, vals)
