"""cgx_dot_noalloc: the dot product for callers that cannot allocate device
memory (a framework that owns all device memory, a loop that forbids
allocation after start-up). It keeps its scratch in a fixed array inside the
library instead of cudaMalloc'ed memory.

Checked through the C ABI against the existing entry point cgx_dot and the
CPU oracle's FP64 dot product, on two calls in a row (the second call starts
from the scratch contents that the first left behind). The test buffers are torch tensors owned by the test;
the entry point itself allocates nothing. This file is collected last so
that a run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import cgxx_b200 as cg
from cgxx_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_TOL = 1e-13  # the dot-product tolerance of the other kernel tests


def _reference_dot(a, b, device=0):
    """cgx_dot (the handle-based entry point) on the same vectors."""
    n = len(a)
    with cg.Handle(device) as h:
        ptr = np.arange(n + 1, dtype=np.int32)  # identity pattern, N = n
        h.upload_crs(ptr, np.arange(n, dtype=np.int32), np.ones(n))
        h.set_vector("P", a)
        h.set_vector("Q", b)
        return h.dot("P", "Q")


def _noalloc_dot(a_dev, b_dev, n, out_dev, stream):
    lib = cg.load()
    _lib.check(lib.cgx_dot_noalloc(C.c_void_p(a_dev.data_ptr()),
                                   C.c_void_p(b_dev.data_ptr()), n,
                                   C.c_void_p(out_dev.data_ptr()),
                                   C.c_void_p(stream or None)))


def _check_twice(n, device):
    import torch
    rng = np.random.default_rng(n)
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    ref = _reference_dot(a, b, device)
    oracle = O.dot(a, b)
    torch.cuda.set_device(device)
    a_dev = torch.from_numpy(a).cuda(device)
    b_dev = torch.from_numpy(b).cuda(device)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device=f"cuda:{device}")
    stream = torch.cuda.current_stream(device).cuda_stream
    _noalloc_dot(a_dev, b_dev, n, out[0:1], stream)
    _noalloc_dot(a_dev, b_dev, n, out[1:2], stream)
    torch.cuda.synchronize(device)
    got = out.cpu().numpy()
    scale = max(1.0, float(np.abs(a) @ np.abs(b)))
    for g in got:
        assert abs(g - ref) <= REL_TOL * scale, (g, ref)
        assert abs(g - oracle) <= REL_TOL * scale, (g, oracle)
    assert got[0] == got[1]  # deterministic across calls


@pytest.mark.parametrize("n", [1, 4095, 4096, 1_000_003])
def test_noalloc_dot_matches_cgx_dot_twice(n):
    _check_twice(n, 0)


def test_noalloc_dot_on_second_device():
    """The scratch address is looked up per device: a call on device 1 must
    use device 1's copy of the array."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs a second GPU")
    try:
        _check_twice(1_000_003, 1)
    finally:
        torch.cuda.set_device(0)


def test_noalloc_dot_rejects_oversize_and_bad_arguments():
    import torch
    lib = cg.load()
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = C.c_void_p(x.data_ptr())
    too_big = 268_435_456 + 1
    st = lib.cgx_dot_noalloc(p, p, too_big, p, None)
    assert st == 1
    assert b"exceeds the maximum" in lib.cgx_last_error()
    assert lib.cgx_dot_noalloc(p, p, -1, p, None) == 1
    assert lib.cgx_dot_noalloc(p, p, 4, None, None) == 1
