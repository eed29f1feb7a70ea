"""Parity of the plain FP64 path with the reference's own CG at the benchmark
sizes, where the kernels take the code paths that small matrices never reach:
full 256-row staged CRS tiles and the tile-major ELL at 160^3, the per-warp
staged CRS (k_crs_warp) for the 27-point rows at 128^3, and irregular rows of
1 to 40 entries on the 2M-point geometric graph.

Each case runs the reference's CG::solve (CG.cpp:284-385) through its OpenMP
backend (oracle/_ref/ref_harness_omp, built from the unmodified sources) on
the same MatrixMarket file with its own right-hand side k = A * 1
(CG.cpp:256-261), and this library's FP64 solve on the same matrix and k.
Bar: iterations within 2 %, ||x - x_ref|| / ||x_ref|| <= 1e-8, and the
reference's check (|x_i - 1| <= CG_CHECK_TOLERANCE = 1e-5, CG.cpp:387-408)
gives the same verdict on both solutions.

The matrices are the benchmark's seeded synthetic families (no dataset).
"""
import os
import tempfile

import numpy as np
import pytest

import cgxx_b200 as cg
from cgxx_b200 import generators as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-9
MAX_ITER = 5000
CHECK_TOL = 1e-5  # the reference's default CG_CHECK_TOLERANCE (CG.h:71)

CONFIGS = {
    # 7-point diffusion, 160^3, exp(GRF) coefficients: the benchmark matrix.
    "diffusion7_160": lambda: G.diffusion3d(160, 7, sigma=1.0, corr_len=8.0, seed=2024),
    # 27-point diffusion, 128^3 (rows of 27 entries overflow 256-row tiles).
    "diffusion27_128": lambda: G.diffusion3d(128, 27, sigma=1.0, corr_len=8.0, seed=2024),
    # Random geometric graph Laplacian, 2M points, mean degree 12.
    "graph_2M": lambda: G.geometric_graph(2_000_000, mean_degree=12.0, seed=2024),
}

_cache = {}


def _workload(name):
    """Matrix, its MatrixMarket file, and the reference's k = A * 1 summed in
    file order (the COO order CG::init uses)."""
    if name not in _cache:
        A = CONFIGS[name]()
        d = tempfile.mkdtemp(prefix="cgx_parity_")
        path = os.path.join(d, name + ".mtx")
        G.write_mtx_symmetric(path, A)
        I, J, V = G.symmetric_file_coo(A)
        k = O.rhs_ones(A.N, I, J, V)
        _cache[name] = (A, path, k)
    return _cache[name]


def _reference(path, fmt):
    if O.ref_binary("ref_harness_omp") is None:
        pytest.fail("oracle/_ref/ref_harness_omp is not built")
    env = {"CG_MAX_ITER": str(MAX_ITER), "CG_TOLERANCE": repr(TOL),
           "CG_MATRIX_FORMAT": fmt, "CG_PRECONDITIONER": "jacobi",
           "OMP_NUM_THREADS": str(len(os.sched_getaffinity(0)))}
    summ, x = O.run_ref_harness(path, backend="omp", env=env)
    return summ, x


def _ours(A, k, fmt):
    with cg.Handle(0) as h:
        if fmt == "CRS":
            h.upload_crs(A.ptr, A.index, A.value)
        else:
            m, l, i, d = G.to_ell(A)
            h.upload_ell(A.N, A.nz, m, l, i, d)
        h.upload_jacobi(1.0 / A.diagonal())
        h.set_vector("K", k)
        h.fill_vector("X", 0.0)
        res = h.solve(max_iterations=MAX_ITER, tolerance=TOL)
        return res, h.get_vector("X")


@pytest.mark.parametrize("name,fmt", [("diffusion7_160", "CRS"), ("diffusion7_160", "ELL"),
                                      ("diffusion27_128", "CRS"), ("graph_2M", "CRS")])
def test_fp64_solve_matches_reference_at_benchmark_size(name, fmt):
    A, path, k = _workload(name)
    summ, x_ref = _reference(path, fmt)
    res, x = _ours(A, k, fmt)
    it_ref = summ["iterations"][-1]
    assert res["converged"] == 1
    assert abs(res["iterations"] - it_ref) <= 0.02 * it_ref, (res["iterations"], it_ref)
    relx = np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref)
    assert relx <= 1e-8, relx
    ref_ok = summ["correct"] == 1
    ours_bad = int(np.sum(np.abs(x - 1.0) > CHECK_TOL))
    assert (ours_bad == 0) == ref_ok, (ours_bad, summ["incorrect"])
    assert ref_ok, f"the reference's own check failed: {summ['incorrect']}"


def test_band_inner_product_at_benchmark_size():
    """The FP32 symmetric-band product that the mixed and learned paths time
    at 160^3 (offsets 0, 1, 160, 25600), against the FP64 product of the same
    FP32 x: within 4e-6 of sum_j |a_ij x_j| per row."""
    A, _, _ = _workload("diffusion7_160")
    x = np.random.default_rng(12).standard_normal(A.N).astype(np.float32)
    x[:3] = 1e3
    x[-3:] = -1e3
    with cg.Handle(0) as h:
        h.upload_crs(A.ptr, A.index, A.value)
        h.upload_jacobi(1.0 / A.diagonal())
        y = h.inner_matvec(x)
        assert h.inner_band() == [0, 1, 160, 160 * 160]
    xd = x.astype(np.float64)
    ref = A.matvec(xd)
    absA = G.Crs(A.N, A.ptr, A.index, np.abs(A.value))
    bound = 4e-6 * absA.matvec(np.abs(xd)) + 1e-30
    assert np.all(np.abs(y.astype(np.float64) - ref) <= bound)


@pytest.mark.parametrize("name", ["diffusion7_160", "diffusion27_128"])
@pytest.mark.parametrize("learned", [False, True])
def test_mixed_paths_at_benchmark_size(name, learned):
    """The mixed and learned solves on the benchmark matrices (7-point
    160^3: the split persistent kernel on the band form with its L2 prefetch
    of the band values; 27-point 128^3: the split persistent kernel on
    SELL-U; with the fused form and the per-iteration kernels for
    comparison): every loop mode reaches the FP64 1e-9 true residual with
    inner iteration counts within 2 %, and its solution is within 1e-6 of
    the FP64 solve's (the plain path, the reference's algorithm)."""
    from cgxx_b200 import learned as LRN
    A, _, k = _workload(name)
    with cg.Handle(0) as h:
        h.upload_crs(A.ptr, A.index, A.value)
        h.upload_jacobi(1.0 / A.diagonal())
        h.set_vector("K", k)
        h.fill_vector("X", 0.0)
        r64 = h.solve(max_iterations=MAX_ITER, tolerance=TOL)
        x64 = h.get_vector("X")
        assert r64["converged"] == 1
        pc = cg.PRECOND_JACOBI
        if learned:
            net = cg.Gnn(0, LRN.load_weights(LRN.DEFAULT_WEIGHTS)[0])
            h.learned_setup()
            h.learned_factor(net, 1e-4)
            net.close()
            pc = cg.PRECOND_LEARNED
        out = {}
        for loop in (cg.LOOP_GRAPH, cg.LOOP_PERSISTENT, cg.LOOP_KERNELS):
            h.fill_vector("X", 0.0)
            r = h.solve(max_iterations=20000, tolerance=TOL, precision=cg.PRECISION_MIXED,
                        preconditioner=pc, loop=loop)
            x = h.get_vector("X")
            assert r["converged"] == 1 and r["fell_back"] == 0, (loop, r)
            assert np.linalg.norm(k - A.matvec(x)) / np.linalg.norm(k) <= TOL, loop
            assert np.linalg.norm(x - x64) / np.linalg.norm(x64) <= 1e-6, loop
            out[loop] = r
    band = name == "diffusion7_160"
    assert out[cg.LOOP_GRAPH]["inner_form"] == (2 if band else 3)
    assert out[cg.LOOP_PERSISTENT]["inner_form"] == (1 if band else 0)
    ik = out[cg.LOOP_KERNELS]["iterations"]
    for loop in (cg.LOOP_GRAPH, cg.LOOP_PERSISTENT):
        assert abs(out[loop]["iterations"] - ik) <= 0.02 * ik + 2, (loop, out[loop], ik)
