#!/usr/bin/env python3
"""Benchmark: milliseconds to a 1e-9 relative residual on one B200.

Workload (default): 3-D 7-point variable-coefficient diffusion on a 160^3
grid (N = 4,096,000, nnz = 28,518,400), face coefficients exp(g) with g a
seeded Gaussian random field (sigma 1, correlation length 8 cells), FP64
values in CRS, Jacobi preconditioner, b = A x* with x* ~ U[-1, 1], tolerance
1e-9. Synthetic and seeded: the reference ships no matrices.

One step = one complete solve from x0 = 0 to the tolerance, inputs resident
in device memory. The matrix (342 MB) is larger than the 126 MB L2, so no
flush is needed between steps.

Paths (--path):
  learned (default) = FP32 inner PCG with the learned factor M^-1 = G G^T +
      eps D^-1 inside FP64 iterative refinement, stopping on the FP64 true
      residual; every step includes the scaled-graph set-up and the network
      inference that produce G (the weights come from --weights, else the
      untrained initialisation, and the line says which);
  mixed = the same refinement with FP32 Jacobi-PCG inside;
  plain = FP64 Jacobi-PCG, the reference's arithmetic.
`value` is the time of the path named in config.path; the other two paths'
times are reported next to it under `paths`.

--impl reference runs the reference's own OpenMP CG (oracle/_ref, built from
the unmodified reference sources) on the box's host cores instead.

Prints one JSON line (rank 0).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "ms to 1e-9 rel. residual: learned-precond mixed CG vs plain FP64 Jacobi CG"
CACHE = os.path.join(tempfile.gettempdir(), "cgxx_b200_bench")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=160, help="grid edge (default 160)")
    ap.add_argument("--stencil", type=int, choices=[7, 27], default=7)
    ap.add_argument("--graph", type=int, default=0,
                    help="points of a random geometric graph instead of the grid")
    ap.add_argument("--path", choices=["learned", "mixed", "plain"], default="learned")
    ap.add_argument("--weights", default=None,
                    help="weight file of the learned preconditioner (default: the "
                         "weights trained on the workload's family, diffusion7.gnn for the "
                         "grids and graph12.gnn for --graph); 'init' for the untrained network")
    ap.add_argument("--eps", type=float, default=1e-4)
    ap.add_argument("--max-iter", type=int, default=5000)
    ap.add_argument("--tol", type=float, default=1e-9)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--loop", choices=["graph", "chunked", "kernels", "persistent", "split"],
                    default="graph",
                    help="device loop of the timed solves (graph: the default, which runs "
                         "the mixed paths' inner solves as persistent launches where they "
                         "apply; profilers cannot see inside a graph with a while node)")
    ap.add_argument("--quick", action="store_true",
                    help="timed solves only (for profiler runs): no other path, "
                         "no per-kernel pass, no e2e, no CPU baseline")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# Distributed plumbing (one process per GPU; replicas, no data exchange)

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, v):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v)], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# Workload

def workload(n, stencil=7, graph=0):
    """The 3D diffusion matrix on an n^3 grid (7- or 27-point stencil), or
    with graph > 0 the random geometric graph Laplacian on that many points,
    and b = A x* for a seeded x*."""
    from cgxx_b200 import generators as G
    if graph:
        A = G.geometric_graph(graph, mean_degree=12.0, seed=2024)
    else:
        A = G.diffusion3d(n, stencil=stencil, sigma=1.0, corr_len=8.0, seed=2024)
    b, xs = G.rhs_for(A, seed=7)
    return A, b, xs


def workload_name(args):
    if args.graph:
        return f"geometric-graph-{args.graph}-deg12"
    return f"diffusion3d-{args.stencil}pt-{args.n}^3"


def workload_config(args, A):
    field = ("random geometric graph, uniform points in the unit cube, mean degree 12, "
             "w = exp(-d/r), L + 1e-3 I, seed 2024" if args.graph else
             "exp(GRF sigma=1, corr_len=8 cells), seed 2024")
    return {
        "workload": workload_name(args),
        "N": A.N, "nnz": A.nz, "format": "CRS", "preconditioner": "jacobi",
        "field": field,
        "rhs": "A x*, x* ~ U[-1,1] seed 7", "tolerance": args.tol,
        "max_iterations": args.max_iter, "l2": "inputs larger than L2 (no flush)",
        "parallelism": "replicas" if args.gpus > 1 else "single GPU",
    }


# ---------------------------------------------------------------------------
# Clocks during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ---------------------------------------------------------------------------
# Reference CPU implementation (oracle/_ref, built from the reference sources)

def mtx_cache_path(A, name, native=False):
    """The workload as a symmetric MatrixMarket file (cached per machine).
    native=True writes it with libcgb200's parallel writer (our arm, which
    loads that library anyway); the reference arm uses the pure-Python
    writer and maps none of this project's native libraries."""
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, name.replace("^", "_") + ".mtx")
    if not os.path.exists(path):
        tmp = path + f".tmp{os.getpid()}"
        from cgxx_b200 import generators as G
        if native:
            G.write_mtx_symmetric(tmp, A)
        else:
            G.write_mtx_symmetric_py(tmp, A)
        os.replace(tmp, path)
    return path


def run_reference(A, b, name, reps, max_iter, tol, threads, backend="omp", native=False):
    """Runs the reference's OpenMP (or serial) CG in-process harness on the
    workload with right-hand side b. Returns the list of per-repetition solve
    times (s) and the iteration counts."""
    from oracle import oracle as O
    path = mtx_cache_path(A, name, native)
    env = {"CG_MAX_ITER": str(max_iter), "CG_TOLERANCE": repr(tol),
           "CG_MATRIX_FORMAT": "CRS", "CG_PRECONDITIONER": "jacobi"}
    if backend == "omp":
        env.update({"OMP_NUM_THREADS": str(threads), "OMP_PROC_BIND": "spread"})
    summ, x = O.run_ref_harness(path, rhs=b, backend=backend, reps=reps, env=env)
    return summ["solve_time"], summ["iterations"], x


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_arm(args, world, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    if O.ref_binary("ref_harness_omp") is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/ref_harness_omp was not built (reference sources absent)"}))
        return
    A, b, _ = workload(args.n, args.stencil, args.graph)
    threads = host_threads()
    # Warm-up repetitions are full solves; they also give the iteration count
    # and the time of one full solve.
    wt, witers, _ = run_reference(A, b, workload_name(args), max(1, args.warmup), args.max_iter,
                                  args.tol, threads)
    full_iters, full_s = witers[-1], min(wt)
    if full_s * args.steps <= 240.0:
        times, iters, _ = run_reference(A, b, workload_name(args), args.steps, args.max_iter, args.tol,
                                        threads)
        ms = 1e3 * sum(times) / len(times)
        sample = (f"{args.steps} full solves ({iters[-1]} iterations) by the reference's "
                  f"CGOpenMP, OMP_NUM_THREADS={threads}")
    else:
        # Bounded sample: each step runs `cap` iterations; the time is scaled
        # to the full iteration count.
        cap = max(10, int(full_iters * 240.0 / (full_s * args.steps)))
        times, iters, _ = run_reference(A, b, workload_name(args), args.steps, cap, args.tol, threads)
        ms = 1e3 * (sum(times) / len(times)) * full_iters / iters[-1]
        sample = (f"{args.steps} solves capped at {iters[-1]} iterations (CG_MAX_ITER), "
                  f"scaled to the full {full_iters}; CGOpenMP, OMP_NUM_THREADS={threads}")
    iters = [full_iters]
    line = {
        "metric": METRIC, "value": ms, "unit": "ms", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, A),
        "path": "reference OpenMP Jacobi-CG (CRS)",
        "iterations": iters[-1],
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# Our arm

def read_traffic_profile(name, args):
    """ncu DRAM traffic per launch committed under profiles/ for the default
    workload (7-point 160^3); None for other workloads."""
    if workload_name(args) != "diffusion3d-7pt-160^3":
        return None
    return _read_profile(name)


def _read_profile(name):
    p = os.path.join(REPO, "profiles", name)
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return None


# Algorithmic bytes per row of one inner iteration of the persistent inner
# solves (persist.cuh), full and for the last iteration of a launch (which
# stops after its residual test): FP32 vectors 4 bytes, U 16, the factor 8.
#   split learned: q=Ap 24 | r, d 24 | y=G^T r 16 | z 24 | p 12
#   split Jacobi:  q=Ap 24 | r, d, <r,Cr> 28 | p = C r + b p 16
#   fused learned: p, d, q 40 | r, y 24 | z 24
#   fused Jacobi:  p, d, q 40 | r, z 20
PERSIST_BYTES = {(2, True): (100, 48), (2, False): (68, 52),
                 (1, True): (88, 64), (1, False): (60, 60)}
# The learned split form on grids of at least 3M rows (its L2-prefetch
# variant) applies d += a p in the direction phase, reading p once.
PERSIST_DEFER_MIN_ROWS = 3_000_000
PERSIST_BYTES_DEFERRED = {(2, True): (96, 36)}
PERSIST_KERNEL = {(2, True): "k_inner_persist_split<learned>", (2, False): "k_inner_persist_split<Jacobi>",
                  (1, True): "k_inner_persist<learned>", (1, False): "k_inner_persist<Jacobi>"}


def persist_roofline(args, results, N, peak, peak_kind):
    """Roofline of the persistent inner-solve launches of the timed solves:
    their algorithmic bytes over their device time (CUDA events around each
    launch, recorded by the library on its stream)."""
    if args.path == "plain" or not results or results[-1]["inner_form"] == 0:
        return None
    form = results[-1]["inner_form"]
    if (form, args.path == "learned") not in PERSIST_BYTES:
        return None  # the SELL-U form: its bytes depend on the slot counts
    key = (form, args.path == "learned")
    full, last = (PERSIST_BYTES_DEFERRED[key] if key in PERSIST_BYTES_DEFERRED
                  and N >= PERSIST_DEFER_MIN_ROWS else PERSIST_BYTES[key])
    bytes_, ms, launches, its = 0, 0.0, 0, 0
    for r in results:
        if r["fell_back"] or r["inner_launches"] == 0:
            continue
        bytes_ += (r["iterations"] * full - r["inner_launches"] * (full - last)) * N
        ms += r["inner_ms"]
        launches += r["inner_launches"]
        its += r["iterations"]
    if launches == 0 or ms <= 0:
        return None
    out = {"bound": "hbm", "achieved": bytes_ / (ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
           "kernel": PERSIST_KERNEL[key] + ": one inner solve per launch",
           "launch_us": 1e3 * ms / launches, "launches": launches,
           "iterations_per_launch": its / launches,
           "algorithmic_bytes": bytes_ / launches, "peak_kind": peak_kind}
    out["frac"] = out["achieved"] / peak
    prof = read_traffic_profile(f"persist_{'split' if form == 2 else 'fused'}_"
                                f"{args.path}_diffusion7_160.json", args)
    per_it = prof.get("dram_bytes_per_iteration") if prof else None
    out["traffic"] = per_it * its / launches if per_it else None
    return out


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


LOOPS = {"graph": 0, "chunked": 1, "kernels": 2, "persistent": 3, "split": 4}
PATHS = ("learned", "mixed", "plain")


def solve_opts(cg, args, path, loop=None):
    pc = {"learned": cg.PRECOND_LEARNED}.get(path, cg.PRECOND_JACOBI)
    prec = cg.PRECISION_FP64 if path == "plain" else cg.PRECISION_MIXED
    return cg.default_options(
        max_iterations=args.max_iter, tolerance=args.tol, preconditioner=pc,
        precision=prec, loop=LOOPS[args.loop] if loop is None else loop,
        inner_tolerance=3e-6, max_outer=30)


def load_network(args):
    """Parameters of the learned preconditioner: the trained weight file if
    present, else the untrained initialisation (reported as such)."""
    from cgxx_b200 import learned as LRN
    path = args.weights
    if path is None:
        path = os.path.join(REPO, "cgxx_b200", "weights",
                            "graph12.gnn" if args.graph else "diffusion7.gnn")
    if path == "init":
        return LRN.init_params(0), {"weights": "untrained initialisation (--weights init)"}
    if path and os.path.exists(path):
        params, head = LRN.load_weights(path)
        return params, {"weights": os.path.relpath(path, REPO),
                        "trained_steps": head.get("steps"),
                        "config_sha256": head.get("config_sha256")}
    return LRN.init_params(0), {"weights": "untrained initialisation (no weight file)"}


def our_arm(args, world, rank, local):
    import torch

    import cgxx_b200 as cg

    A, b, xs = workload(args.n, args.stencil, args.graph)
    Cd = 1.0 / A.diagonal()
    N, nnz = A.N, A.nz
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream()
    h = cg.Handle(dev)
    h.set_stream(stream.cuda_stream)
    h.upload_crs(A.ptr, A.index, A.value)
    h.upload_jacobi(Cd)
    h.set_vector("K", b)
    params, net_info = load_network(args)
    net = cg.Gnn(dev, params)

    def one_solve(path, loop=None):
        """One complete solve from x0 = 0. The learned path includes, every
        step, the scaled-graph set-up and the network inference of G."""
        h.fill_vector("X", 0.0)
        if path == "learned":
            h.learned_setup()
            h.learned_factor(net, args.eps)
        return h.solve(solve_opts(cg, args, path, loop))

    # Warm-up (also builds the CUDA graphs of every path).
    for _ in range(args.warmup):
        one_solve(args.path)
    others = [p for p in PATHS if p != args.path]
    if not args.quick:
        for p in others:
            one_solve(p)

    # Timed region: K complete solves, device-timed with CUDA events on the
    # stream the library launches on, bracketed by barrier + synchronize.
    results = []
    with ClockSampler(dev) as clk:
        barrier(world)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            results.append(one_solve(args.path))
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(world, ms)
    clocks = clk.summary()
    res = results[-1]
    x = h.get_vector("X")
    true_rel = float(np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b))
    err_vs_exact = float(np.linalg.norm(x - xs) / np.linalg.norm(xs))
    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": ms, "unit": "ms", "quick": True,
                              "path": args.path, "iterations": res["iterations"],
                              "true_residual": true_rel, "config": workload_config(args, A),
                              "clocks": clocks}))
        h.close()
        return

    # The other paths, side by side (median of two solves each; the learned
    # path's time includes its set-up and inference).
    def timed(path):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = one_solve(path)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), r

    solutions = {args.path: x}

    def accuracy(p):
        """FP64 true relative residual of the current X, and its relative
        error against the exact solution x* of b = A x* (FP64, on the CPU)."""
        xv = h.get_vector("X")
        solutions[p] = xv
        return {"true_residual": float(np.linalg.norm(b - A.matvec(xv)) / np.linalg.norm(b)),
                "rel_error_vs_exact": float(np.linalg.norm(xv - xs) / np.linalg.norm(xs))}

    side = {args.path: {"ms": ms, "iterations": res["iterations"],
                        "outer_iterations": res["outer_iterations"],
                        "fell_back": bool(res["fell_back"]),
                        "true_residual": true_rel, "rel_error_vs_exact": err_vs_exact}}
    for p in others:
        runs = [timed(p) for _ in range(2)]
        side[p] = {"ms": statistics.median(t for t, _ in runs),
                   "iterations": runs[-1][1]["iterations"],
                   "outer_iterations": runs[-1][1]["outer_iterations"],
                   "fell_back": bool(runs[-1][1]["fell_back"])}
        side[p].update(accuracy(p))
    # Every path's error against the FP64 solve of the plain path (the
    # reference's algorithm, bit-identical to its serial kernels).
    xp = solutions["plain"]
    for p, xv in solutions.items():
        side[p]["rel_error_vs_fp64_solve"] = float(np.linalg.norm(xv - xp) / np.linalg.norm(xp))
    # Learned path: network set-up + inference alone.
    fe0 = torch.cuda.Event(enable_timing=True)
    fe1 = torch.cuda.Event(enable_timing=True)
    fe0.record(stream)
    h.learned_setup()
    h.learned_factor(net, args.eps)
    fe1.record(stream)
    torch.cuda.synchronize()
    side["learned"]["factor_ms"] = fe0.elapsed_time(fe1)

    # Per-launch kernel times (roofline), one solve per path with every fused
    # kernel bracketed by CUDA events.
    kern = {}
    for p in ("plain", args.path) if args.path != "plain" else ("plain",):
        r = one_solve(p, loop=cg.LOOP_KERNELS)
        kern[p] = {"spmv_us": 1e3 * r["spmv_ms"] / max(1, r["spmv_launches"]),
                   "update_us": 1e3 * r["update_ms"] / max(1, r["update_launches"]),
                   "direction_us": 1e3 * r["direction_ms"] / max(1, r["direction_launches"]),
                   "launches": r["spmv_launches"]}
    # The dominant kernel alone: 20 back-to-back launches of the solver's
    # fused SpMV captured in a CUDA graph and timed with CUDA events on the
    # handle's stream (the per-kernel mode above brackets every launch with
    # events, which adds a few microseconds to each segment).
    spmv_us = {"plain": h.time_spmv(cg.PRECISION_FP64, reps=20)}
    if args.path != "plain":
        spmv_us[args.path] = h.time_spmv(cg.PRECISION_MIXED, reps=20)
    peak, peak_kind = peaks()
    fp64_spmv_bytes = 12 * nnz + 4 * (N + 1) + 16 * N  # values+cols, ptr, p once, q
    fp32_spmv_bytes = 8 * nnz + 4 * (N + 1) + 8 * N  # FP32 CRS
    plain_iter_bytes = fp64_spmv_bytes + 32 * N + 48 * N
    kp = kern["plain"]
    plain_iter_us = kp["spmv_us"] + kp["update_us"] + kp["direction_us"]
    fp64_roof = {"bound": "hbm", "achieved": fp64_spmv_bytes / (spmv_us["plain"] * 1e-6) / 1e9,
                 "launch_us": spmv_us["plain"],
                 "peak": peak, "unit": "GB/s",
                 "kernel": "k_crs<double, OpPcgQ>: q = A p fused with <p,q> (FP64 CRS)",
                 "algorithmic_bytes": fp64_spmv_bytes, "peak_kind": peak_kind}
    fp64_roof["frac"] = fp64_roof["achieved"] / peak
    prof = read_traffic_profile("spmv_crs_fp64_diffusion7_160.json", args)
    fp64_roof["traffic"] = prof.get("dram_bytes_per_launch") if prof else None
    inner_roof = None
    if args.path != "plain":
        kk = kern[args.path]
        slots, uniform, slices = h.inner_layout()
        band = h.inner_band()
        prof_name = None  # ncu traffic is committed for the band form only
        if band:
            # Symmetric band: 4 FP32 values per row (diagonal and upper half;
            # the lower half is read from the rows above, in L1/L2), p once,
            # q written.
            fp32_spmv_bytes = 16 * N + 8 * N
            kname = (f"k_band<4, OpInnerQ>: q = A p fused with <p,q> (FP32 symmetric band, "
                     f"offsets {band})")
            prof_name = "spmv_band_fp32_diffusion7_160.json"
        elif slots:
            # SELL-U: FP32 values, 16-byte slice descriptors, p once, q
            # written (a uniform slice carries no per-entry index).
            fp32_spmv_bytes = 4 * nnz + 16 * slices + 8 * N
            kname = (f"k_sellu<float, OpInnerQ>: q = A p fused with <p,q> (FP32 SELL-U, "
                     f"{uniform}/{slices} slices uniform, {slots} value slots)")
        else:
            kname = "k_crs<float, OpInnerQ>: q = A p fused with <p,q> (FP32 CRS, inner)"
        inner_roof = {"bound": "hbm", "achieved": fp32_spmv_bytes / (spmv_us[args.path] * 1e-6) / 1e9,
                      "launch_us": spmv_us[args.path],
                      "peak": peak, "unit": "GB/s", "kernel": kname,
                      "algorithmic_bytes": fp32_spmv_bytes, "peak_kind": peak_kind}
        inner_roof["frac"] = inner_roof["achieved"] / peak
        prof32 = read_traffic_profile(prof_name, args) if prof_name else None
        inner_roof["traffic"] = prof32.get("dram_bytes_per_launch") if prof32 else None
    roof = fp64_roof if args.path == "plain" else inner_roof
    persist = persist_roofline(args, results, N, peak, peak_kind)
    if persist is not None:
        roof = persist

    # End to end through the public C ABI: pinned host inputs uploaded every
    # step (matrix, Jacobi C, right-hand side), the learned set-up and
    # inference, the solve, x read back.
    ptr_h = cg.pinned_empty(N + 1, np.int32)
    idx_h = cg.pinned_empty(nnz, np.int32)
    val_h = cg.pinned_empty(nnz, np.float64)
    b_h = cg.pinned_empty(N, np.float64)
    c_h = cg.pinned_empty(N, np.float64)
    x_h = cg.pinned_empty(N, np.float64)
    ptr_h[:] = A.ptr
    idx_h[:] = A.index
    val_h[:] = A.value
    b_h[:] = b
    c_h[:] = Cd
    e2e_steps = max(2, min(args.steps, 5))

    def e2e_step():
        h.upload_crs(ptr_h, idx_h, val_h)
        h.upload_jacobi(c_h)
        h.set_vector("K", b_h)
        if args.path == "learned":
            h.learned_setup()
            h.learned_factor(net, args.eps)
        r = h.solve(solve_opts(cg, args, args.path))
        h.get_vector("X", out=x_h)
        return r

    e2e_step()  # warm-up (graphs are rebuilt after a re-upload)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    barrier(world)
    e2e_ms = max_over_ranks(world, wall_ms)
    h2d = 4 * (N + 1) + 12 * nnz + 16 * N
    d2h = 8 * N

    iters = res["iterations"]
    outer = res["outer_iterations"]
    # Persistent inner solves: one cooperative launch per refinement step
    # after its start.
    persist = args.path != "plain" and res["inner_form"] != 0
    # Per solve: the fill of x, the dot of ||b||, a true-residual product per
    # refinement check (outer + 1), and per refinement step its start, the
    # inner solve and the update of x; the learned path adds its set-up
    # (2 kernels), inference (6) and the start's apply (2 per step).
    if args.path == "plain":
        per_solve = 2 + 4 * iters                   # fill, set-up, 3 fused + guard
    elif args.path == "mixed":
        inner = outer if persist else 4 * iters     # one launch, or 3 kernels + guard
        per_solve = 2 + (outer + 1) + 2 * outer + inner
    else:
        inner = outer if persist else 6 * iters     # one launch, or 5 kernels + guard
        per_solve = 2 + 8 + (outer + 1) + 4 * outer + inner
    launches = args.steps * per_solve

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(A, b, args, side["plain"]["iterations"])

    if rank == 0:
        line = {
            "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": {"plain": "f64", "mixed": "f32+f64"}.get(args.path, "bf16+f32+f64"),
            "data": "synthetic (seeded generator; no dataset)",
            "config": workload_config(args, A),
            "path": args.path, "network": net_info,
            "iterations": iters, "outer_iterations": outer,
            "residual": res["residual"], "true_residual": true_rel,
            "rel_error_vs_exact": err_vs_exact, "converged": bool(res["converged"]),
            "paths": side,
            "speedup_vs_plain_fp64": side["plain"]["ms"] / ms,
            "kernel_us": kern,
            "plain_iteration_gbs": plain_iter_bytes / (plain_iter_us * 1e-6) / 1e9,
            "plain_iteration_frac": plain_iter_bytes / (plain_iter_us * 1e-6) / 1e9 / peak,
            "roofline": roof,
            "roofline_inner_spmv": inner_roof,
            "roofline_fp64_spmv": fp64_roof,
            "clocks": clocks,
            "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps},
            "gpu_launches": launches,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    h.close()
    net.close()


def cpu_baseline(A, b, args, full_iters):
    """The reference's OpenMP CG on a bounded sample: `sample` iterations of
    the same solve (CG_MAX_ITER), scaled to the full iteration count."""
    from oracle import oracle as O
    if O.ref_binary("ref_harness_omp") is None:
        return None
    threads = host_threads()
    sample = 100
    try:
        times, iters, _ = run_reference(A, b, workload_name(args), 2, sample, args.tol, threads,
                                        native=True)
    except Exception as e:  # pragma: no cover - reported, not fatal
        return {"value": None, "error": str(e)[:200]}
    t = min(times)
    per_iter_ms = 1e3 * t / iters[-1]
    full = full_iters or iters[-1]
    out = {"value": per_iter_ms * full, "unit": "ms", "cores": threads, "kind": "reference",
           "sample": f"{iters[-1]} iterations (CG_MAX_ITER={sample}) of the same solve by the "
                     f"reference's CGOpenMP, best of 2, scaled to {full} iterations",
           "ms_per_iteration": per_iter_ms}
    # The reference's serial CG beside it, on one core: a smaller sample
    # (an estimate: per-iteration time of the first 50 iterations, scaled).
    if O.ref_binary("ref_harness_serial") is not None:
        ssample = 50
        try:
            st, si, _ = run_reference(A, b, workload_name(args), 1, ssample, args.tol, 1,
                                      backend="serial", native=True)
            s_ms = 1e3 * min(st) / si[-1]
            out["serial"] = {"value": s_ms * full, "unit": "ms", "cores": 1,
                             "kind": "reference",
                             "sample": f"{si[-1]} iterations (CG_MAX_ITER={ssample}) of the same "
                                       f"solve by the reference's serial CG, scaled to {full} "
                                       "iterations (an estimate, not a full solve)",
                             "ms_per_iteration": s_ms}
        except Exception as e:  # pragma: no cover - reported, not fatal
            out["serial"] = {"value": None, "error": str(e)[:200]}
    return out


def main():
    args = parse_args()
    world, rank, local = dist_setup(args)
    args.gpus = world if world > 1 else args.gpus
    try:
        if args.impl == "reference":
            reference_arm(args, world, rank)
        else:
            our_arm(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
