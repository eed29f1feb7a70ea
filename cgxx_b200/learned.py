"""Learned preconditioner: weight files, training and evaluation driver.

The network and its training run on the GPU in libcgb200 (cgx_gnn_*,
cgx_learned_*); this module orchestrates them through the C ABI:

  python -m cgxx_b200.learned train --family graph --out cgxx_b200/weights/graph12.gnn
      256 seeded random geometric graphs of 200k points (mean degree 12),
      16 held-out, the same loss, probes and selection.

  python -m cgxx_b200.learned train --out cgxx_b200/weights/diffusion7.gnn
      512 seeded training fields and 64 held-out fields on a 96^3 grid
      (7-point diffusion, coefficient exp(g), g a Gaussian random field with
      sigma ~ U[0.5, 2] and correlation length ~ U[4, 16] cells), Adam on
      the Hutchinson loss ||(Ghat^T Ahat Ghat - I) V||^2 with Rademacher
      probes V (by default half of the 8 columns smoothed by 3 damped-Jacobi
      steps and scaled by 3, which weights the smooth end of the spectrum
      that limits CG; --residual-probes k takes k columns from residuals of
      the solver's own plain Jacobi-CG iterates on each training matrix),
      then PCG on the held-out fields: learned G G^T
      against Jacobi, both FP32-inner / FP64-refinement to a 1e-9 FP64 true
      residual, and plain FP64 Jacobi-CG.

      Checkpoint selection: the untrained network and the network after
      each epoch are scored by the median learned-PCG iteration count on 16
      held-out fields; the best is written (the untrained network when no
      epoch improves on it). On this family the untrained network already
      reproduces the quality of a factorized sparse approximate inverse on
      the pattern of tril(A), so training has little room to gain.

Weight file: 8-byte magic b"CGXGNN01", uint32 header length, UTF-8 JSON
header (parameter count, dtype, layout, seed, training configuration and its
SHA-256), then the float32 parameters (little endian).
"""
import argparse
import hashlib
import json
import os
import struct
import sys
import time

import numpy as np

MAGIC = b"CGXGNN01"
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "diffusion7.gnn")
LAYOUT = "W_in[32x4] b_in[32] (W_l[32x64] b_l[32]) x3 W_h[10x32] b_h[10]"


def save_weights(path, params, meta):
    params = np.ascontiguousarray(params, dtype="<f4")
    head = dict(meta)
    head.update({"param_count": int(params.size), "dtype": "float32", "layout": LAYOUT})
    cfg = json.dumps(head.get("config", {}), sort_keys=True).encode()
    head["config_sha256"] = hashlib.sha256(cfg).hexdigest()
    blob = json.dumps(head, sort_keys=True).encode()
    tmp = path + ".tmp"
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(tmp, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<I", len(blob)))
        f.write(blob)
        f.write(params.tobytes())
    os.replace(tmp, path)


def load_weights(path):
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path}: not a cgxx_b200 weight file")
        (n,) = struct.unpack("<I", f.read(4))
        head = json.loads(f.read(n).decode())
        params = np.frombuffer(f.read(), dtype="<f4").copy()
    if params.size != head["param_count"]:
        raise ValueError(f"{path}: truncated parameters")
    return params, head


# ---------------------------------------------------------------------------
# Data

def _field_values(args):
    n, sigma, ell, seed = args
    from cgxx_b200 import generators as G
    fam = G.Diffusion7Family(n)
    return fam.values(G.diffusion_field(n, sigma, ell, seed))


def family_specs(count, seed0, rng_seed):
    rng = np.random.default_rng(rng_seed)
    return [(float(rng.uniform(0.5, 2.0)), float(rng.uniform(4.0, 16.0)), seed0 + k)
            for k in range(count)]


def generate_values(n, specs, workers):
    """Value arrays of the 7-point family for (sigma, ell, seed) specs, made
    by a spawn process pool (no CUDA state is inherited)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        return pool.map(_field_values, [(n, s, l, sd) for (s, l, sd) in specs], chunksize=4)


# ---------------------------------------------------------------------------
# Training and evaluation

def solve_pair(h, A_ptr, A_index, vals, b, learned_ok, net, eps, max_iter=20000):
    """Returns dict of ms / iterations for jacobi-mixed, learned-mixed,
    plain-fp64 on the matrix currently in h (values `vals`)."""
    import cgxx_b200 as cg
    out = {}
    h.set_vector("K", b)
    t0 = time.perf_counter()
    h.learned_setup()
    h.learned_factor(net, eps)
    h.synchronize()
    out["factor_ms"] = (time.perf_counter() - t0) * 1e3
    for name, pc, prec in (("learned_mixed", cg.PRECOND_LEARNED, cg.PRECISION_MIXED),
                           ("jacobi_mixed", cg.PRECOND_JACOBI, cg.PRECISION_MIXED),
                           ("plain_fp64", cg.PRECOND_JACOBI, cg.PRECISION_FP64)):
        h.fill_vector("X", 0.0)
        r = h.solve(max_iterations=max_iter, tolerance=1e-9, preconditioner=pc,
                    precision=prec)
        out[name] = {"ms": r["solve_ms"], "iterations": r["iterations"],
                     "converged": bool(r["converged"]), "fell_back": bool(r["fell_back"])}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--family", choices=["diffusion7", "graph"], default="diffusion7")
    t.add_argument("--n", type=int, default=96, help="grid edge (diffusion7)")
    t.add_argument("--points", type=int, default=200000, help="points per graph (graph)")
    t.add_argument("--train", type=int, default=None,
                   help="training matrices (default 512 fields, 256 graphs)")
    t.add_argument("--heldout", type=int, default=None,
                   help="held-out matrices (default 64 fields, 16 graphs)")
    t.add_argument("--epochs", type=int, default=4)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--eps", type=float, default=1e-4)
    t.add_argument("--smooth-steps", type=int, default=3)
    t.add_argument("--smooth-cols", type=int, default=4)
    t.add_argument("--smooth-scale", type=float, default=3.0)
    t.add_argument("--residual-probes", type=int, default=0,
                   help="probe columns taken from residuals of the solver's own "
                        "plain Jacobi-CG iterates on each training matrix")
    t.add_argument("--residual-its", default="5,10,20,40",
                   help="iterations of the restarted solves before each snapshot")
    t.add_argument("--select", type=int, default=16,
                   help="held-out fields scored for checkpoint selection")
    t.add_argument("--seed", type=int, default=0)
    t.add_argument("--workers", type=int, default=min(16, os.cpu_count() or 1))
    t.add_argument("--out", default=DEFAULT_WEIGHTS)
    t.add_argument("--report", default=None)
    t.add_argument("--eval-only", action="store_true")
    a = ap.parse_args(argv)
    if a.cmd == "train":
        graph = a.family == "graph"
        if a.train is None:
            a.train = 256 if graph else 512
        if a.heldout is None:
            a.heldout = 16 if graph else 64
        if graph:
            run_graph_training(a)
        else:
            run_training(a)


def init_params(seed=0):
    """The network's initial parameters: He-normal weights (layer weights
    halved), a near-zero head, zero biases. The factor's head carries no
    hand-set prior, so the untrained factor is Ghat ~ I (G G^T ~ D^-1, the
    Jacobi preconditioner) and training learns every off-diagonal value.
    Same as the oracle's init_params."""
    W, NIN, NOUT = 32, 4, 10
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0, np.sqrt(2.0 / NIN), (W, NIN)), np.zeros(W)]
    for _ in range(3):
        parts += [0.5 * rng.normal(0, np.sqrt(2.0 / (2 * W)), (W, 2 * W)), np.zeros(W)]
    parts += [rng.normal(0, 0.01, (NOUT, W)), np.zeros(NOUT)]
    return np.concatenate([p.ravel() for p in parts]).astype(np.float32)


def run_training(a):
    # Data first (spawn pool), before any CUDA work in this process.
    t0 = time.time()
    tr_specs = family_specs(a.train, 100000, 1000 + a.seed)
    ho_specs = family_specs(a.heldout, 900000, 2000 + a.seed)
    ho_vals = generate_values(a.n, ho_specs, a.workers)

    import torch

    import cgxx_b200 as cg
    from cgxx_b200 import generators as G
    fam = G.Diffusion7Family(a.n)
    dev = torch.device("cuda", 0)
    # All training matrices resident in HBM (nnz doubles each), generated in
    # batches so that the host holds one batch at a time.
    tr_dev = []
    if not a.eval_only:
        for b0 in range(0, len(tr_specs), 64):
            batch = generate_values(a.n, tr_specs[b0:b0 + 64], a.workers)
            tr_dev += [torch.from_numpy(v).to(dev) for v in batch]
            del batch
    gen_s = time.time() - t0
    h = cg.Handle(0)
    h.upload_crs(fam.ptr, fam.index, ho_vals[0])
    h.learned_setup()
    if a.eval_only:
        params, head = load_weights(a.out)
    else:
        params = init_params(a.seed)
    net = cg.Gnn(0, params)
    net.set_probes(a.smooth_steps, a.smooth_cols, a.smooth_scale, a.residual_probes)
    res_its = [int(t) for t in a.residual_its.split(",")][:a.residual_probes]
    rhs = [np.random.default_rng(7 + k).uniform(-1.0, 1.0, fam.N) for k in range(4)]

    def snapshots(k):
        """Residual snapshots of training matrix k: plain Jacobi-CG from x = 0
        on a random right-hand side, restarted after each res_its entry, with
        r = b - A x captured after each part."""
        h.jacobi_from_matrix()
        h.set_vector("K", rhs[k % len(rhs)])
        h.fill_vector("X", 0.0)
        for j, its in enumerate(res_its):
            h.solve(max_iterations=its, tolerance=1e-30)
            h.learned_capture_residual(8 - a.residual_probes + j)

    def selection_score(gnn):
        its = []
        for k, v in enumerate(ho_vals[:a.select]):
            h.update_crs_values(v)
            h.upload_jacobi(_diag_inv(fam, v))
            b, _ = G.rhs_for(G.Crs(fam.N, fam.ptr, fam.index, v), seed=k)
            h.set_vector("K", b)
            h.learned_setup()
            h.learned_factor(gnn, a.eps)
            h.fill_vector("X", 0.0)
            r = h.solve(max_iterations=20000, tolerance=1e-9,
                        preconditioner=cg.PRECOND_LEARNED, precision=cg.PRECISION_MIXED)
            its.append(r["iterations"] if r["converged"] else 10 ** 9)
        return float(np.median(its))

    log = []
    t1 = time.time()
    steps = 0
    selected = 0
    if not a.eval_only:
        best = (selection_score(net), 0, net.get_params())
        log.append({"epoch": -1, "selection_median_iterations": best[0]})
        print(json.dumps(log[-1]), flush=True)
        rng = np.random.default_rng(a.seed)
        for ep in range(a.epochs):
            order = rng.permutation(len(tr_dev))
            losses = []
            lr = a.lr * (0.5 ** ep)
            for k in order:
                h.update_crs_values_ptr(tr_dev[k].data_ptr())
                h.learned_setup()
                if a.residual_probes:
                    snapshots(int(k))
                losses.append(net.train_step(h, seed=int(rng.integers(1 << 62)), lr=lr))
                steps += 1
            score = selection_score(net)
            log.append({"epoch": ep, "lr": lr, "mean_loss": float(np.mean(losses)),
                        "selection_median_iterations": score})
            print(json.dumps(log[-1]), flush=True)
            if score < best[0]:
                best = (score, ep + 1, net.get_params())
        torch.cuda.synchronize()
        selected = best[1]
        net.set_params(best[2])
    train_s = time.time() - t1
    params = net.get_params()

    # Held-out evaluation.
    res = []
    init_net = cg.Gnn(0, init_params(a.seed))
    for k, v in enumerate(ho_vals):
        h.update_crs_values(v)
        h.upload_jacobi(_diag_inv(fam, v))
        b, _ = G.rhs_for(G.Crs(fam.N, fam.ptr, fam.index, v), seed=k)
        r = solve_pair(h, fam.ptr, fam.index, v, b, True, net, a.eps)
        h.learned_setup()
        h.learned_factor(init_net, a.eps)
        h.fill_vector("X", 0.0)
        ri = h.solve(max_iterations=20000, tolerance=1e-9,
                     preconditioner=cg.PRECOND_LEARNED, precision=cg.PRECISION_MIXED)
        r["untrained_learned_mixed"] = {"ms": ri["solve_ms"], "iterations": ri["iterations"]}
        res.append(r)
    summary = summarize(res)
    meta = {"seed": a.seed, "steps": steps, "train_seconds": train_s,
            "selected_epoch": selected,
            "generate_seconds": gen_s,
            "config": {"grid": a.n, "stencil": 7, "train": a.train, "heldout": a.heldout,
                       "sigma": [0.5, 2.0], "corr_len": [4.0, 16.0], "epochs": a.epochs,
                       "lr": a.lr, "eps": a.eps, "probes": 8,
                       "smooth_steps": a.smooth_steps, "smooth_cols": a.smooth_cols,
                       "smooth_scale": a.smooth_scale, "select": a.select,
                       "residual_probes": a.residual_probes,
                       "residual_its": res_its,
                       "loss": "||(Ghat^T Ahat Ghat - I) V||^2 / (N S), Rademacher V"},
            "log": log, "heldout": summary}
    if not a.eval_only:
        save_weights(a.out, params, meta)
    if a.report:
        with open(a.report, "w") as f:
            json.dump({"meta": meta, "per_matrix": res}, f, indent=1)
    print(json.dumps({"summary": summary, "train_seconds": train_s, "steps": steps}))


def _graph_arrays(args):
    npts, seed = args
    from cgxx_b200 import generators as G
    A = G.geometric_graph(npts, mean_degree=12.0, seed=seed)
    return A.ptr, A.index, A.value


def _arrays_diag_inv(ptr, index, value):
    rows = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
    d = np.zeros(len(ptr) - 1)
    m = rows == index
    d[rows[m]] = value[m]
    return 1.0 / d


def run_graph_training(a):
    """The irregular family: random geometric graph Laplacians (a.points
    uniform points in the unit cube, mean degree 12, w = exp(-d/r), L + 1e-3 I),
    one seeded graph per training step. Every graph has its own pattern, so
    each step uploads it and runs a fresh set-up; the graphs of an epoch are
    generated by a spawn process pool (created before any CUDA work)
    while the GPU trains on the previous batch."""
    import multiprocessing as mp
    t0 = time.time()
    tr_seeds = [300000 + 1000 * a.seed + k for k in range(a.train)]
    ho_seeds = [700000 + 1000 * a.seed + k for k in range(a.heldout)]
    pool = mp.get_context("spawn").Pool(a.workers)
    ho = pool.map(_graph_arrays, [(a.points, sd) for sd in ho_seeds], chunksize=1)
    gen_s = time.time() - t0

    import cgxx_b200 as cg
    from cgxx_b200 import generators as G
    h = cg.Handle(0)
    if a.eval_only:
        params, head = load_weights(a.out)
    else:
        params = init_params(a.seed)
    net = cg.Gnn(0, params)
    net.set_probes(a.smooth_steps, a.smooth_cols, a.smooth_scale, a.residual_probes)
    res_its = [int(t) for t in a.residual_its.split(",")][:a.residual_probes]

    def load(arrs, k):
        ptr, index, value = arrs
        h.upload_crs(ptr, index, value)
        h.upload_jacobi(_arrays_diag_inv(ptr, index, value))
        b, _ = G.rhs_for(G.Crs(len(ptr) - 1, ptr, index, value), seed=k)
        h.set_vector("K", b)
        h.learned_setup()
        return b

    def selection_score(gnn):
        its = []
        for k, arrs in enumerate(ho[:a.select]):
            load(arrs, k)
            h.learned_factor(gnn, a.eps)
            h.fill_vector("X", 0.0)
            r = h.solve(max_iterations=20000, tolerance=1e-9,
                        preconditioner=cg.PRECOND_LEARNED, precision=cg.PRECISION_MIXED)
            its.append(r["iterations"] if r["converged"] else 10 ** 9)
        return float(np.median(its))

    log = []
    t1 = time.time()
    steps = 0
    selected = 0
    if not a.eval_only:
        best = (selection_score(net), 0, net.get_params())
        log.append({"epoch": -1, "selection_median_iterations": best[0]})
        print(json.dumps(log[-1]), flush=True)
        rng = np.random.default_rng(a.seed)
        for ep in range(a.epochs):
            order = [tr_seeds[k] for k in rng.permutation(len(tr_seeds))]
            losses = []
            lr = a.lr * (0.5 ** ep)
            for arrs in pool.imap(_graph_arrays, [(a.points, sd) for sd in order], chunksize=1):
                load(arrs, steps)
                if a.residual_probes:
                    h.fill_vector("X", 0.0)
                    for j, its in enumerate(res_its):
                        h.solve(max_iterations=its, tolerance=1e-30)
                        h.learned_capture_residual(8 - a.residual_probes + j)
                losses.append(net.train_step(h, seed=int(rng.integers(1 << 62)), lr=lr))
                steps += 1
            score = selection_score(net)
            log.append({"epoch": ep, "lr": lr, "mean_loss": float(np.mean(losses)),
                        "selection_median_iterations": score})
            print(json.dumps(log[-1]), flush=True)
            if score < best[0]:
                best = (score, ep + 1, net.get_params())
        selected = best[1]
        net.set_params(best[2])
    pool.close()
    train_s = time.time() - t1
    params = net.get_params()

    res = []
    init_net = cg.Gnn(0, init_params(a.seed))
    for k, arrs in enumerate(ho):
        b = load(arrs, k)
        r = solve_pair(h, arrs[0], arrs[1], arrs[2], b, True, net, a.eps)
        h.learned_setup()
        h.learned_factor(init_net, a.eps)
        h.fill_vector("X", 0.0)
        ri = h.solve(max_iterations=20000, tolerance=1e-9,
                     preconditioner=cg.PRECOND_LEARNED, precision=cg.PRECISION_MIXED)
        r["untrained_learned_mixed"] = {"ms": ri["solve_ms"], "iterations": ri["iterations"]}
        res.append(r)
    summary = summarize(res)
    meta = {"seed": a.seed, "steps": steps, "train_seconds": train_s,
            "selected_epoch": selected, "generate_seconds": gen_s,
            "config": {"family": "geometric graph", "points": a.points, "mean_degree": 12,
                       "weights": "exp(-d/r)", "shift": 1e-3, "train": a.train,
                       "heldout": a.heldout, "epochs": a.epochs, "lr": a.lr, "eps": a.eps,
                       "probes": 8, "smooth_steps": a.smooth_steps,
                       "smooth_cols": a.smooth_cols, "smooth_scale": a.smooth_scale,
                       "select": a.select, "residual_probes": a.residual_probes,
                       "residual_its": res_its,
                       "loss": "||(Ghat^T Ahat Ghat - I) V||^2 / (N S), Rademacher V"},
            "log": log, "heldout": summary}
    if not a.eval_only:
        save_weights(a.out, params, meta)
    if a.report:
        with open(a.report, "w") as f:
            json.dump({"meta": meta, "per_matrix": res}, f, indent=1)
    print(json.dumps({"summary": summary, "train_seconds": train_s, "steps": steps}))


def _diag_inv(fam, v):
    rows = np.repeat(np.arange(fam.N), np.diff(fam.ptr))
    d = np.zeros(fam.N)
    m = rows == fam.index
    d[rows[m]] = v[m]
    return 1.0 / d


def summarize(res):
    def med(key, field):
        return float(np.median([r[key][field] for r in res if key in r]))
    out = {}
    for key in ("learned_mixed", "jacobi_mixed", "plain_fp64", "untrained_learned_mixed"):
        if any(key in r for r in res):
            out[key] = {"median_ms": med(key, "ms"), "median_iterations": med(key, "iterations")}
    out["factor_ms_median"] = float(np.median([r["factor_ms"] for r in res]))
    out["all_converged"] = all(r[k]["converged"] for r in res
                               for k in ("learned_mixed", "jacobi_mixed", "plain_fp64"))
    out["fell_back"] = sum(r["learned_mixed"]["fell_back"] for r in res)
    it_l = np.array([r["learned_mixed"]["iterations"] for r in res], float)
    it_j = np.array([r["plain_fp64"]["iterations"] for r in res], float)
    ms_l = np.array([r["learned_mixed"]["ms"] + r["factor_ms"] for r in res])
    ms_p = np.array([r["plain_fp64"]["ms"] for r in res])
    out["iteration_ratio_plain_over_learned_median"] = float(np.median(it_j / it_l))
    out["speedup_vs_plain_incl_factor_median"] = float(np.median(ms_p / ms_l))
    return out


if __name__ == "__main__":
    sys.exit(main())
