"""CPU oracle of the learned preconditioner -- TEST INFRASTRUCTURE ONLY.

No counterpart exists in the reference (hahnjo/CGxx has Jacobi only), so the
parity of this part is pinned to this restatement, not to the reference.
It states, in torch on the CPU, exactly what the device kernels compute:

  Jacobi-scaled matrix  Ahat = D^-1/2 A D^-1/2,  w_ij = |Ahat_ij| (i != j)
  node features         f_i = [1, sum_j w_ij, deg_i / 6, max_j w_ij]
  embedding             h0 = bf16(relu(W_in f + b_in))                (32)
  3 message-passing layers, l = 0..2:
      agg_i = bf16(sum_{j != i} w_ij h_j)          (FP32 accumulation)
      h_i  <- bf16(h_i + relu(W_l [h_i ; agg_i] + b_l))   (BF16 operands,
                                                          FP32 accumulation)
  head                  o_i = W_h h_i + b_h = [a, dg, u(4), v(4)]     (FP32)
  factor G (lower triangular on the pattern of tril(A)):
      Ghat_ii = softplus(dg_i + 0.5413)
      Ghat_ij = w_ij (a_i + u_i . v_j)                         (i > j)
      G = D^-1/2 Ghat,   M^-1 = G G^T + eps D^-1
  loss (Hutchinson)     L = ||(Ghat^T Ahat Ghat - I) V||_F^2 / (N S)
                        for S probe columns V.

bf16 rounding (round to nearest even) is emulated with a straight-through
identity gradient, as the device backward pass treats it.
"""
import numpy as np
import torch

WIDTH = 32
RANK = 4
NIN = 4
NOUT = 2 + 2 * RANK
DIAG_OFFSET = 0.5413  # softplus(0.5413) = 1.0000


def param_shapes():
    shapes = [("W_in", (WIDTH, NIN)), ("b_in", (WIDTH,))]
    for l in range(3):
        shapes += [(f"W_{l}", (WIDTH, 2 * WIDTH)), (f"b_{l}", (WIDTH,))]
    shapes += [("W_h", (NOUT, WIDTH)), ("b_h", (NOUT,))]
    return shapes


def param_count():
    return sum(int(np.prod(s)) for _, s in param_shapes())


def unflatten(flat):
    out, o = {}, 0
    for name, shp in param_shapes():
        n = int(np.prod(shp))
        out[name] = flat[o:o + n].reshape(shp)
        o += n
    return out


def init_params(seed=0):
    """Default initialisation (also used by the device trainer's driver)."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, shp in param_shapes():
        if name.startswith("W_h"):
            p[name] = rng.normal(0, 0.01, shp)
        elif name.startswith("W"):
            fan_in = shp[1]
            p[name] = rng.normal(0, np.sqrt(2.0 / fan_in), shp)
        else:
            p[name] = np.zeros(shp)
    for name in ("W_0", "W_1", "W_2"):
        p[name] *= 0.5
    return np.concatenate([p[n].ravel() for n, _ in param_shapes()]).astype(np.float32)


def bf16(x):
    """Round to bfloat16 (nearest even), identity gradient."""
    return x + (x.to(torch.bfloat16).to(x.dtype) - x).detach()


class Graph:
    """Scaled-graph arrays of one CRS matrix (0-based, any row order)."""

    def __init__(self, ptr, index, value):
        ptr = np.asarray(ptr, np.int64)
        index = np.asarray(index, np.int64)
        value = np.asarray(value, np.float64)
        N = len(ptr) - 1
        rows = np.repeat(np.arange(N), np.diff(ptr))
        diag = np.zeros(N)
        dm = rows == index
        diag[rows[dm]] = value[dm]
        self.N = N
        self.d = diag
        ah = value / np.sqrt(diag[rows] * diag[index])
        off = rows != index
        low = rows > index
        t = lambda a: torch.tensor(a)
        self.r, self.c = t(rows), t(index)
        self.ah = t(ah.astype(np.float32))
        self.orow, self.ocol = t(rows[off]), t(index[off])
        self.ow = t(np.abs(ah[off]).astype(np.float32))
        self.lr, self.lc = t(rows[low]), t(index[low])
        self.lw = t(np.abs(ah[low]).astype(np.float32))
        deg = np.bincount(rows[off], minlength=N).astype(np.float64)
        s = np.bincount(rows[off], weights=np.abs(ah[off]), minlength=N)
        mx = np.zeros(N)
        np.maximum.at(mx, rows[off], np.abs(ah[off]))
        self.feat = t(np.stack([np.ones(N), s, deg / 6.0, mx], 1).astype(np.float32))

    def ahat_mv(self, V):
        return torch.zeros_like(V).index_add_(0, self.r, self.ah[:, None] * V[self.c])


def rademacher(N, seed):
    """Probes V[i, s] = +-1 from the counter-based hash of the device's
    probe generator (splitmix64 finalizer of seed + golden-ratio * (t + 1),
    t = i * 8 + s; odd -> +1)."""
    t = np.arange(N * 8, dtype=np.uint64) + np.uint64(1)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + np.uint64(0x9E3779B97F4A7C15) * t
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z ^= z >> np.uint64(31)
    return np.where(z & np.uint64(1), 1.0, -1.0).astype(np.float32).reshape(N, 8)


def smooth_probes(g: Graph, V, steps, cols, scale, omega=2.0 / 3.0):
    """The probe recipe's smoothing: the last `cols` columns take `steps`
    damped-Jacobi steps V <- V - omega Ahat V and are then multiplied by
    `scale`."""
    V = torch.tensor(np.asarray(V, np.float32))
    if steps <= 0 or cols <= 0:
        return V.numpy()
    for k in range(steps):
        T = g.ahat_mv(V)
        W = V - omega * T
        if k == steps - 1:
            W = scale * W
        V = torch.cat([V[:, :8 - cols], W[:, 8 - cols:]], 1)
    return V.numpy()


def residual_probe(g: Graph, r):
    """A residual snapshot as a probe column: the Jacobi-scaled residual
    D^-1/2 r normalized to unit RMS (computed in FP64, stored in FP32)."""
    v = np.asarray(r, np.float64) / np.sqrt(g.d)
    s = float(v @ v)
    return (v * np.sqrt(g.N / s) if s > 0 else 0.0 * v).astype(np.float32)


def forward(g: Graph, flat):
    """Returns (gdiag[N], goff[n_lower]) in lower-pattern order (row-major,
    storage order within a row) as float32 tensors with autograd."""
    P = unflatten(flat)
    h = bf16(torch.relu(g.feat @ P["W_in"].T + P["b_in"]))
    for l in range(3):
        agg = torch.zeros_like(h).index_add_(0, g.orow, g.ow[:, None] * h[g.ocol])
        X = torch.cat([h, bf16(agg)], 1)
        pre = X @ bf16(P[f"W_{l}"]).T + P[f"b_{l}"]
        h = bf16(h + torch.relu(pre))
    o = h @ P["W_h"].T + P["b_h"]
    a, dg = o[:, 0], o[:, 1]
    u, v = o[:, 2:2 + RANK], o[:, 2 + RANK:]
    gdiag = torch.nn.functional.softplus(dg + DIAG_OFFSET)
    goff = g.lw * (a[g.lr] + (u[g.lr] * v[g.lc]).sum(1))
    return gdiag, goff


def g_mv(g, gdiag, goff, V):
    return gdiag[:, None] * V + torch.zeros_like(V).index_add_(0, g.lr, goff[:, None] * V[g.lc])


def gt_mv(g, gdiag, goff, W):
    return gdiag[:, None] * W + torch.zeros_like(W).index_add_(0, g.lc, goff[:, None] * W[g.lr])


def loss(g, gdiag, goff, V):
    R = gt_mv(g, gdiag, goff, g.ahat_mv(g_mv(g, gdiag, goff, V))) - V
    return (R * R).sum() / V.numel()


def loss_and_grad(g: Graph, flat_np, V_np):
    """Loss and gradient w.r.t. the flat parameter vector (float32)."""
    flat = torch.tensor(np.asarray(flat_np, np.float32), requires_grad=True)
    V = torch.tensor(np.asarray(V_np, np.float32))
    gd, go = forward(g, flat)
    L = loss(g, gd, go, V)
    L.backward()
    return float(L), flat.grad.numpy().copy()


def factor(g: Graph, flat_np):
    """G values (no autograd): (gdiag, goff) as numpy float32."""
    with torch.no_grad():
        gd, go = forward(g, torch.tensor(np.asarray(flat_np, np.float32)))
    return gd.numpy(), go.numpy()
