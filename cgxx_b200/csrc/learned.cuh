// Learned preconditioner M^-1 = G G^T + eps D^-1 (no counterpart in the
// reference): device kernels for
//   - the Jacobi-scaled graph of A: 1/sqrt(A_ii), |Ahat_ij|, node features,
//     the pattern of G (lower triangle of A, diagonal included, storage
//     order) and of G^T (upper triangle), and the maps between them;
//   - the message-passing network that emits G's values (forward on BF16
//     tensor cores, mma.sync m16n8k16, FP32 accumulation);
//   - its training: the Hutchinson loss ||(Ghat^T Ahat Ghat - I) V||^2 and the
//     backward pass through the factor, the head, the three layers and the
//     embedding (gathers over the symmetric pattern; no atomics, so the
//     gradient is deterministic);
//   - Adam.
// The exact arithmetic is stated in oracle/gnn_oracle.py, the CPU oracle the
// tests compare these kernels with.
#pragma once

#include <cuda_bf16.h>

#include "device.cuh"

namespace cgx {
namespace learned {

constexpr int W = 32;       // feature width
constexpr int RANK = 4;     // rank of the off-diagonal bilinear term
constexpr int NIN = 4;      // node input features
constexpr int NOUT = 2 + 2 * RANK;
constexpr float DIAG_OFFSET = 0.5413f;
constexpr int S = 8;        // Hutchinson probe columns per training step

// Flat parameter layout (FP32), identical to oracle/gnn_oracle.py.
constexpr int OFF_WIN = 0;
constexpr int OFF_BIN = OFF_WIN + W * NIN;
constexpr int OFF_L0 = OFF_BIN + W;
constexpr int L_STRIDE = W * 2 * W + W;  // W_l then b_l
constexpr int OFF_WH = OFF_L0 + 3 * L_STRIDE;
constexpr int OFF_BH = OFF_WH + NOUT * W;
constexpr int NPARAMS = OFF_BH + NOUT;

__device__ __forceinline__ float softplus(float x) {
  return x > 20.f ? x : log1pf(expf(x));
}
__device__ __forceinline__ float sigmoid(float x) {
  return 1.f / (1.f + expf(-x));
}

// ---------------------------------------------------------------------------
// Scaled graph

// dis_i = 1 / sqrt(A_ii) (last diagonal entry of the row; 0 if none -> the
// set-up reports an error).
__global__ void k_inv_sqrt_diag(int N, const int *__restrict__ ptr,
                                const int *__restrict__ index,
                                const double *__restrict__ value,
                                double *dis, int *flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int j = ptr[i]; j < ptr[i + 1]; j++)
      if (index[j] == i) d = value[j];
    if (!(d > 0.0)) {
      atomicOr(flag, 1);
      dis[i] = 0.0;
    } else {
      dis[i] = 1.0 / sqrt(d);
    }
  }
}

// Ahat entries (FP32), node features and the lower/upper counts per row.
__global__ void k_scaled_rows(int N, const int *__restrict__ ptr,
                              const int *__restrict__ index,
                              const double *__restrict__ value,
                              const double *__restrict__ dis,
                              float *__restrict__ ahat, float *__restrict__ feat,
                              int *__restrict__ nlow, int *__restrict__ nup) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x) {
    const double di = dis[i];
    float s = 0.f, mx = 0.f;
    int deg = 0, lo = 0, up = 0;
    for (int j = ptr[i]; j < ptr[i + 1]; j++) {
      const int c = index[j];
      const float a = (float)(value[j] * di * dis[c]);
      ahat[j] = a;
      if (c != i) {
        s += fabsf(a);
        mx = fmaxf(mx, fabsf(a));
        deg++;
      }
      lo += c <= i;
      up += c >= i;
    }
    feat[i * NIN + 0] = 1.f;
    feat[i * NIN + 1] = s;
    feat[i * NIN + 2] = (float)deg / 6.f;
    feat[i * NIN + 3] = mx;
    nlow[i] = lo;
    nup[i] = up;
  }
}

// Block-level exclusive scan helpers for the pattern build: three launches
// (per-block totals, scan of the totals, add offsets), out[0] = 0 and
// out[n] = total.
constexpr int kScanBlock = 1024;

__global__ void k_scan_blocks(int n, const int *__restrict__ in,
                              int *__restrict__ out, int *__restrict__ sums) {
  __shared__ int sh[kScanBlock];
  const int i = blockIdx.x * kScanBlock + threadIdx.x;
  sh[threadIdx.x] = i < n ? in[i] : 0;
  __syncthreads();
  for (int o = 1; o < kScanBlock; o <<= 1) {
    int v = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += v;
    __syncthreads();
  }
  if (i < n) out[i + 1] = sh[threadIdx.x];  // inclusive, shifted by one
  if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = sh[threadIdx.x];
}

__global__ void k_scan_sums(int nb, int *sums) {
  // One block; nb may exceed the block size: serial carry over chunks.
  __shared__ int sh[kScanBlock];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += kScanBlock) {
    const int i = base + threadIdx.x;
    sh[threadIdx.x] = i < nb ? sums[i] : 0;
    __syncthreads();
    for (int o = 1; o < kScanBlock; o <<= 1) {
      int v = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
      __syncthreads();
      sh[threadIdx.x] += v;
      __syncthreads();
    }
    const int excl = carry + sh[threadIdx.x] - (i < nb ? sums[i] : 0);
    __syncthreads();
    if (i < nb) sums[i] = excl;  // exclusive block offsets
    if (threadIdx.x == kScanBlock - 1) carry += sh[kScanBlock - 1];
    __syncthreads();
  }
}

__global__ void k_scan_add(int n, int *__restrict__ out,
                           const int *__restrict__ sums) {
  const int i = blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n) out[i + 1] += sums[blockIdx.x];
  if (i == 0) out[0] = 0;
}

// Fills the G (lower) and G^T (upper) patterns in A's storage order, and for
// each G entry the position of the same entry in A (g2a).
__global__ void k_fill_patterns(int N, const int *__restrict__ ptr,
                                const int *__restrict__ index,
                                const int *__restrict__ gptr,
                                const int *__restrict__ tptr,
                                int *__restrict__ gcol, int *__restrict__ grow,
                                int *__restrict__ tcol,
                                int *__restrict__ g2a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x) {
    int g = gptr[i], t = tptr[i];
    for (int j = ptr[i]; j < ptr[i + 1]; j++) {
      const int c = index[j];
      if (c <= i) {
        gcol[g] = c;
        grow[g] = i;
        g2a[g++] = j;
      }
      if (c >= i) tcol[t++] = c;
    }
  }
}

// For every G entry (i, j): its position in G^T row j (entry with column i),
// found by scanning that row. A missing mirror entry (pattern not symmetric)
// sets the flag.
__global__ void k_transpose_map(int nnzL, const int *__restrict__ grow,
                                const int *__restrict__ gcol,
                                const int *__restrict__ tptr,
                                const int *__restrict__ tcol,
                                int *__restrict__ g2t, int *__restrict__ t2g,
                                int *flag) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnzL;
       e += gridDim.x * blockDim.x) {
    const int i = grow[e], j = gcol[e];
    int pos = -1;
    for (int k = tptr[j]; k < tptr[j + 1]; k++)
      if (tcol[k] == i) {
        pos = k;
        break;
      }
    g2t[e] = pos;
    if (pos < 0)
      atomicOr(flag, 2);
    else
      t2g[pos] = e;
  }
}

// ---------------------------------------------------------------------------
// Network forward

__device__ __forceinline__ float relu(float x) { return x > 0.f ? x : 0.f; }

// h0 = bf16(relu(W_in f + b_in)); also keeps pre0 for the backward pass.
__global__ void k_embed(int N, const float *__restrict__ feat,
                        const float *__restrict__ P, __nv_bfloat16 *__restrict__ h,
                        float *__restrict__ pre) {
  // One thread per node: W_in and b_in (contiguous in P) from shared memory,
  // the node's 4 features in one 16-byte load, its 32 outputs in four
  // 16-byte stores.
  __shared__ float sW[W * NIN + W];
  for (int t = threadIdx.x; t < W * NIN + W; t += blockDim.x) sW[t] = P[OFF_WIN + t];
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x) {
    const float4 f4 = *reinterpret_cast<const float4 *>(feat + (size_t)i * NIN);
    const float fv[NIN] = {f4.x, f4.y, f4.z, f4.w};
    uint4 out[W / 8];
    __nv_bfloat16 *ob = reinterpret_cast<__nv_bfloat16 *>(out);
#pragma unroll
    for (int f = 0; f < W; f++) {
      float s = sW[W * NIN + f];
#pragma unroll
      for (int k = 0; k < NIN; k++) s = fmaf(sW[f * NIN + k], fv[k], s);
      if (pre) pre[(size_t)i * W + f] = s;
      ob[f] = __float2bfloat16_rn(relu(s));
    }
    uint4 *dst = reinterpret_cast<uint4 *>(h + (size_t)i * W);
#pragma unroll
    for (int q = 0; q < W / 8; q++) dst[q] = out[q];
  }
}

// Packs two bf16 values into the 32-bit register layout of an mma operand.
__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) |
         ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4],
                                               const uint32_t (&a)[4],
                                               const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One message-passing layer. A warp owns 16 nodes: it gathers
// agg_i = sum_{j != i} |Ahat_ij| h_j (lane f accumulates feature f, FP32),
// stages X = [h_i ; bf16(agg_i)] (16 x 64, BF16) in shared memory, multiplies
// by W_l^T on the tensor cores (4 k-steps x 4 n-tiles of m16n8k16, FP32
// accumulators), adds the bias and writes h_i + relu(pre) as BF16.
constexpr int kLayerWarps = 8;

__global__ void __launch_bounds__(32 * kLayerWarps)
    k_layer(int N, const int *__restrict__ ptr, const int *__restrict__ index,
            const float *__restrict__ ahat, const float *__restrict__ P,
            int layer, const __nv_bfloat16 *__restrict__ hin,
            __nv_bfloat16 *__restrict__ hout, __nv_bfloat16 *__restrict__ agg_out,
            float *__restrict__ pre_out) {
  __shared__ __align__(16) __nv_bfloat16 sW[W][2 * W + 8];  // W_l[n][k], rows padded (banks)
  __shared__ __align__(16) __nv_bfloat16 sX[kLayerWarps][16][2 * W + 8];  // padded rows
  __shared__ float sB[W];
  const float *Wl = P + OFF_L0 + layer * L_STRIDE;
  for (int t = threadIdx.x; t < W * 2 * W; t += blockDim.x)
    sW[t / (2 * W)][t % (2 * W)] = __float2bfloat16_rn(Wl[t]);
  for (int t = threadIdx.x; t < W; t += blockDim.x) sB[t] = Wl[W * 2 * W + t];
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tq = lane & 3;
  const int groups = (N + 15) / 16;
  for (int grp = blockIdx.x * kLayerWarps + warp; grp < groups;
       grp += gridDim.x * kLayerWarps) {
    const int base = grp * 16;
    // Gather: the warp's 16 nodes x 4 chunks of 8 features are 64 tasks,
    // two per lane, so all 16 nodes' neighbour rows are in flight at once;
    // a task reads 16 bytes (8 BF16 features) per neighbour, up to 4
    // neighbours requested before they are summed (in entry order).
    const uint4 *hin4 = reinterpret_cast<const uint4 *>(hin);
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int task = lane + 32 * q;
      const int r = task >> 2, c4 = task & 3;
      const int i = base + r;
      float a[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      uint4 own = make_uint4(0u, 0u, 0u, 0u);
      if (i < N) {
        own = hin4[(size_t)i * (W / 8) + c4];
        const int j0 = ptr[i], j1 = ptr[i + 1];
        for (int j = j0; j < j1; j += 4) {
          float w[4];
          uint4 hv[4];
          int cc[4];
          // All four entries' columns and weights first, then the four
          // gathers: one round trip for each instead of one per entry
          // (measured: inference 6 % faster at 160^3).
#pragma unroll
          for (int u = 0; u < 4; u++)
            if (j + u < j1) {
              cc[u] = index[j + u];
              w[u] = fabsf(ahat[j + u]);
            }
#pragma unroll
          for (int u = 0; u < 4; u++) {
            if (j + u < j1) {
              const int c = cc[u];
              w[u] = c != i ? w[u] : 0.f;
              hv[u] = hin4[(size_t)c * (W / 8) + c4];
            }
          }
#pragma unroll
          for (int u = 0; u < 4; u++) {
            if (j + u < j1) {
              const __nv_bfloat162 *b2 = reinterpret_cast<const __nv_bfloat162 *>(&hv[u]);
#pragma unroll
              for (int k = 0; k < 4; k++) {
                a[2 * k] = fmaf(w[u], __low2float(b2[k]), a[2 * k]);
                a[2 * k + 1] = fmaf(w[u], __high2float(b2[k]), a[2 * k + 1]);
              }
            }
          }
        }
      }
      uint4 ag;
      __nv_bfloat162 *ag2 = reinterpret_cast<__nv_bfloat162 *>(&ag);
#pragma unroll
      for (int k = 0; k < 4; k++) ag2[k] = __floats2bfloat162_rn(a[2 * k], a[2 * k + 1]);
      *reinterpret_cast<uint4 *>(&sX[warp][r][8 * c4]) = own;
      *reinterpret_cast<uint4 *>(&sX[warp][r][W + 8 * c4]) = ag;
      if (agg_out && i < N)
        reinterpret_cast<uint4 *>(agg_out)[(size_t)i * (W / 8) + c4] = ag;
    }
    __syncwarp();
    // pre = X W^T on the tensor cores.
    float acc[4][4];
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[nt][q] = 0.f;
#pragma unroll
    for (int ks = 0; ks < 4; ks++) {
      const int k0 = ks * 16;
      uint32_t a[4];
      a[0] = pack2(sX[warp][g][k0 + 2 * tq], sX[warp][g][k0 + 2 * tq + 1]);
      a[1] = pack2(sX[warp][g + 8][k0 + 2 * tq], sX[warp][g + 8][k0 + 2 * tq + 1]);
      a[2] = pack2(sX[warp][g][k0 + 8 + 2 * tq], sX[warp][g][k0 + 8 + 2 * tq + 1]);
      a[3] = pack2(sX[warp][g + 8][k0 + 8 + 2 * tq],
                   sX[warp][g + 8][k0 + 8 + 2 * tq + 1]);
#pragma unroll
      for (int nt = 0; nt < 4; nt++) {
        const int n = nt * 8 + g;
        uint32_t b[2];
        b[0] = pack2(sW[n][k0 + 2 * tq], sW[n][k0 + 2 * tq + 1]);
        b[1] = pack2(sW[n][k0 + 8 + 2 * tq], sW[n][k0 + 8 + 2 * tq + 1]);
        mma_bf16_16816(acc[nt], a, b);
      }
    }
    // Epilogue: rows g and g+8, columns nt*8 + 2tq + {0,1}. The new h
    // replaces h_i in the staging rows (each element is read and written by
    // the lane that owns it), then the warp stores its 16 rows as 16-byte
    // chunks.
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int r = g + (q >= 2 ? 8 : 0);
        const int col = nt * 8 + 2 * tq + (q & 1);
        const float pre = acc[nt][q] + sB[col];
        if (pre_out && base + r < N) pre_out[(size_t)(base + r) * W + col] = pre;
        const float hv = __bfloat162float(sX[warp][r][col]) + relu(pre);
        sX[warp][r][col] = __float2bfloat16_rn(hv);
      }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int task = lane + 32 * q;
      const int r = task >> 2, c4 = task & 3;
      if (base + r < N)
        reinterpret_cast<uint4 *>(hout)[(size_t)(base + r) * (W / 8) + c4] =
            *reinterpret_cast<const uint4 *>(&sX[warp][r][8 * c4]);
    }
    __syncwarp();
  }
}

// o_i = W_h h_i + b_h (FP32): one thread per node, its 32 features loaded
// once (four 16-byte loads), W_h from shared memory.
__global__ void k_head(int N, const __nv_bfloat16 *__restrict__ h,
                       const float *__restrict__ P, float *__restrict__ o) {
  __shared__ float sW[NOUT * W + NOUT];
  for (int t = threadIdx.x; t < NOUT * W + NOUT; t += blockDim.x)
    sW[t] = P[OFF_WH + t];
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x) {
    float hv[W];
    const uint4 *src = reinterpret_cast<const uint4 *>(h + (size_t)i * W);
#pragma unroll
    for (int q = 0; q < W / 8; q++) {
      const uint4 u = src[q];
      const __nv_bfloat162 *b2 = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        hv[q * 8 + 2 * k] = __low2float(b2[k]);
        hv[q * 8 + 2 * k + 1] = __high2float(b2[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < NOUT; k++) {
      float s = sW[NOUT * W + k];
#pragma unroll
      for (int f = 0; f < W; f++) s = fmaf(sW[k * W + f], hv[f], s);
      o[(size_t)i * NOUT + k] = s;
    }
  }
}

// Values of Ghat on its pattern from the head outputs,
//   Ghat_ii = softplus(dg_i + DIAG_OFFSET),  Ghat_ij = w_ij (a_i + u_i . v_j),
// with no constant term: a head near zero (the untrained network) gives
// Ghat = I, i.e. G G^T = D^-1, Jacobi; every off-diagonal value is learned.
// Optionally the scaled factor G = D^-1/2 Ghat for the apply, in G order and
// in G^T order.
__global__ void k_assemble(int nnzL, const int *__restrict__ grow,
                           const int *__restrict__ gcol,
                           const int *__restrict__ g2a,
                           const float *__restrict__ ahat,
                           const float *__restrict__ o, float *__restrict__ ghat,
                           const double *__restrict__ dis,
                           const int *__restrict__ g2t, float *__restrict__ gs,
                           float *__restrict__ gts, __nv_bfloat16 *__restrict__ sgv,
                           __nv_bfloat16 *__restrict__ stv,
                           const int *__restrict__ g2sg,
                           const int *__restrict__ t2st,
                           __nv_bfloat16 *__restrict__ gbv,
                           const int *__restrict__ g2b) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnzL;
       e += gridDim.x * blockDim.x) {
    const int i = grow[e], j = gcol[e];
    float v;
    if (i == j) {
      v = softplus(o[i * NOUT + 1] + DIAG_OFFSET);
    } else {
      float uv = 0.f;
#pragma unroll
      for (int k = 0; k < RANK; k++)
        uv = fmaf(o[i * NOUT + 2 + k], o[j * NOUT + 2 + RANK + k], uv);
      v = fabsf(ahat[g2a[e]]) * (o[i * NOUT + 0] + uv);
    }
    ghat[e] = v;
    if (gbv) {  // the band copy of G (BF16), which serves G and G^T
      gbv[g2b[e]] = __float2bfloat16_rn((float)(dis[i] * (double)v));
    } else if (sgv) {  // the SELL-U copies of G and G^T (BF16)
      const __nv_bfloat16 bv = __float2bfloat16_rn((float)(dis[i] * (double)v));
      sgv[g2sg[e]] = bv;
      stv[t2st[g2t[e]]] = bv;
    } else if (gs) {  // FP32 CRS copies when the SELL-U layouts do not fit
      const float sv = (float)(dis[i] * (double)v);
      gs[e] = sv;
      gts[g2t[e]] = sv;
    }
  }
}

// ---------------------------------------------------------------------------
// Training: Hutchinson loss with S probe columns (node-major: V[i*S + s])

__device__ __forceinline__ void load8(const float *p, float (&v)[S]) {
  const float4 a = *reinterpret_cast<const float4 *>(p);
  const float4 b = *reinterpret_cast<const float4 *>(p + 4);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void store8(float *p, const float (&v)[S]) {
  *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  *reinterpret_cast<float4 *>(p + 4) = make_float4(v[4], v[5], v[6], v[7]);
}

// OUT = M IN for an S-column block, M in CRS with values val[map[e]] (map may
// be null: val[e]).
__global__ void k_spmm8(int N, const int *__restrict__ rp,
                        const int *__restrict__ col, const float *__restrict__ val,
                        const int *__restrict__ map, const float *__restrict__ in,
                        float *__restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x) {
    float acc[S] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int e = rp[i]; e < rp[i + 1]; e++) {
      const float a = val[map ? map[e] : e];
      float v[S];
      load8(in + (size_t)col[e] * S, v);
#pragma unroll
      for (int s = 0; s < S; s++) acc[s] = fmaf(a, v[s], acc[s]);
    }
    store8(out + (size_t)i * S, acc);
  }
}

// T3 = G^T T2 (G^T rows with values ghat[t2g[t]]), R = T3 - V,
// rho = 2 R / (N S), partial sums of R^2 -> *loss (last CTA).
__global__ void __launch_bounds__(kThreads)
    k_loss_residual(int N, const int *__restrict__ tptr,
                    const int *__restrict__ tcol, const float *__restrict__ ghat,
                    const int *__restrict__ t2g, const float *__restrict__ T2,
                    const float *__restrict__ V, float *__restrict__ rho,
                    double *partials, unsigned *ticket, float *loss) {
  const float scale = 2.f / ((float)N * S);
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x) {
    float t3[S] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int e = tptr[i]; e < tptr[i + 1]; e++) {
      const float a = ghat[t2g[e]];
      float v[S];
      load8(T2 + (size_t)tcol[e] * S, v);
#pragma unroll
      for (int s = 0; s < S; s++) t3[s] = fmaf(a, v[s], t3[s]);
    }
    float v[S], r[S];
    load8(V + (size_t)i * S, v);
#pragma unroll
    for (int s = 0; s < S; s++) {
      const float d = t3[s] - v[s];
      acc += (double)d * d;
      r[s] = scale * d;
    }
    store8(rho + (size_t)i * S, r);
  }
  double in[1] = {acc}, out[1];
  if (grid_reduce<1>(in, partials, ticket, out) && threadIdx.x == 0)
    *loss = (float)(out[0] / ((double)N * S));
}

// dGhat for every G entry e = (i, j): sum_s T2[i,s] rho[j,s] + dT1[i,s] V[j,s].
__global__ void k_grad_factor(int N, const int *__restrict__ gptr,
                              const int *__restrict__ gcol,
                              const float *__restrict__ T2,
                              const float *__restrict__ dT1,
                              const float *__restrict__ rho,
                              const float *__restrict__ V,
                              float *__restrict__ dg) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x) {
    float t2[S], d1[S];
    load8(T2 + (size_t)i * S, t2);
    load8(dT1 + (size_t)i * S, d1);
    for (int e = gptr[i]; e < gptr[i + 1]; e++) {
      const int j = gcol[e];
      float r[S], v[S];
      load8(rho + (size_t)j * S, r);
      load8(V + (size_t)j * S, v);
      float s = 0.f;
#pragma unroll
      for (int q = 0; q < S; q++) s = fmaf(t2[q], r[q], fmaf(d1[q], v[q], s));
      dg[e] = s;
    }
  }
}

// Gradient w.r.t. the head outputs o_i = [a, dg, u, v]:
//   d dg_i = dGhat_ii sigmoid(dg_i + offset)
//   d a_i  = sum_{(i,j), j<i} dGhat_ij w_ij
//   d u_i  = sum_{(i,j), j<i} dGhat_ij w_ij v_j
//   d v_j  = sum_{(i,j), i>j} dGhat_ij w_ij u_i   (over row j of G^T)
__global__ void k_grad_head_out(int N, const int *__restrict__ gptr,
                                const int *__restrict__ gcol,
                                const int *__restrict__ g2a,
                                const int *__restrict__ tptr,
                                const int *__restrict__ tcol,
                                const int *__restrict__ t2g,
                                const float *__restrict__ ahat,
                                const float *__restrict__ o,
                                const float *__restrict__ dg,
                                float *__restrict__ dO) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x) {
    float da = 0.f, ddg = 0.f, du[RANK] = {0.f, 0.f, 0.f, 0.f},
          dv[RANK] = {0.f, 0.f, 0.f, 0.f};
    for (int e = gptr[i]; e < gptr[i + 1]; e++) {
      const int j = gcol[e];
      if (j == i) {
        ddg += dg[e] * sigmoid(o[i * NOUT + 1] + DIAG_OFFSET);
      } else {
        const float c = dg[e] * fabsf(ahat[g2a[e]]);
        da += c;
#pragma unroll
        for (int k = 0; k < RANK; k++)
          du[k] = fmaf(c, o[j * NOUT + 2 + RANK + k], du[k]);
      }
    }
    for (int t = tptr[i]; t < tptr[i + 1]; t++) {
      const int r = tcol[t];  // G entry (r, i), r > i
      if (r == i) continue;
      const int e = t2g[t];
      const float c = dg[e] * fabsf(ahat[g2a[e]]);
#pragma unroll
      for (int k = 0; k < RANK; k++) dv[k] = fmaf(c, o[r * NOUT + 2 + k], dv[k]);
    }
    float *d = dO + (size_t)i * NOUT;
    d[0] = da;
    d[1] = ddg;
#pragma unroll
    for (int k = 0; k < RANK; k++) {
      d[2 + k] = du[k];
      d[2 + RANK + k] = dv[k];
    }
  }
}

// dh_i = W_h^T dO_i (FP32).
__global__ void k_grad_head_in(int N, const float *__restrict__ P,
                               const float *__restrict__ dO,
                               float *__restrict__ dh) {
  const int total = N * W;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += gridDim.x * blockDim.x) {
    const int i = t / W, f = t % W;
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < NOUT; k++)
      s = fmaf(P[OFF_WH + k * W + f], dO[(size_t)i * NOUT + k], s);
    dh[t] = s;
  }
}

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__nv_bfloat16 v) {
  return __bfloat162float(v);
}

// Per-CTA partial sums of a_i b_i^T (NA x NB) and of a_i (NA), for weight
// and bias gradients: partial[blockIdx.x][NA*NB + NA]. Rows of a and b are
// contiguous (lda = NA, ldb = NB). A fixed split of nodes over CTAs and a
// fixed order inside each makes the sums deterministic.
template <int NA, int NB, typename TB>
__global__ void __launch_bounds__(kThreads)
    k_outer_partials(int N, const float *__restrict__ a,
                     const TB *__restrict__ b, float *__restrict__ partial) {
  constexpr int CH = 32;  // nodes per chunk
  __shared__ float sa[CH][NA];
  __shared__ float sb[CH][NB];
  constexpr int NOUTS = NA * NB + NA;
  constexpr int PER = (NOUTS + kThreads - 1) / kThreads;
  float acc[PER];
#pragma unroll
  for (int q = 0; q < PER; q++) acc[q] = 0.f;
  const int chunks = (N + CH - 1) / CH;
  const int per_cta = (chunks + gridDim.x - 1) / gridDim.x;
  const int c0 = blockIdx.x * per_cta, c1 = min(chunks, c0 + per_cta);
  for (int c = c0; c < c1; c++) {
    const int n0 = c * CH;
    for (int t = threadIdx.x; t < CH * NA; t += kThreads) {
      const int r = t / NA, k = t % NA, i = n0 + r;
      sa[r][k] = i < N ? a[(size_t)i * NA + k] : 0.f;
    }
    for (int t = threadIdx.x; t < CH * NB; t += kThreads) {
      const int r = t / NB, k = t % NB, i = n0 + r;
      sb[r][k] = i < N ? to_f(b[(size_t)i * NB + k]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PER; q++) {
      const int o = threadIdx.x + q * kThreads;
      if (o < NA * NB) {
        const int fa = o / NB, fb = o % NB;
        float s = acc[q];
        for (int r = 0; r < CH; r++) s = fmaf(sa[r][fa], sb[r][fb], s);
        acc[q] = s;
      } else if (o < NOUTS) {
        const int fa = o - NA * NB;
        float s = acc[q];
        for (int r = 0; r < CH; r++) s += sa[r][fa];
        acc[q] = s;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < PER; q++) {
    const int o = threadIdx.x + q * kThreads;
    if (o < NOUTS) partial[(size_t)blockIdx.x * NOUTS + o] = acc[q];
  }
}

// out[k] = sum over CTAs of partial[cta][k], CTA order fixed.
__global__ void k_reduce_partials(int nparts, int len,
                                  const float *__restrict__ partial,
                                  float *__restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < len;
       k += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int c = 0; c < nparts; c++) s += partial[(size_t)c * len + k];
    out[k] = s;
  }
}

// Layer gradient in parameter layout: W_l[n][k] (k < W from the h block,
// k >= W from the agg block of tmp, each [W*W | W]) followed by b_l[n].
__global__ void k_pack_layer_grad(const float *__restrict__ tmp,
                                  float *__restrict__ out) {
  for (int t = threadIdx.x; t < W * 2 * W + W; t += blockDim.x) {
    if (t < W * 2 * W) {
      const int n = t / (2 * W), k = t % (2 * W);
      out[t] = k < W ? tmp[n * W + k] : tmp[(W * W + W) + n * W + (k - W)];
    } else {
      out[t] = tmp[W * W + (t - W * 2 * W)];
    }
  }
}

// Backward through one layer, part 1 (per node): dpre = dh_out * [pre > 0];
// dX = bf16(W_l)^T dpre; dself = dh_out + dX[0:W]; dagg = dX[W:2W].
__global__ void k_layer_back1(int N, const float *__restrict__ P, int layer,
                              const float *__restrict__ dh_out,
                              const float *__restrict__ pre,
                              float *__restrict__ dpre,
                              float *__restrict__ dself,
                              float *__restrict__ dagg) {
  __shared__ float sW[W][2 * W];
  const float *Wl = P + OFF_L0 + layer * L_STRIDE;
  for (int t = threadIdx.x; t < W * 2 * W; t += blockDim.x)
    sW[t / (2 * W)][t % (2 * W)] =
        __bfloat162float(__float2bfloat16_rn(Wl[t]));
  __syncthreads();
  const int total = N * W;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += gridDim.x * blockDim.x)
    dpre[t] = pre[t] > 0.f ? dh_out[t] : 0.f;
  // dX_i needs all 32 values of dpre_i, which other threads write: each
  // thread recomputes them from dh_out and pre instead of synchronising.
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += gridDim.x * blockDim.x) {
    const int i = t / W, f = t % W;
    const float *dho = dh_out + (size_t)i * W;
    const float *pr = pre + (size_t)i * W;
    float xs = 0.f, xa = 0.f;
#pragma unroll 8
    for (int n = 0; n < W; n++) {
      const float dp = pr[n] > 0.f ? dho[n] : 0.f;
      xs = fmaf(sW[n][f], dp, xs);
      xa = fmaf(sW[n][W + f], dp, xa);
    }
    dself[t] = dh_out[t] + xs;
    dagg[t] = xa;
  }
}

// Backward through one layer, part 2 (gather): dh_in_j = dself_j +
// sum_{i != j} |Ahat_ji| dagg_i (the aggregation weights are symmetric).
__global__ void k_layer_back2(int N, const int *__restrict__ ptr,
                              const int *__restrict__ index,
                              const float *__restrict__ ahat,
                              const float *__restrict__ dself,
                              const float *__restrict__ dagg,
                              float *__restrict__ dh_in) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int j = warp; j < N; j += nwarps) {
    float s = dself[(size_t)j * W + lane];
    for (int e = ptr[j]; e < ptr[j + 1]; e++) {
      const int i = index[e];
      if (i != j) s = fmaf(fabsf(ahat[e]), dagg[(size_t)i * W + lane], s);
    }
    dh_in[(size_t)j * W + lane] = s;
  }
}

// Embedding backward: dpre0 = dh0 * [pre0 > 0] (in place).
__global__ void k_relu_back(int total, const float *__restrict__ pre,
                            float *__restrict__ d) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += gridDim.x * blockDim.x)
    if (!(pre[t] > 0.f)) d[t] = 0.f;
}

// Adam (bias-corrected), in place.
__global__ void k_adam(int n, float *__restrict__ p, float *__restrict__ m,
                       float *__restrict__ v, const float *__restrict__ g,
                       float lr, float b1, float b2, float eps, int step) {
  const float c1 = 1.f - powf(b1, (float)step);
  const float c2 = 1.f - powf(b2, (float)step);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += gridDim.x * blockDim.x) {
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    p[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
  }
}

// Smoothed probe columns: for columns [c0, c1) of the S columns, V <- sc (V -
// om T) with T = Ahat V (one damped-Jacobi step on the Jacobi-scaled matrix;
// sc is the column scale, applied once after the last step).
__global__ void k_smooth_probes(int N, float *__restrict__ V,
                                const float *__restrict__ T, float om, float sc,
                                int c0, int c1) {
  const size_t n = (size_t)N * S;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % S);
    if (c >= c0 && c < c1) V[i] = sc * fmaf(-om, T[i], V[i]);
  }
}

// Residual snapshot of the solver: s = sum_i (dis_i r_i)^2 over the FP64
// residual r = b - A x; the last CTA stores the unit-RMS scale sqrt(N / s).
__global__ void __launch_bounds__(kThreads)
    k_snap_norm(int N, const double *__restrict__ r,
                const double *__restrict__ dis, double *partials,
                unsigned *ticket, double *scale) {
  double a = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads) {
    const double v = dis[i] * r[i];
    a = fma(v, v, a);
  }
  double in[1] = {a}, out[1];
  if (grid_reduce<1>(in, partials, ticket, out) && threadIdx.x == 0)
    *scale = out[0] > 0.0 ? sqrt((double)N / out[0]) : 0.0;
}

// snap[i*S + col] = dis_i r_i * scale: the Jacobi-scaled residual with unit
// RMS, the coordinates of the scaled system the probes live in.
__global__ void k_snap_store(int N, const double *__restrict__ r,
                             const double *__restrict__ dis,
                             const double *__restrict__ scale,
                             float *__restrict__ snap, int col) {
  const double sc = *scale;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x)
    snap[(size_t)i * S + col] = (float)(dis[i] * r[i] * sc);
}

// V[:, c0:S) = snap[:, c0:S) (the residual probe columns).
__global__ void k_copy_probe_cols(int N, const float *__restrict__ snap,
                                  float *__restrict__ V, int c0) {
  const size_t n = (size_t)N * S;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    if ((int)(i % S) >= c0) V[i] = snap[i];
}

// Rademacher probes from a counter-based hash: V[i*S+s] = +-1.
__global__ void k_rademacher(int N, unsigned long long seed, float *V) {
  const int total = N * S;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += gridDim.x * blockDim.x) {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(t + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    V[t] = (z & 1ull) ? 1.f : -1.f;
  }
}

}  // namespace learned
}  // namespace cgx
