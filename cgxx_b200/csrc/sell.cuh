// Sliced ELL with per-slice uniform offsets (SELL-U) for the FP32 inner
// solves: A's FP32 copy and the learned factor's G and G^T (BF16).
//
// Rows are taken in order in slices of 32 (lane = row). Slice s is described
// by meta[s] = {vb, w, ob, uniform}: w slots per row, stored in groups of 4
// slots per lane: slot k of row 32 s + l is value 4 (32 (vb + k / 4) + l) +
// k % 4, so one 16-byte (FP32) or 8-byte (BF16) load per lane fetches four
// slots and a warp's load of a group is one coalesced access; w is padded
// to a multiple of 4 with zero values. A slot's column is row + offset:
//  - uniform slice: one offset per slot for all 32 rows, off[ob + k]. The
//    slots are the union of the rows' column offsets in ascending order, and
//    a row without one of them holds value 0 there. A stencil-like matrix
//    (every row of a slice reaching the same relative neighbours) stores no
//    per-entry index at all, only 4 (FP32) or 2 (BF16) bytes per slot;
//  - per-row slice (rows not sorted, or the union wider than twice the
//    longest row or than 32): off[ob + 32 k + l], zero-valued padding after
//    each row's own entries.
// Gather addresses are clamped to [0, N): a zero-valued slot may name a
// column outside the matrix (a missing neighbour of a boundary row), and
// padding lanes of the last slice take row N - 1. The product of such a slot
// is 0 * x[clamped], so x must be finite, as it is for every operand of the
// inner solves.
//
// The layout is built on the device from a CRS pattern whose rows need not
// be sorted (k_sellu_plan, k_sellu_fill); map[e] gives the value slot of CRS
// entry e, so new values of the same pattern are scattered with
// k_sellu_scatter.
#pragma once

#include <cuda_bf16.h>

#include <climits>

#include "device.cuh"

namespace cgx {

__device__ __forceinline__ int warp_min_int(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ int warp_max_int(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ float to_float(float v) { return v; }
__device__ __forceinline__ float to_float(__nv_bfloat16 v) {
  return __bfloat162float(v);
}

// Four consecutive slots of one lane (16 bytes of FP32, 8 of BF16). The
// values are read once per product, so they bypass L1 (no_allocate) and
// leave it to the gathers of x, whose windows neighbouring slices share.
__device__ __forceinline__ float4 load_group(const float *p) {
  float4 v;
  asm("ld.global.nc.L1::no_allocate.v4.f32 {%0,%1,%2,%3}, [%4];"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "l"(p));
  return v;
}
__device__ __forceinline__ float4 load_group(const __nv_bfloat16 *p) {
  uint2 u;
  asm("ld.global.nc.L1::no_allocate.v2.u32 {%0,%1}, [%2];"
      : "=r"(u.x), "=r"(u.y)
      : "l"(p));
  return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u),
                     __uint_as_float(u.y << 16), __uint_as_float(u.y & 0xffff0000u));
}

// SELL-U SpMV with the row epilogue of Op (the same Ops as k_crs, with the
// row's own operands prefetched). Warps take SPW slices per step
// (grid-stride, so the warps of the grid sweep the value array together)
// and load the next step's slice meta one step ahead: two slices on a
// uniform layout, one on a layout with per-row slices, whose steps run to
// the wider slice's width (measured on the 2M-point geometric graph's
// factor: the learned solve 43.4 against 46.2 ms with one slice per warp;
// chunks of 16 slots instead of 8, 47.6 ms). A
// uniform slice is processed in chunks of U slots whose loads are all
// unconditional: groups and gathers past the slice's width re-read its last
// ones (L1 hits) and are masked out, so every value load and gather of a
// chunk is issued before the first multiply-add (predicated loads would
// split the chunk into branches and serialize the round trips). Steps whose
// slices are all per-row take the same chunks with per-entry offset loads;
// a step that mixes both kinds takes a plain loop.
template <typename VT>
struct SellUView {
  const int4 *meta;  // per slice {vb (groups), w (slots), ob, uniform}
  const int *off;
  const VT *val;
  int N;
};

// Gathers of x: through the read-only path (a kernel whose x is not written
// while it runs), or with weak loads (a persistent launch, whose x another
// CTA wrote before the last grid barrier).
struct GatherLdg {
  __device__ float operator()(const float *p) const { return __ldg(p); }
};
struct GatherWeak {
  __device__ float operator()(const float *p) const { return __ldca(p); }
};

// The product's row loop over TPB-wide CTAs (k_sellu's body).
// ALL_UNIFORM: the layout has no per-row slice, and its instantiation
// leaves out the chunked per-row path (measured: carrying it costs the
// uniform kernels 1-3 %).
template <typename VT, int U, bool ALL_UNIFORM, int TPB, typename XL, typename Op>
__device__ __forceinline__ void sellu_rows(const SellUView<VT> &A, const float *x, XL xld,
                                           const Op &op, typename Op::Acc &acc) {
  constexpr int SPW = ALL_UNIFORM ? 2 : 1, NG = U / 4;
  const int lane = threadIdx.x & 31;
  const int nslices = (A.N + 31) >> 5;
  const int nwarps = (gridDim.x * TPB) >> 5;
  const int stride = nwarps * SPW;
  auto meta_of = [&](int s0) {
    return (lane < SPW && s0 + lane < nslices) ? __ldg(&A.meta[s0 + lane])
                                                : make_int4(0, 0, 0, 0);
  };
  int s0 = ((blockIdx.x * TPB + threadIdx.x) >> 5) * SPW;
  int4 ml = meta_of(s0);
  for (; s0 < nslices; s0 += stride) {
    const int4 mn = meta_of(s0 + stride);
    int vb[SPW], w[SPW], ob[SPW], uni[SPW], row[SPW];
    bool fast = true, perrow = true;
    int wmax = 0;
#pragma unroll
    for (int q = 0; q < SPW; q++) {
      vb[q] = __shfl_sync(0xffffffffu, ml.x, q);
      w[q] = __shfl_sync(0xffffffffu, ml.y, q);
      ob[q] = __shfl_sync(0xffffffffu, ml.z, q);
      uni[q] = __shfl_sync(0xffffffffu, ml.w, q);
      row[q] = ((s0 + q) << 5) + lane;
      fast = fast && (uni[q] || w[q] == 0);
      perrow = !ALL_UNIFORM && perrow && (!uni[q] || w[q] == 0);
      wmax = max(wmax, w[q]);
    }
    typename Op::Pre pre[SPW];
#pragma unroll
    for (int q = 0; q < SPW; q++) pre[q] = op.prefetch(min(row[q], A.N - 1));
    float sum[SPW];
#pragma unroll
    for (int q = 0; q < SPW; q++) sum[q] = 0.f;
    if (fast) {
      // Slots past a slice's width: inside its last group they hold value 0
      // and offset 0 (lanes >= w of ol load 0); whole groups past it re-read
      // the last group and are zeroed. Gathers are clamped to [0, N) with one
      // unsigned min (a negative column wraps to a large value).
      int ol[SPW], ng[SPW];
#pragma unroll
      for (int q = 0; q < SPW; q++) {
        ol[q] = lane < w[q] ? __ldg(&A.off[ob[q] + lane]) : 0;
        ng[q] = (w[q] + 3) >> 2;
      }
      const unsigned nmax = (unsigned)(A.N - 1);
      for (int k0 = 0; k0 < wmax; k0 += U) {
        float4 a[SPW][NG];
        float b[SPW][U];
#pragma unroll
        for (int q = 0; q < SPW; q++) {
#pragma unroll
          for (int g = 0; g < NG; g++) {
            const int gi = (k0 >> 2) + g;
            a[q][g] = load_group(A.val + ((((vb[q] + min(gi, max(ng[q] - 1, 0))) << 5) + lane) << 2));
          }
#pragma unroll
          for (int u = 0; u < U; u++) {
            const int o = __shfl_sync(0xffffffffu, ol[q], (k0 + u) & 31);
            b[q][u] = xld(&x[min((unsigned)(row[q] + o), nmax)]);
          }
        }
#pragma unroll
        for (int q = 0; q < SPW; q++)
#pragma unroll
          for (int g = 0; g < NG; g++) {
            const float4 v = (k0 >> 2) + g < ng[q] ? a[q][g] : make_float4(0.f, 0.f, 0.f, 0.f);
            sum[q] = fmaf(v.x, b[q][4 * g + 0], sum[q]);
            sum[q] = fmaf(v.y, b[q][4 * g + 1], sum[q]);
            sum[q] = fmaf(v.z, b[q][4 * g + 2], sum[q]);
            sum[q] = fmaf(v.w, b[q][4 * g + 3], sum[q]);
          }
      }
    } else if (perrow) {
      // Per-row slices, the same chunks: a slot's offset is the lane's own
      // (one coalesced load per slot, clamped to the slice's last slot), and
      // all offset loads of a chunk are issued before its gathers.
      int ng[SPW];
#pragma unroll
      for (int q = 0; q < SPW; q++) ng[q] = (w[q] + 3) >> 2;
      const unsigned nmax = (unsigned)(A.N - 1);
      for (int k0 = 0; k0 < wmax; k0 += U) {
        float4 a[SPW][NG];
        int o[SPW][U];
        float b[SPW][U];
#pragma unroll
        for (int q = 0; q < SPW; q++) {
#pragma unroll
          for (int g = 0; g < NG; g++) {
            const int gi = (k0 >> 2) + g;
            a[q][g] = load_group(A.val + ((((vb[q] + min(gi, max(ng[q] - 1, 0))) << 5) + lane) << 2));
          }
#pragma unroll
          for (int u = 0; u < U; u++) {
            const int kk = min(k0 + u, max(w[q] - 1, 0));
            o[q][u] = w[q] > 0 ? __ldg(&A.off[ob[q] + (kk << 5) + lane]) : 0;
          }
        }
#pragma unroll
        for (int q = 0; q < SPW; q++)
#pragma unroll
          for (int u = 0; u < U; u++)
            b[q][u] = xld(&x[min((unsigned)(row[q] + o[q][u]), nmax)]);
#pragma unroll
        for (int q = 0; q < SPW; q++)
#pragma unroll
          for (int g = 0; g < NG; g++) {
            const float4 v = (k0 >> 2) + g < ng[q] ? a[q][g] : make_float4(0.f, 0.f, 0.f, 0.f);
            sum[q] = fmaf(v.x, b[q][4 * g + 0], sum[q]);
            sum[q] = fmaf(v.y, b[q][4 * g + 1], sum[q]);
            sum[q] = fmaf(v.z, b[q][4 * g + 2], sum[q]);
            sum[q] = fmaf(v.w, b[q][4 * g + 3], sum[q]);
          }
      }
    } else {
#pragma unroll
      for (int q = 0; q < SPW; q++) {
        const int olq = (uni[q] && lane < w[q]) ? __ldg(&A.off[ob[q] + lane]) : 0;
        float t = 0.f;
        for (int k = 0; k < w[q]; k++) {
          const int o = uni[q] ? __shfl_sync(0xffffffffu, olq, k & 31)
                               : __ldg(&A.off[ob[q] + (k << 5) + lane]);
          const float v = to_float(
              __ldg(A.val + ((((vb[q] + (k >> 2)) << 5) + lane) << 2) + (k & 3)));
          t = fmaf(v, xld(&x[min(max(row[q] + o, 0), A.N - 1)]), t);
        }
        sum[q] = t;
      }
    }
#pragma unroll
    for (int q = 0; q < SPW; q++)
      if (row[q] < A.N) op.row(row[q], sum[q], acc, pre[q]);
    ml = mn;
  }
}

template <typename VT, int U, bool ALL_UNIFORM, typename Op>
__global__ void __launch_bounds__(kThreads)
    k_sellu(SellUView<VT> A, const float *__restrict__ x, Op op, CgState *st,
            double *partials) {
  if (op.skip(st)) return;
  typename Op::Acc acc;
  sellu_rows<VT, U, ALL_UNIFORM, kThreads>(A, x, GatherLdg{}, op, acc);
  op.finish(acc, st, partials);
}

// ---------------------------------------------------------------------------
// Build (a warp per slice). The union of a slice's column offsets is merged
// from the rows' sorted offsets: each step takes the smallest head over the
// lanes, and the lanes holding it advance.

// Plan: per slice the slot count w (wid), its groups of 4 (gcnt), the
// offset count (ocnt: w for a uniform slice, 32 w for a per-row one) and the
// kind (uni); tot[0] and tot[1] accumulate the gcnt and ocnt totals (64-bit,
// for the size checks before the int scans), tot[2] the number of uniform
// slices, tot[3] the largest slot count.
__global__ void k_sellu_plan(int N, const int *__restrict__ ptr,
                             const int *__restrict__ col, int *__restrict__ wid,
                             int *__restrict__ gcnt, int *__restrict__ ocnt,
                             int *__restrict__ uni, unsigned long long *tot) {
  const int lane = threadIdx.x & 31;
  const int nsl = (N + 31) >> 5;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nsl;
       s += (gridDim.x * blockDim.x) >> 5) {
    const int r = (s << 5) + lane;
    int j = 0, j1 = 0;
    if (r < N) {
      j = ptr[r];
      j1 = ptr[r + 1];
    }
    bool sorted = true;
    for (int t = j + 1; t < j1; t++)
      if (col[t] <= col[t - 1]) {
        sorted = false;
        break;
      }
    const int wmax = warp_max_int(j1 - j);
    const int cap = min(32, 2 * wmax);
    int wu = 0;
    const bool all_sorted = __all_sync(0xffffffffu, sorted);
    if (all_sorted) {
      while (wu <= cap) {
        const int my = j < j1 ? col[j] - r : INT_MAX;
        const int m = warp_min_int(my);
        if (m == INT_MAX) break;
        if (my == m) j++;
        wu++;
      }
    }
    const bool u = all_sorted && wmax > 0 && wu <= cap;
    if (lane == 0) {
      const int w = u ? wu : wmax, oc = u ? wu : 32 * wmax;
      wid[s] = w;
      gcnt[s] = (w + 3) >> 2;
      ocnt[s] = oc;
      uni[s] = u ? 1 : 0;
      atomicAdd(&tot[0], (unsigned long long)((w + 3) >> 2));
      atomicAdd(&tot[1], (unsigned long long)oc);
      if (u) atomicAdd(&tot[2], 1ull);
      atomicMax(&tot[3], (unsigned long long)w);
    }
  }
}

// Value index of slot k of lane l in a slice whose groups start at vb.
__host__ __device__ inline int sellu_slot(int vb, int k, int l) {
  return ((((vb + (k >> 2)) << 5) + l) << 2) + (k & 3);
}

// Fill: meta, offsets and the value slot of every CRS entry; vb and ob are
// the exclusive scans of gcnt and ocnt. Offsets of per-row padding keep the
// zero they were cleared to.
__global__ void k_sellu_fill(int N, const int *__restrict__ ptr,
                             const int *__restrict__ col,
                             const int *__restrict__ vb,
                             const int *__restrict__ ob,
                             const int *__restrict__ wid,
                             const int *__restrict__ uni, int4 *__restrict__ meta,
                             int *__restrict__ off, int *__restrict__ map) {
  const int lane = threadIdx.x & 31;
  const int nsl = (N + 31) >> 5;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nsl;
       s += (gridDim.x * blockDim.x) >> 5) {
    const int r = (s << 5) + lane;
    int j = 0, j1 = 0;
    if (r < N) {
      j = ptr[r];
      j1 = ptr[r + 1];
    }
    const int v0 = vb[s], o0 = ob[s], w = wid[s], u = uni[s];
    if (lane == 0) meta[s] = make_int4(v0, w, o0, u);
    if (u) {
      for (int k = 0; k < w; k++) {
        const int my = j < j1 ? col[j] - r : INT_MAX;
        const int m = warp_min_int(my);
        if (lane == 0) off[o0 + k] = m;
        if (my == m) {
          map[j] = sellu_slot(v0, k, lane);
          j++;
        }
      }
    } else {
      for (int k = 0; k < j1 - j; k++) {
        off[o0 + (k << 5) + lane] = col[j + k] - r;
        map[j + k] = sellu_slot(v0, k, lane);
      }
    }
  }
}

// New values of the same pattern: out[map[e]] = in[e] (padding slots keep
// their zero).
template <typename In, typename Out>
__global__ void k_sellu_scatter(size_t nnz, const int *__restrict__ map,
                                const In *__restrict__ in, Out *__restrict__ out) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nnz;
       e += (size_t)gridDim.x * blockDim.x)
    out[map[e]] = (Out)in[e];
}

}  // namespace cgx
