// Symmetric band layout for the FP32 inner SpMV of the mixed paths.
//
// It applies when every column offset col - row of A lies in one small set D
// that is symmetric (d in D <=> -d in D) and A is symmetric. Then only the
// diagonal and the upper half are stored: U[i][k] = A(i, i + d_k) for the K
// non-negative offsets d_0 = 0 < d_1 < ... < d_{K-1} of D, zero where row i
// has no such entry, row-major with K4 = 4 floats per row (one 16-byte
// load). Row i's lower entries are read from the rows above it:
// A(i, i - d_k) = A(i - d_k, i) = U[i - d_k][k]. The 7-point structured-grid
// stencil fits (D = {0, +-1, +-n, +-n^2}): its values cost 16 bytes per row
// instead of 28 (32 with SELL-U's padding), and the lower entries come from
// rows the product read a moment earlier, which L1 and L2 still hold.
//
// The kernels here take any such offsets, one row per thread. Measured
// against them (160^3, back to back): a slot-major layout (every load of a
// slot coalesced) and warp shuffles for the +-1 neighbours were 4-40 %
// slower, because the products are bound by the latency of their loads, not
// by sectors; one 16-byte load per row beats four 4-byte ones. Kernels that
// march along z through a tile of x-y columns and take the neighbours from
// shared memory (a register ring, or a four-stage asynchronous-copy
// pipeline of planes) were 2-4 times slower still: each CTA streams a long
// dependent sequence of planes, with too few loads in flight to cover HBM
// latency.
//
// Wider sets are left to SELL-U. On the 27-point stencil (14 stored
// offsets), row-major rows of 64 bytes spread each warp's lower-entry loads
// over 16 times the sectors they use (87 us per product at 128^3, against
// 45.8 us for SELL-U), and a slot-major layout with coalesced loads only
// tied SELL-U (45.6 us): with 62 loads per row instead of 35 the product is
// bound by load issue, not by DRAM.
//
// The layout is built on the device from A's FP64 CRS (k_band_offsets,
// k_band_fill, k_band_check) and used only if the check finds the FP32
// values exactly symmetric, the pattern symmetric and no entry twice.
#pragma once

#include <cuda_bf16.h>

#include <climits>

#include "device.cuh"

namespace cgx {

constexpr int kBandMaxK = 4;     // stored offsets (diagonal + upper)
constexpr int kBandTable = 64;   // hash table of the distinct offsets
constexpr int kBandEmpty = INT_MIN;

template <int K4>
struct BandView {
  const float *U;  // N x K4, row-major
  int N;
  int d[K4];       // d[0] = 0 < d[1] < ... ; 0 for padding slots
};

// Offsets of D as the build kernels' argument.
struct BandOffsets {
  int K;
  int d[kBandMaxK];
};

__device__ __forceinline__ unsigned band_hash(int d) {
  return ((unsigned)d * 2654435761u) >> 26;  // 64 buckets
}

// Inserts d into a 64-entry open-addressing table; false if it is full.
__device__ __forceinline__ bool band_insert(int *table, int d) {
  unsigned h = band_hash(d);
  for (int probe = 0; probe < kBandTable; probe++, h = (h + 1) & (kBandTable - 1)) {
    const int v = *(volatile int *)&table[h];
    if (v == d) return true;
    if (v == kBandEmpty) {
      const int old = atomicCAS(&table[h], kBandEmpty, d);
      if (old == kBandEmpty || old == d) return true;
    }
  }
  return false;
}

// Distinct offsets col - row of all entries, collected per CTA in shared
// memory and merged into the global table. *flag |= 1 on overflow.
__global__ void __launch_bounds__(kThreads)
    k_band_offsets(int N, const int *__restrict__ ptr, const int *__restrict__ col,
                   int *table, int *flag) {
  __shared__ int local[kBandTable];
  __shared__ int full;
  if (threadIdx.x < kBandTable) local[threadIdx.x] = kBandEmpty;
  if (threadIdx.x == 0) full = 0;
  __syncthreads();
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N; i += gridDim.x * kThreads) {
    const int j1 = ptr[i + 1];
    for (int j = ptr[i]; j < j1; j++)
      if (!band_insert(local, col[j] - i)) {
        full = 1;
        break;
      }
  }
  __syncthreads();
  if (threadIdx.x < kBandTable && local[threadIdx.x] != kBandEmpty)
    if (!band_insert(table, local[threadIdx.x])) atomicOr(flag, 1);
  if (threadIdx.x == 0 && full) atomicOr(flag, 1);
}

__device__ __forceinline__ int band_slot(const BandOffsets &o, int d) {
#pragma unroll
  for (int k = 0; k < kBandMaxK; k++)
    if (k < o.K && o.d[k] == d) return k;
  return -1;
}

// U[i][k] = (float) A(i, i + d_k) for the diagonal and upper entries.
// counts[0] += upper entries (d > 0). *flag |= 2 for an offset outside D
// or an entry stored twice.
__global__ void __launch_bounds__(kThreads)
    k_band_fill(int N, const int *__restrict__ ptr, const int *__restrict__ col,
                const double *__restrict__ val, BandOffsets o,
                float *__restrict__ U, unsigned long long *counts, int *flag) {
  unsigned long long upper = 0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N; i += gridDim.x * kThreads) {
    unsigned mask = 0;
    const int j1 = ptr[i + 1];
    for (int j = ptr[i]; j < j1; j++) {
      const int d = col[j] - i;
      if (d < 0) continue;
      const int k = band_slot(o, d);
      if (k < 0 || (mask >> k) & 1u) {
        atomicOr(flag, 2);
        continue;
      }
      mask |= 1u << k;
      U[(size_t)i * kBandMaxK + k] = (float)val[j];
      upper += d > 0;
    }
  }
  for (int s = 16; s > 0; s >>= 1) upper += __shfl_xor_sync(0xffffffffu, upper, s);
  if ((threadIdx.x & 31) == 0 && upper) atomicAdd(&counts[0], upper);
}

// Every lower entry A(i, i - d) must equal U[i - d][slot of d], once per
// (i, d). counts[1] += lower entries; equal counts of upper and lower
// entries then make the pairing one to one. *flag |= 4 on a mismatch or a
// repeat.
__global__ void __launch_bounds__(kThreads)
    k_band_check(int N, const int *__restrict__ ptr, const int *__restrict__ col,
                 const double *__restrict__ val, BandOffsets o,
                 const float *__restrict__ U, unsigned long long *counts,
                 int *flag) {
  unsigned long long lower = 0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N; i += gridDim.x * kThreads) {
    unsigned mask = 0;
    const int j1 = ptr[i + 1];
    for (int j = ptr[i]; j < j1; j++) {
      const int d = i - col[j];
      if (d <= 0) continue;
      const int k = band_slot(o, d);
      if (k < 0 || (mask >> k) & 1u ||
          U[(size_t)col[j] * kBandMaxK + k] != (float)val[j]) {
        atomicOr(flag, 4);
        continue;
      }
      mask |= 1u << k;
      lower++;
    }
  }
  for (int s = 16; s > 0; s >>= 1) lower += __shfl_xor_sync(0xffffffffu, lower, s);
  if ((threadIdx.x & 31) == 0 && lower) atomicAdd(&counts[1], lower);
}

// FP32 SpMV on the band layout with the row epilogue of Op, one thread per
// row: the row's own K4 values (one 16-byte load), the upper gathers of x,
// and for each positive offset the value of the row d_k above and its x.
// All loads are unconditional: padding slots hold value 0 with offset 0,
// rows above row 0 are clamped to it and their products masked, and upper
// columns past N - 1 (value 0) are clamped. x must be finite, as it is for
// every operand of the inner solves.
template <int K4, typename Op>
__global__ void __launch_bounds__(kThreads)
    k_band(BandView<K4> B, const float *__restrict__ x, Op op, CgState *st,
           double *partials) {
  static_assert(K4 == 4, "one row of the band layout is one float4");
  if (op.skip(st)) return;
  typename Op::Acc acc;
  const int N = B.N;
  const unsigned nmax = (unsigned)(N - 1);
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N; i += gridDim.x * kThreads) {
    const typename Op::Pre pre = op.prefetch(i);
    const float4 u = __ldg(reinterpret_cast<const float4 *>(B.U) + i);
    float xu[K4], lv[K4], xl[K4];
#pragma unroll
    for (int k = 0; k < K4; k++)
      xu[k] = __ldg(&x[min((unsigned)i + (unsigned)B.d[k], nmax)]);
#pragma unroll
    for (int k = 1; k < K4; k++) {
      const int j = i - B.d[k];
      const int jc = max(j, 0);
      lv[k] = __ldg(&B.U[(size_t)jc * K4 + k]);
      xl[k] = __ldg(&x[jc]);
      lv[k] = j < 0 ? 0.f : lv[k];
    }
    float sum = fmaf(u.x, xu[0], 0.f);
    sum = fmaf(u.y, xu[1], sum);
    sum = fmaf(u.z, xu[2], sum);
    sum = fmaf(u.w, xu[3], sum);
#pragma unroll
    for (int k = 1; k < K4; k++) sum = fmaf(lv[k], xl[k], sum);
    op.row(i, sum, acc, pre);
  }
  op.finish(acc, st, partials);
}

// ---------------------------------------------------------------------------
// The learned factor G on the band: G lies on A's lower triangle, so its
// column offsets are 0, -d_1, ..., -d_{K-1}, and one BF16 array
// Gb[i][k] = G(i, i - d_k) (8 bytes per row, zero where row i has no such
// entry) serves both products of the apply:
//   z = G y:    z_i = sum_k Gb[i][k] y[i - d_k]          (the row's own values)
//   y = G^T r:  y_i = sum_k Gb[i + d_k][k] r[i + d_k]    (values of the rows below)
// Neither needs slice descriptors or offset loads: one memory round trip
// per row.

struct GBandView {
  const __nv_bfloat16 *val;  // N x 4, row-major
  int N;
  int d[kBandMaxK];          // 0 for padding slots
};

// Slot of every entry of G (CRS order): map[e] = 4 i + k for the entry
// (i, i - d_k). *flag |= 8 for an offset that is not one of -d_k.
__global__ void __launch_bounds__(kThreads)
    k_gband_map(int nnz, const int *__restrict__ grow, const int *__restrict__ gcol,
                BandOffsets o, int *__restrict__ map, int *flag) {
  for (int e = blockIdx.x * kThreads + threadIdx.x; e < nnz; e += gridDim.x * kThreads) {
    const int i = grow[e];
    const int k = band_slot(o, i - gcol[e]);
    if (k < 0) {
      atomicOr(flag, 8);
      map[e] = 4 * i;
    } else {
      map[e] = 4 * i + k;
    }
  }
}

__device__ __forceinline__ float bf16_bits_to_float(unsigned short b) {
  return __uint_as_float((unsigned)b << 16);
}

// TRANS = false: z = G x; TRANS = true: y = G^T x; with the row epilogue of
// Op. Gathers are clamped into [0, N); a clamped slot's value is 0 (G) or
// masked (G^T, rows below N - 1). x must be finite.
template <bool TRANS, typename Op>
__global__ void __launch_bounds__(kThreads)
    k_gband(GBandView B, const float *__restrict__ x, Op op, CgState *st,
            double *partials) {
  if (op.skip(st)) return;
  typename Op::Acc acc;
  const int N = B.N;
  const unsigned short *gv = reinterpret_cast<const unsigned short *>(B.val);
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N; i += gridDim.x * kThreads) {
    const typename Op::Pre pre = op.prefetch(i);
    float v[kBandMaxK], xv[kBandMaxK];
    if (!TRANS) {
      const uint2 raw = __ldg(reinterpret_cast<const uint2 *>(B.val) + i);
      v[0] = __uint_as_float(raw.x << 16);
      v[1] = __uint_as_float(raw.x & 0xffff0000u);
      v[2] = __uint_as_float(raw.y << 16);
      v[3] = __uint_as_float(raw.y & 0xffff0000u);
#pragma unroll
      for (int k = 0; k < kBandMaxK; k++) xv[k] = __ldg(&x[max(i - B.d[k], 0)]);
    } else {
      v[0] = bf16_bits_to_float(__ldg(&gv[(size_t)i * 4]));
      xv[0] = __ldg(&x[i]);
#pragma unroll
      for (int k = 1; k < kBandMaxK; k++) {
        const unsigned j = (unsigned)i + (unsigned)B.d[k];
        const int jc = (int)min(j, (unsigned)(N - 1));
        v[k] = bf16_bits_to_float(__ldg(&gv[(size_t)jc * 4 + k]));
        xv[k] = __ldg(&x[jc]);
        v[k] = j < (unsigned)N ? v[k] : 0.f;
      }
    }
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < kBandMaxK; k++) sum = fmaf(v[k], xv[k], sum);
    op.row(i, sum, acc, pre);
  }
  op.finish(acc, st, partials);
}

}  // namespace cgx
