// Symmetric band layout for the FP32 inner SpMV of the mixed paths.
//
// It applies when every column offset col - row of A lies in one small set D
// that is symmetric (d in D <=> -d in D) and A is symmetric. Then only the
// diagonal and the upper half are stored: U_k[i] = A(i, i + d_k) for the K
// non-negative offsets d_0 = 0 < d_1 < ... < d_{K-1} of D, zero where row i
// has no such entry. Row i's lower entries are read from the rows above it:
// A(i, i - d_k) = A(i - d_k, i) = U_k[i - d_k]. The 7-point structured-grid
// stencil fits (D = {0, +-1, +-n, +-n^2}): its values cost 16 bytes per row
// instead of 28 (32 with SELL-U's padding), and the lower entries come from
// rows the product read a moment earlier, which L1 and L2 still hold.
//
// Slot-major storage: slot k of every row is one array (U_k[i] at
// U[k * ld + i]). A warp owns 32 consecutive rows, so each of its loads of a
// slot -- the row's own values and the lower entries U_k[i - d_k] -- is one
// coalesced 128-byte access, where a row-major layout spreads the lower-entry
// loads over four times the sectors they use. When d_1 = 1 (every structured
// grid numbered x fastest), the x and U_1 values of rows i - 1 and i + 1 are
// the adjacent lanes' own values, passed by warp shuffles; only the two rows
// past the warp's ends take a (broadcast) load.
//
// Wider sets are left to SELL-U. On the 27-point stencil (14 stored
// offsets), the product is bound by load issue (62 loads per row against
// SELL-U's 35), not by DRAM; a band form measured no faster than SELL-U.
//
// The layout is built on the device from A's FP64 CRS (k_band_offsets,
// k_band_fill, k_band_check) and used only if the check finds the FP32
// values exactly symmetric, the pattern symmetric and no entry twice.
//
// Fused inner iterations. On the band, one inner PCG iteration of the mixed
// paths runs as
//   k_band_dir:   p = z + b p_old, d += a_old p_old, q = A p, <p,q> -> a
//   (Jacobi)      k_inner_update_jz: r -= a q, z = C r, <r,r>, <r,z> -> test, b
//   (learned)     k_gband_res: r = r_old - a q, y = G^T r, <r,r> -> test
//                 k_gband<false>: z = G y + eps C r, <r,z> -> b
// The products read p and r of neighbouring rows; those values are formed
// from the previous iteration's vectors by every thread that needs them (the
// same single-rounding operations as the owner's, so the same bits), and the
// new vectors go to the other buffer of a ping-pong pair. The update of d
// lags one iteration (it needs p_old, which the next k_band_dir reads
// anyway); the refinement step's epilogue applies the last one.
#pragma once

#include <cuda_bf16.h>

#include <climits>

#include "device.cuh"

namespace cgx {

constexpr int kBandMaxK = 4;     // stored offsets (diagonal + upper)
constexpr int kBandTable = 64;   // hash table of the distinct offsets
constexpr int kBandEmpty = INT_MIN;
constexpr unsigned kFullMask = 0xffffffffu;

// Elements per slot of a slot-major band array for N rows: N rounded up to
// a multiple of 64 (every slot starts 256-byte aligned for FP32).
__host__ __device__ inline size_t band_ld(int N) {
  return ((size_t)N + 63) / 64 * 64;
}

template <int K4>
struct BandView {
  const float *U;  // K4 slots, slot k at U + k * ld
  size_t ld;
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

// U_k[i] = (float) A(i, i + d_k) for the diagonal and upper entries.
// counts[0] += upper entries (d > 0). *flag |= 2 for an offset outside D
// or an entry stored twice.
__global__ void __launch_bounds__(kThreads)
    k_band_fill(int N, const int *__restrict__ ptr, const int *__restrict__ col,
                const double *__restrict__ val, BandOffsets o, size_t ld,
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
      U[(size_t)k * ld + i] = (float)val[j];
      upper += d > 0;
    }
  }
  for (int s = 16; s > 0; s >>= 1) upper += __shfl_xor_sync(kFullMask, upper, s);
  if ((threadIdx.x & 31) == 0 && upper) atomicAdd(&counts[0], upper);
}

// Every lower entry A(i, i - d) must equal U_k[i - d] (k the slot of d),
// once per (i, d). counts[1] += lower entries; equal counts of upper and
// lower entries then make the pairing one to one. *flag |= 4 on a mismatch
// or a repeat.
__global__ void __launch_bounds__(kThreads)
    k_band_check(int N, const int *__restrict__ ptr, const int *__restrict__ col,
                 const double *__restrict__ val, BandOffsets o, size_t ld,
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
          U[(size_t)k * ld + col[j]] != (float)val[j]) {
        atomicOr(flag, 4);
        continue;
      }
      mask |= 1u << k;
      lower++;
    }
  }
  for (int s = 16; s > 0; s >>= 1) lower += __shfl_xor_sync(kFullMask, lower, s);
  if ((threadIdx.x & 31) == 0 && lower) atomicAdd(&counts[1], lower);
}

// --- warp neighbours ----------------------------------------------------------
// A warp holds rows base .. base + 31 in lanes 0 .. 31 (base a multiple of 32,
// rows past N - 1 clamped to it). Given each lane's value v of an array a at
// its own row, these return the value at the next / previous row: from the
// adjacent lane, or, for the lane at the warp's end, from one load of the row
// past it (the same address in every lane: one broadcast access). Rows
// outside [0, N) are clamped; callers mask the products that need it.

__device__ __forceinline__ float lane_next(float v, float edge) {
  const float s = __shfl_down_sync(kFullMask, v, 1);
  return (threadIdx.x & 31) == 31 ? edge : s;
}

__device__ __forceinline__ float lane_prev(float v, float edge) {
  const float s = __shfl_up_sync(kFullMask, v, 1);
  return (threadIdx.x & 31) == 0 ? edge : s;
}

// Row after the warp's last lane, clamped to N - 1 (no int overflow).
__device__ __forceinline__ int warp_hi(int base, int nmax) {
  return (int)min((unsigned)base + 32u, (unsigned)nmax);
}

__device__ __forceinline__ int warp_lo(int base) { return max(base - 1, 0); }

// FP32 y = A x on the band with the row epilogue of Op (Op::row_x receives
// x_i, which the product loads anyway). D1: d_1 = 1, whose neighbours come
// from the adjacent lanes. All loads are unconditional: padding slots hold
// value 0 with offset 0, rows above row 0 are clamped to it and their
// products masked, and upper columns past N - 1 (value 0) are clamped. x
// must be finite, as it is for every operand of the inner solves.
template <bool D1, typename Op>
__global__ void __launch_bounds__(kThreads)
    k_band(BandView<4> B, const float *__restrict__ x, Op op, CgState *st,
           double *partials) {
  if (op.skip(st)) return;
  typename Op::Acc acc;
  const int N = B.N, nmax = N - 1;
  const size_t ld = B.ld;
  const float *U0 = B.U, *U1 = B.U + ld, *U2 = B.U + 2 * ld, *U3 = B.U + 3 * ld;
  const unsigned un = (unsigned)nmax;
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * kThreads + (threadIdx.x & ~31); base < N;
       base += gridDim.x * kThreads) {
    const int i = base + lane, ic = min(i, nmax);
    const float u0 = __ldg(U0 + ic), u1 = __ldg(U1 + ic);
    const float u2 = __ldg(U2 + ic), u3 = __ldg(U3 + ic);
    const float x0 = __ldg(x + ic);
    float xu1, xl1, lv1;
    if (D1) {
      const int hi = warp_hi(base, nmax), lo = warp_lo(base);
      xu1 = lane_next(x0, __ldg(x + hi));
      xl1 = lane_prev(x0, __ldg(x + lo));
      lv1 = lane_prev(u1, __ldg(U1 + lo));
      lv1 = i < 1 ? 0.f : lv1;
    } else {
      xu1 = __ldg(x + min((unsigned)ic + (unsigned)B.d[1], un));
      const int j = ic - B.d[1], jc = max(j, 0);
      lv1 = __ldg(U1 + jc);
      xl1 = __ldg(x + jc);
      lv1 = j < 0 ? 0.f : lv1;
    }
    const float xu2 = __ldg(x + min((unsigned)ic + (unsigned)B.d[2], un));
    const float xu3 = __ldg(x + min((unsigned)ic + (unsigned)B.d[3], un));
    const int j2 = ic - B.d[2], j2c = max(j2, 0);
    const int j3 = ic - B.d[3], j3c = max(j3, 0);
    float lv2 = __ldg(U2 + j2c), lv3 = __ldg(U3 + j3c);
    const float xl2 = __ldg(x + j2c), xl3 = __ldg(x + j3c);
    lv2 = j2 < 0 ? 0.f : lv2;
    lv3 = j3 < 0 ? 0.f : lv3;
    float sum = fmaf(u0, x0, 0.f);
    sum = fmaf(u1, xu1, sum);
    sum = fmaf(u2, xu2, sum);
    sum = fmaf(u3, xu3, sum);
    sum = fmaf(lv1, xl1, sum);
    sum = fmaf(lv2, xl2, sum);
    sum = fmaf(lv3, xl3, sum);
    if (i < N) op.row_x(i, sum, acc, x0);
  }
  op.finish(acc, st, partials);
}

// Step 1 of a fused inner iteration on the band (both mixed paths):
//   p = z + b p_old      for the own row, and for every neighbour row the
//                        product reads (formed from z and p_old there);
//   d += a_old p_old     (the previous iteration's update of d);
//   q = A p, partials of <p,q>; last CTA: a = rho / <p,q>.
// p goes to the other buffer of the ping-pong pair: p_old is read by other
// rows' threads while this kernel runs. The first iteration of an inner
// solve runs with a_old = b = 0 and p_old = z, so that p = z and d stays 0.
struct DirArgs {
  const float *z;     // preconditioned residual
  const float *pold;  // search direction of the last iteration
  float *pnew;        // the new search direction
  float *d;           // inner solution
  float *q;           // A p
  unsigned *ticket;
  int pnew_slot;      // which buffer of the pair pnew is (0 or 1)
};

template <bool D1>
__global__ void __launch_bounds__(kThreads)
    k_band_dir(BandView<4> B, DirArgs a, CgState *st, double *partials) {
  if (st->in_stop) return;
  const float al = (float)st->in_alpha, be = (float)st->in_beta;
  const int N = B.N, nmax = N - 1;
  const size_t ld = B.ld;
  const float *U0 = B.U, *U1 = B.U + ld, *U2 = B.U + 2 * ld, *U3 = B.U + 3 * ld;
  const float *__restrict__ z = a.z;
  const float *__restrict__ pold = a.pold;
  const unsigned un = (unsigned)nmax;
  const int lane = threadIdx.x & 31;
  double acc = 0.0;
  for (int base = blockIdx.x * kThreads + (threadIdx.x & ~31); base < N;
       base += gridDim.x * kThreads) {
    const int i = base + lane, ic = min(i, nmax);
    const float u0 = __ldg(U0 + ic), u1 = __ldg(U1 + ic);
    const float u2 = __ldg(U2 + ic), u3 = __ldg(U3 + ic);
    const float po = __ldg(pold + ic);
    const float p0 = fmaf(be, po, __ldg(z + ic));
    float pu1, pl1, lv1;
    if (D1) {
      const int hi = warp_hi(base, nmax), lo = warp_lo(base);
      pu1 = lane_next(p0, fmaf(be, __ldg(pold + hi), __ldg(z + hi)));
      pl1 = lane_prev(p0, fmaf(be, __ldg(pold + lo), __ldg(z + lo)));
      lv1 = lane_prev(u1, __ldg(U1 + lo));
      lv1 = i < 1 ? 0.f : lv1;
    } else {
      const int ju = (int)min((unsigned)ic + (unsigned)B.d[1], un);
      pu1 = fmaf(be, __ldg(pold + ju), __ldg(z + ju));
      const int j = ic - B.d[1], jc = max(j, 0);
      lv1 = __ldg(U1 + jc);
      pl1 = fmaf(be, __ldg(pold + jc), __ldg(z + jc));
      lv1 = j < 0 ? 0.f : lv1;
    }
    const int ju2 = (int)min((unsigned)ic + (unsigned)B.d[2], un);
    const int ju3 = (int)min((unsigned)ic + (unsigned)B.d[3], un);
    const int j2 = ic - B.d[2], j2c = max(j2, 0);
    const int j3 = ic - B.d[3], j3c = max(j3, 0);
    const float pu2 = fmaf(be, __ldg(pold + ju2), __ldg(z + ju2));
    const float pu3 = fmaf(be, __ldg(pold + ju3), __ldg(z + ju3));
    float lv2 = __ldg(U2 + j2c), lv3 = __ldg(U3 + j3c);
    const float pl2 = fmaf(be, __ldg(pold + j2c), __ldg(z + j2c));
    const float pl3 = fmaf(be, __ldg(pold + j3c), __ldg(z + j3c));
    lv2 = j2 < 0 ? 0.f : lv2;
    lv3 = j3 < 0 ? 0.f : lv3;
    float sum = fmaf(u0, p0, 0.f);
    sum = fmaf(u1, pu1, sum);
    sum = fmaf(u2, pu2, sum);
    sum = fmaf(u3, pu3, sum);
    sum = fmaf(lv1, pl1, sum);
    sum = fmaf(lv2, pl2, sum);
    sum = fmaf(lv3, pl3, sum);
    if (i < N) {
      a.d[i] = fmaf(al, po, a.d[i]);
      a.pnew[i] = p0;
      a.q[i] = sum;
      acc = fma((double)p0, (double)sum, acc);
    }
  }
  double in[1] = {acc}, out[1];
  if (grid_reduce<1>(in, partials, a.ticket, out) && threadIdx.x == 0) {
    st->in_alpha = st->in_rho / out[0];
    st->in_pslot = a.pnew_slot;
  }
}

// ---------------------------------------------------------------------------
// The learned factor G on the band: G lies on A's lower triangle, so its
// column offsets are 0, -d_1, ..., -d_{K-1}, and one slot-major BF16 array
// Gb_k[i] = G(i, i - d_k) (8 bytes per row, zero where row i has no such
// entry) serves both products of the apply:
//   z = G y:    z_i = sum_k Gb_k[i] y[i - d_k]             (the row's own values)
//   y = G^T r:  y_i = sum_k Gb_k[i + d_k] r[i + d_k]       (values of the rows below)
// Neither needs slice descriptors or offset loads: one memory round trip
// per row, and every load of a slot is coalesced across the warp.

struct GBandView {
  const __nv_bfloat16 *val;  // 4 slots, slot k at val + k * ld
  size_t ld;
  int N;
  int d[kBandMaxK];          // 0 for padding slots
};

// Slot of every entry of G (CRS order): map[e] = k * ld + i for the entry
// (i, i - d_k). *flag |= 8 for an offset that is not one of -d_k.
__global__ void __launch_bounds__(kThreads)
    k_gband_map(int nnz, const int *__restrict__ grow, const int *__restrict__ gcol,
                BandOffsets o, size_t ld, int *__restrict__ map, int *flag) {
  for (int e = blockIdx.x * kThreads + threadIdx.x; e < nnz; e += gridDim.x * kThreads) {
    const int i = grow[e];
    const int k = band_slot(o, i - gcol[e]);
    if (k < 0) {
      atomicOr(flag, 8);
      map[e] = i;
    } else {
      map[e] = (int)((size_t)k * ld + i);
    }
  }
}

__device__ __forceinline__ float bf16_bits_to_float(unsigned short b) {
  return __uint_as_float((unsigned)b << 16);
}

__device__ __forceinline__ float ld_bf16(const unsigned short *p) {
  return bf16_bits_to_float(__ldg(p));
}

// TRANS = false: z = G x; TRANS = true: y = G^T x; with the row epilogue of
// Op (its prefetch takes the clamped row). Gathers are clamped into [0, N);
// a clamped slot's value is 0 (G) or masked (G^T, rows below N - 1). x must
// be finite.
template <bool TRANS, bool D1, typename Op>
__global__ void __launch_bounds__(kThreads)
    k_gband(GBandView B, const float *__restrict__ x, Op op, CgState *st,
            double *partials) {
  if (op.skip(st)) return;
  typename Op::Acc acc;
  const int N = B.N, nmax = N - 1;
  const unsigned un = (unsigned)nmax;
  const size_t ld = B.ld;
  const unsigned short *g0 = reinterpret_cast<const unsigned short *>(B.val);
  const unsigned short *g1 = g0 + ld, *g2 = g0 + 2 * ld, *g3 = g0 + 3 * ld;
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * kThreads + (threadIdx.x & ~31); base < N;
       base += gridDim.x * kThreads) {
    const int i = base + lane, ic = min(i, nmax);
    const typename Op::Pre pre = op.prefetch(ic);
    const float x0 = __ldg(x + ic);
    float v0, v1, v2, v3, x1, x2, x3;
    if (!TRANS) {
      v0 = ld_bf16(g0 + ic);
      v1 = ld_bf16(g1 + ic);
      v2 = ld_bf16(g2 + ic);
      v3 = ld_bf16(g3 + ic);
      x1 = D1 ? lane_prev(x0, __ldg(x + warp_lo(base)))
              : __ldg(x + max(ic - B.d[1], 0));
      x2 = __ldg(x + max(ic - B.d[2], 0));
      x3 = __ldg(x + max(ic - B.d[3], 0));
    } else {
      v0 = ld_bf16(g0 + ic);
      if (D1) {
        const int hi = warp_hi(base, nmax);
        v1 = lane_next(ld_bf16(g1 + ic), ld_bf16(g1 + hi));
        x1 = lane_next(x0, __ldg(x + hi));
        v1 = (unsigned)i + 1u < (unsigned)N ? v1 : 0.f;
      } else {
        const unsigned j = (unsigned)ic + (unsigned)B.d[1];
        const int jc = (int)min(j, un);
        v1 = ld_bf16(g1 + jc);
        x1 = __ldg(x + jc);
        v1 = j < (unsigned)N ? v1 : 0.f;
      }
      const unsigned j2 = (unsigned)ic + (unsigned)B.d[2];
      const unsigned j3 = (unsigned)ic + (unsigned)B.d[3];
      const int j2c = (int)min(j2, un), j3c = (int)min(j3, un);
      v2 = ld_bf16(g2 + j2c);
      v3 = ld_bf16(g3 + j3c);
      x2 = __ldg(x + j2c);
      x3 = __ldg(x + j3c);
      v2 = j2 < (unsigned)N ? v2 : 0.f;
      v3 = j3 < (unsigned)N ? v3 : 0.f;
    }
    float sum = fmaf(v0, x0, 0.f);
    sum = fmaf(v1, x1, sum);
    sum = fmaf(v2, x2, sum);
    sum = fmaf(v3, x3, sum);
    if (i < N) op.row(i, sum, acc, pre);
  }
  op.finish(acc, st, partials);
}

// Step 2 of a fused learned inner iteration on the band:
//   r = r_old - a q      for the own row, and for the rows below that G^T
//                        reads (formed from r_old and q there);
//   y = G^T r, partials of <r,r>; last CTA: inner residual test, stop flag,
//   graph condition.
// r goes to the other buffer of the ping-pong pair. The r values are the
// same single-rounding fmaf(-a, q, r_old) as the unfused update's.
struct ResArgs {
  const float *rold;  // residual of the last iteration
  const float *q;     // A p of this iteration
  float *rnew;        // the new residual
  float *y;           // G^T r
  unsigned *ticket;
};

template <bool D1>
__global__ void __launch_bounds__(kThreads)
    k_gband_res(GBandView B, ResArgs a, CgState *st, double *partials) {
  if (st->in_stop) return;
  const float na = (float)(-st->in_alpha);
  const int N = B.N, nmax = N - 1;
  const unsigned un = (unsigned)nmax;
  const size_t ld = B.ld;
  const unsigned short *g0 = reinterpret_cast<const unsigned short *>(B.val);
  const unsigned short *g1 = g0 + ld, *g2 = g0 + 2 * ld, *g3 = g0 + 3 * ld;
  const float *__restrict__ rold = a.rold;
  const float *__restrict__ q = a.q;
  const int lane = threadIdx.x & 31;
  double rr = 0.0;
  for (int base = blockIdx.x * kThreads + (threadIdx.x & ~31); base < N;
       base += gridDim.x * kThreads) {
    const int i = base + lane, ic = min(i, nmax);
    const float r0 = fmaf(na, __ldg(q + ic), __ldg(rold + ic));
    const float v0 = ld_bf16(g0 + ic);
    float v1, x1;
    if (D1) {
      const int hi = warp_hi(base, nmax);
      v1 = lane_next(ld_bf16(g1 + ic), ld_bf16(g1 + hi));
      x1 = lane_next(r0, fmaf(na, __ldg(q + hi), __ldg(rold + hi)));
      v1 = (unsigned)i + 1u < (unsigned)N ? v1 : 0.f;
    } else {
      const unsigned j = (unsigned)ic + (unsigned)B.d[1];
      const int jc = (int)min(j, un);
      v1 = ld_bf16(g1 + jc);
      x1 = fmaf(na, __ldg(q + jc), __ldg(rold + jc));
      v1 = j < (unsigned)N ? v1 : 0.f;
    }
    const unsigned j2 = (unsigned)ic + (unsigned)B.d[2];
    const unsigned j3 = (unsigned)ic + (unsigned)B.d[3];
    const int j2c = (int)min(j2, un), j3c = (int)min(j3, un);
    float v2 = ld_bf16(g2 + j2c), v3 = ld_bf16(g3 + j3c);
    const float x2 = fmaf(na, __ldg(q + j2c), __ldg(rold + j2c));
    const float x3 = fmaf(na, __ldg(q + j3c), __ldg(rold + j3c));
    v2 = j2 < (unsigned)N ? v2 : 0.f;
    v3 = j3 < (unsigned)N ? v3 : 0.f;
    float sum = fmaf(v0, r0, 0.f);
    sum = fmaf(v1, x1, sum);
    sum = fmaf(v2, x2, sum);
    sum = fmaf(v3, x3, sum);
    if (i < N) {
      a.rnew[i] = r0;
      a.y[i] = sum;
      rr = fma((double)r0, (double)r0, rr);
    }
  }
  double in[1] = {rr}, out[1];
  if (grid_reduce<1>(in, partials, a.ticket, out) && threadIdx.x == 0) {
    st->in_iter += 1;
    st->total_inner += 1;
    const double res = sqrt(out[0]) / st->in_nrm0;
    st->in_res = res;
    if (!(res > st->in_tol) || inner_broke_down(st) ||
        st->total_inner >= st->max_iter)
      st->in_stop = 1;
    if (st->use_cond)
      cudaGraphSetConditional((cudaGraphConditionalHandle)st->cond,
                              st->in_stop ? 0u : 1u);
  }
}

}  // namespace cgx
