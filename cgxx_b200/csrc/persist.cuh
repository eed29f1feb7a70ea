// Persistent inner solves of the mixed paths on the band form.
//
// Each inner FP32 PCG of a refinement step is one cooperative launch instead
// of a graph of four or five kernels per iteration. The CTAs (all resident:
// a cooperative launch guarantees it) run the phases of the fused band
// iteration (fused.cuh) over the rows and meet at a grid-wide barrier after
// each phase. After a barrier every CTA adds the per-CTA partial sums of the
// phase in the same fixed order, so all CTAs hold the same alpha, beta and
// residual and take the same stop decision; no CTA waits for a last CTA to
// finish a reduction, and no launch separates the phases. Vectors written
// inside the launch are read back through L2 (__ldcg), never through the
// read-only path, whose lines could be stale.
//
//   learned: A  p = z + b p_old, d += a_old p_old, q = A p       | <p,q> -> a
//            B  r = r_old - a q, y = G^T r                        | <r,r> -> test
//            C  z = G y + eps C r                                 | <r,z> -> b
//   Jacobi:  A  as above                                          | <p,q> -> a
//            B  r -= a q, z = C r                                 | <r,r>, <r,z> -> test, b
//
// Every barrier wait is bounded (kSyncPolls polls): a CTA that gives up sets
// kErrGridSync in CgState::error and leaves the loop, so the launch always
// ends and the host reports CGX_ERROR_DEVICE.
#pragma once

#include "fused.cuh"
#include "kernels.cuh"

namespace cgx {

constexpr unsigned kSyncPolls = 1u << 24;
enum : int { kErrGridSync = 4 };  // CgState::error: a grid barrier gave up

// Largest systems the default loop mode solves with persistent inner
// solves. The fused phases read p, z and r of neighbouring rows again, which
// costs more as the vectors outgrow L2, and they save fewer launches on the
// Jacobi path (two phases against five kernels for the learned one):
// measured on the 7-point grids, learned 1.31x faster at 96^3 and 1.03x at
// 128^3, Jacobi 1.31x faster at 96^3 and 1.08x slower at 128^3, both slower
// at 160^3.
#ifndef CGX_PERSIST_MAX_ROWS
#define CGX_PERSIST_MAX_ROWS 2200000
#endif
#ifndef CGX_PERSIST_MAX_ROWS_JACOBI
#define CGX_PERSIST_MAX_ROWS_JACOBI 1500000
#endif
constexpr int kPersistMaxRows = CGX_PERSIST_MAX_ROWS;
constexpr int kPersistMaxRowsJacobi = CGX_PERSIST_MAX_ROWS_JACOBI;

// Partial-sum slots: phase k of an iteration uses slot k, so a slot is
// written again only two barriers after every CTA has read it.
constexpr int kPersistSlots = 3;

__device__ __forceinline__ unsigned long long ld_acquire_u64(
    const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier: every CTA adds one to *count and waits until it reaches
// target (the barrier's number times the grid size; the host zeroes *count
// before the launch). Writes before the barrier are visible after it.
__device__ __forceinline__ bool grid_sync(unsigned long long *count,
                                          unsigned long long target) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(count, 1ull);
    unsigned i = 0;
    while (ld_acquire_u64(count) < target && ++i < kSyncPolls) __nanosleep(32);
    ok = i < kSyncPolls;
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// This CTA's partial (the block sum of v) into slot[blockIdx.x].
__device__ __forceinline__ void put_partial(double v, double *slot) {
  __shared__ double sh[kWarps];
  v = block_sum(v, sh);
  if (threadIdx.x == 0) slot[blockIdx.x] = v;
}

// The sum of the grid's partials in a fixed order, in every thread.
__device__ __forceinline__ double sum_partials(const double *slot) {
  __shared__ double sh[kWarps];
  __shared__ double tot;
  constexpr int kPer = (kMaxGrid + kThreads - 1) / kThreads;
  double v[kPer];
#pragma unroll
  for (int k = 0; k < kPer; k++) {
    const int b = threadIdx.x + k * kThreads;
    v[k] = b < (int)gridDim.x ? __ldcg(&slot[b]) : 0.0;
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kPer; k++) s += v[k];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) tot = s;
  __syncthreads();
  return tot;
}

struct PersistArgs {
  float *p[2];      // ping-pong search directions (slot 0 = the start's p)
  float *r[2];      // ping-pong residuals (slot 0 = the start's r)
  float *z, *d, *q;
  float *y;         // learned: G^T r
  const float *C;   // FP32 Jacobi vector
  float eps;        // learned: eps of eps C r
  double *part;     // kPersistSlots x kMaxGrid partial sums
  unsigned long long *sync;  // barrier counter (zeroed before the launch)
};

// Publishes the loop's scalars for the host and the refinement epilogue
// (the pending d update reads in_alpha and in_pslot).
__device__ __forceinline__ void persist_publish(CgState *st, double alpha, double beta,
                                                double rho, double res, int it,
                                                int total, int pslot, bool ok) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->in_alpha = alpha;
    st->in_beta = beta;
    st->in_rho = rho;
    st->in_res = res;
    st->in_iter = it;
    st->total_inner = total;
    st->in_pslot = pslot;
    st->in_stop = 1;
    st->in_finished = 1;
  }
  if (!ok && threadIdx.x == 0) atomicOr(&st->error, kErrGridSync);
}

template <bool LEARNED>
__global__ void __launch_bounds__(kThreads)
    k_inner_persist(BandView<4> A, GBandView G, PersistArgs a, CgState *st) {
  // Start state (k_inner_start / the learned start): p = z, a = b = 0.
  double rho = st->in_rho, alpha = st->in_alpha, beta = st->in_beta;
  const double nrm0 = st->in_nrm0, tol = st->in_tol;
  int total = st->total_inner;
  const int maxit = st->max_iter;
  const unsigned long long nb = gridDim.x;
  unsigned long long bar = 0;
  double res = 0.0;
  int it = 0, par = 0;
  bool ok = true;
  double *slot0 = a.part, *slot1 = a.part + kMaxGrid, *slot2 = a.part + 2 * kMaxGrid;
  for (;;) {
    // (selects, not a.p[par]: a runtime index would put the arrays in local memory)
    float *p_old = par ? a.p[1] : a.p[0], *p_new = par ? a.p[0] : a.p[1];
    // A: p, d, q = A p, <p,q>.
    const DirArgs da{a.z, p_old, p_new, a.d, a.q};
    put_partial(band_dir_rows(A, da, (float)alpha, (float)beta), slot0);
    if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
    alpha = rho / sum_partials(slot0);
    // B: r and the residual test (learned: also y = G^T r; Jacobi: z, <r,z>).
    if (LEARNED) {
      float *r_old = par ? a.r[1] : a.r[0], *r_new = par ? a.r[0] : a.r[1];
      const ResArgs ra{r_old, a.q, r_new, a.y};
      put_partial(gband_res_rows(G, ra, (float)(-alpha)), slot1);
    } else {
      double rr, rz;
      inner_update_rows<true, true>(A.N, a.r[0], a.q, a.C, a.z, (float)(-alpha), rr, rz);
      put_partial(rr, slot1);
      put_partial(rz, slot2);
    }
    if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
    it++;
    total++;
    res = sqrt(sum_partials(slot1)) / nrm0;
    const bool stop = !(res > tol) || !(fabs(alpha) <= 1.7976931348623157e308) ||
                      alpha == 0.0 || total >= maxit;
    par = 1 - par;  // this iteration's p (and r) are in the other buffers
    if (stop) break;
    if (LEARNED) {
      // C: z = G y + eps C r, <r,z>.
      const GzArgs za{a.y, par ? a.r[1] : a.r[0], a.C, a.z, a.eps};
      put_partial(gband_z_rows(G, za), slot2);
      if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
    }
    const double rzn = sum_partials(slot2);
    beta = rzn / rho;
    rho = rzn;
  }
  // par indexes the buffer the last phase A wrote p into.
  persist_publish(st, alpha, beta, rho, res, it, total, par, ok);
}

}  // namespace cgx
