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
// inside the launch are read with weak loads after the barrier's acquire,
// never through the read-only path (fused.cuh).
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
#include "sell.cuh"

namespace cgx {

constexpr unsigned kSyncPolls = 1u << 24;
enum : int { kErrGridSync = 4 };  // CgState::error: a grid barrier gave up

// Which persistent form the default loop mode takes. Measured on the 7-point
// grids against the graph of per-iteration kernels (learned / Jacobi mixed
// solves): fused 1.62x / 1.77x faster at 96^3; split 1.27x / 1.41x at 128^3
// and 1.15x / 1.18x at 160^3, where the fused form's recomputed neighbour
// values cost more than its saved barriers.
#ifndef CGX_PERSIST_FUSED_MAX_ROWS
#define CGX_PERSIST_FUSED_MAX_ROWS 1300000
#endif
constexpr int kPersistFusedMaxRows = CGX_PERSIST_FUSED_MAX_ROWS;

// Systems from this size on take the split kernel with an L2 prefetch of
// the band values two grid-stride rows ahead (measured at 160^3: learned /
// Jacobi solves 2 % / 6 % faster; at 128^3, where the band stays in L2,
// 1-3 % slower).
#ifndef CGX_PERSIST_PREFETCH_MIN_ROWS
#define CGX_PERSIST_PREFETCH_MIN_ROWS 3000000
#endif
constexpr int kPersistPrefetchMinRows = CGX_PERSIST_PREFETCH_MIN_ROWS;
constexpr int kPersistPrefetchRows = 2;

// CTA width of the persistent launches, and the CTAs per SM each kernel's
// register budget is set for. Wide CTAs keep the grid small (148 or 296
// CTAs), which makes the barriers and the every-CTA partial sums cheap:
// against 256-thread CTAs (888 of them) the learned solves ran 1.2-1.3x
// faster at every size.
#ifndef CGX_PERSIST_THREADS
#define CGX_PERSIST_THREADS 1024
#endif
#ifndef CGX_PERSIST_FUSED_MINB
#define CGX_PERSIST_FUSED_MINB 1
#endif
#ifndef CGX_PERSIST_SPLIT_MINB_LEARNED
#define CGX_PERSIST_SPLIT_MINB_LEARNED 2
#endif
#ifndef CGX_PERSIST_SPLIT_MINB_JACOBI
#define CGX_PERSIST_SPLIT_MINB_JACOBI 1
#endif
constexpr int kPersistThreads = CGX_PERSIST_THREADS;
constexpr int kPersistFusedMinB = CGX_PERSIST_FUSED_MINB;
constexpr int kPersistSplitMinB[2] = {CGX_PERSIST_SPLIT_MINB_JACOBI,
                                      CGX_PERSIST_SPLIT_MINB_LEARNED};
static_assert(kPersistThreads % 128 == 0 && kPersistThreads <= 1024, "CTA width");

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
// before the launch). The add is a release (after the CTA barrier, so it
// covers every thread's writes) and the polls are acquires, so writes before
// the barrier are visible after it without further fences (measured 2-6 %
// faster per solve than a full fence on each side of a relaxed add).
__device__ __forceinline__ bool grid_sync(unsigned long long *count,
                                          unsigned long long target,
                                          unsigned polls = kSyncPolls) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("red.release.gpu.global.add.u64 [%0], 1;" : : "l"(count) : "memory");
    unsigned i = 0;
    while (ld_acquire_u64(count) < target && ++i < polls) __nanosleep(32);
    ok = i < polls;
  }
  __syncthreads();
  return ok != 0;
}

// Diagnostics of the bounded waits: waits that nothing can complete, with a
// short limit, so that the give-up path runs and sets its error bit.
//  - a grid barrier whose target the CTAs' arrivals never reach;
//  - an mbarrier (one expected arrival) that nobody arrives on.
__global__ void k_wait_timeout(unsigned long long *count, int which, unsigned polls,
                               CgState *st) {
  if (which == 0) {
    if (!grid_sync(count, ~0ull, polls) && threadIdx.x == 0) atomicOr(&st->error, kErrGridSync);
    return;
  }
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (!mbar_wait_bounded(&bar, 0u, polls) && threadIdx.x == 0)
    atomicOr(&st->error, kErrBarrierTimeout);
}

// Sum over a TPB-thread CTA, valid in thread 0; sh holds TPB / 32 doubles.
template <int TPB>
__device__ __forceinline__ double block_sum_t(double v, double *sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < TPB / 32 ? sh[lane] : 0.0;
    v = warp_sum(v);
  }
  return v;
}

// This CTA's partial (the block sum of v) into slot[blockIdx.x].
template <int TPB>
__device__ __forceinline__ void put_partial(double v, double *slot) {
  __shared__ double sh[TPB / 32];
  v = block_sum_t<TPB>(v, sh);
  if (threadIdx.x == 0) slot[blockIdx.x] = v;
}

// The sum of the grid's partials in a fixed order, in every thread.
template <int TPB>
__device__ __forceinline__ double sum_partials(const double *slot) {
  __shared__ double sh[TPB / 32];
  __shared__ double tot;
  constexpr int kPer = (kMaxGrid + TPB - 1) / TPB;
  double v[kPer];
#pragma unroll
  for (int k = 0; k < kPer; k++) {
    const int b = threadIdx.x + k * TPB;
    v[k] = b < (int)gridDim.x ? __ldcg(&slot[b]) : 0.0;
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kPer; k++) s += v[k];
  s = block_sum_t<TPB>(s, sh);
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

template <bool LEARNED, int TPB, int MINB>
__global__ void __launch_bounds__(TPB, MINB)
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
    put_partial<TPB>(band_dir_rows<TPB>(A, da, (float)alpha, (float)beta), slot0);
    if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
    alpha = rho / sum_partials<TPB>(slot0);
    // B: r and the residual test (learned: also y = G^T r; Jacobi: z, <r,z>).
    if (LEARNED) {
      float *r_old = par ? a.r[1] : a.r[0], *r_new = par ? a.r[0] : a.r[1];
      const ResArgs ra{r_old, a.q, r_new, a.y};
      put_partial<TPB>(gband_res_rows<TPB>(G, ra, (float)(-alpha)), slot1);
    } else {
      double rr, rz;
      jacobi_res_rows<TPB>(A.N, a.r[0], a.q, a.C, a.z, (float)(-alpha), rr, rz);
      put_partial<TPB>(rr, slot1);
      put_partial<TPB>(rz, slot2);
    }
    if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
    it++;
    total++;
    res = sqrt(sum_partials<TPB>(slot1)) / nrm0;
    const bool stop = !(res > tol) || !(fabs(alpha) <= 1.7976931348623157e308) ||
                      alpha == 0.0 || total >= maxit;
    par = 1 - par;  // this iteration's p (and r) are in the other buffers
    if (stop) break;
    if (LEARNED) {
      // C: z = G y + eps C r, <r,z>.
      const GzArgs za{a.y, par ? a.r[1] : a.r[0], a.C, a.z, a.eps};
      put_partial<TPB>(gband_z_rows<TPB>(G, za), slot2);
      if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
    }
    const double rzn = sum_partials<TPB>(slot2);
    beta = rzn / rho;
    rho = rzn;
  }
  // par indexes the buffer the last phase A wrote p into.
  persist_publish(st, alpha, beta, rho, res, it, total, par, ok);
}

// Where the split form applies d += a p. Deferred: in the direction phase,
// which reads p once for both updates (as k_inner_direction does), the
// loop's last update left pending (k_outer_update_pending applies it with
// p[0] and the published a); 4 bytes fewer per row and iteration. Else in
// the residual phase, d complete when the loop stops. Measured (same box):
// deferred, 160^3 learned 22.93 against 23.66 ms; deferring everywhere made
// 128^3 learned 10.72 against 10.62 ms and the Jacobi and SELL-U forms
// 1-1.5 % slower. So only the learned form with the L2 prefetch (the
// largest grids) defers.
__host__ __device__ constexpr bool persist_defers_d(bool learned, int pf) {
  return learned && pf > 0;
}

// The split form: the graph iteration's kernels as phases (fused.cuh), five
// barriers per learned iteration and three per Jacobi one, no values formed
// twice and no ping-pong buffers (p[0], r[0] only). [d += a p] is in phase B
// or, deferred (persist_defers_d), in phase E.
//
//   learned: A  q = A p                                   | <p,q> -> a
//            B  r -= a q [, d += a p]                     | <r,r> -> test
//            C  y = G^T r                                 |
//            D  z = G y + eps C r                         | <r,z> -> b
//            E  [d += a p,] p = z + b p                   |
//   Jacobi:  A  as above                                  | <p,q> -> a
//            B  r -= a q, d += a p                        | <r,r>, <r,Cr> -> test, b
//            E  p = C r + b p                             |
template <bool LEARNED, int TPB, int MINB, int PF>
__global__ void __launch_bounds__(TPB, MINB)
    k_inner_persist_split(BandView<4> A, GBandView G, PersistArgs a, CgState *st) {
  constexpr bool DEFER = persist_defers_d(LEARNED, PF);
  double rho = st->in_rho, alpha = 0.0, beta = 0.0, res = 0.0;
  const double nrm0 = st->in_nrm0, tol = st->in_tol;
  int total = st->total_inner;
  const int maxit = st->max_iter, N = A.N;
  const unsigned long long nb = gridDim.x;
  unsigned long long bar = 0;
  int it = 0;
  bool ok = true;
  double *slot0 = a.part, *slot1 = a.part + kMaxGrid, *slot2 = a.part + 2 * kMaxGrid;
  float *p = a.p[0], *r = a.r[0];
  for (;;) {
    put_partial<TPB>(band_q_rows<TPB, PF>(A, p, a.q), slot0);
    if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
    alpha = rho / sum_partials<TPB>(slot0);
    {
      double rr, rz;
      update_rows<TPB, !DEFER>(N, r, a.q, a.d, p, LEARNED ? nullptr : a.C, (float)alpha,
                               rr, rz);
      put_partial<TPB>(rr, slot1);
      if (!LEARNED) put_partial<TPB>(rz, slot2);
    }
    if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
    it++;
    total++;
    res = sqrt(sum_partials<TPB>(slot1)) / nrm0;
    const bool stop = !(res > tol) || !(fabs(alpha) <= 1.7976931348623157e308) ||
                      alpha == 0.0 || total >= maxit;
    if (stop) break;
    if (LEARNED) {
      gband_t_rows<TPB, PF>(G, r, a.y);
      if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
      const GzArgs za{a.y, r, a.C, a.z, a.eps};
      put_partial<TPB>(gband_z_rows<TPB, PF>(G, za), slot2);
      if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
    }
    const double rzn = sum_partials<TPB>(slot2);
    beta = rzn / rho;
    rho = rzn;
    direction_rows<TPB, DEFER>(N, p, a.d, LEARNED ? a.z : nullptr, r, a.C, (float)alpha,
                               (float)beta);
    if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
  }
  persist_publish(st, alpha, beta, rho, res, it, total, 0, ok);
}

// The split form on SELL-U (sell.cuh): A, G and G^T in uniform slices (the
// 27-point stencils and other matrices whose rows in a slice reach the same
// neighbours), the products as sellu_rows phases with weak gathers; the
// streaming phases and barriers are those of k_inner_persist_split.
struct PersistQ {  // q = A p, <p,q>
  using Acc = Acc1;
  struct Pre {
    float p;
  };
  const float *p;
  float *q;
  __device__ Pre prefetch(int i) const { return Pre{ldv(p + i)}; }
  __device__ void row(int i, float s, Acc &a, const Pre &pr) const {
    q[i] = s;
    a.a0 = fma((double)pr.p, (double)s, a.a0);
  }
};
struct PersistZ {  // z = G y + eps C r, <r,z> (OpLearnedZ's arithmetic)
  using Acc = Acc1;
  struct Pre {
    float r, c;
  };
  const float *r, *C;
  float *z;
  float eps;
  __device__ Pre prefetch(int i) const { return Pre{ldv(r + i), __ldg(C + i)}; }
  __device__ void row(int i, float s, Acc &a, const Pre &pr) const {
    const float zi = fmaf(eps * pr.c, pr.r, s);
    z[i] = zi;
    a.a0 = fma((double)pr.r, (double)zi, a.a0);
  }
};

// Slots per chunk of the SELL-U products in the persistent form, its CTA
// width and CTAs per SM.
// Measured on the 27-point grids (Jacobi / learned mixed solves against the
// graph of per-iteration kernels): 1.30x / 1.29x faster at 96^3, 1.17x /
// 1.20x at 128^3, with 512-thread CTAs two per SM (64 registers, a few
// spilled) ahead of 384 x 2 and 256 x 3 (80 registers, no spills).
constexpr int kPersistSellU = 8;
#ifndef CGX_PERSIST_SELL_THREADS
#define CGX_PERSIST_SELL_THREADS 512
#endif
#ifndef CGX_PERSIST_SELL_MINB
#define CGX_PERSIST_SELL_MINB 2
#endif
constexpr int kPersistSellThreads = CGX_PERSIST_SELL_THREADS;
constexpr int kPersistSellMinB = CGX_PERSIST_SELL_MINB;

template <bool LEARNED, int TPB, int MINB>
__global__ void __launch_bounds__(TPB, MINB)
    k_inner_persist_sell(SellUView<float> A, SellUView<__nv_bfloat16> G,
                         SellUView<__nv_bfloat16> GT, PersistArgs a, CgState *st) {
  constexpr int U = kPersistSellU;
  double rho = st->in_rho, alpha = 0.0, beta = 0.0, res = 0.0;
  const double nrm0 = st->in_nrm0, tol = st->in_tol;
  int total = st->total_inner;
  const int maxit = st->max_iter, N = A.N;
  const unsigned long long nb = gridDim.x;
  unsigned long long bar = 0;
  int it = 0;
  bool ok = true;
  double *slot0 = a.part, *slot1 = a.part + kMaxGrid, *slot2 = a.part + 2 * kMaxGrid;
  float *p = a.p[0], *r = a.r[0];
  for (;;) {
    {
      Acc1 acc;
      sellu_rows<float, U, true, TPB>(A, p, GatherWeak{}, PersistQ{p, a.q}, acc);
      put_partial<TPB>(acc.a0, slot0);
    }
    if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
    alpha = rho / sum_partials<TPB>(slot0);
    {
      double rr, rz;
      update_rows<TPB, true>(N, r, a.q, a.d, p, LEARNED ? nullptr : a.C, (float)alpha, rr,
                             rz);
      put_partial<TPB>(rr, slot1);
      if (!LEARNED) put_partial<TPB>(rz, slot2);
    }
    if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
    it++;
    total++;
    res = sqrt(sum_partials<TPB>(slot1)) / nrm0;
    const bool stop = !(res > tol) || !(fabs(alpha) <= 1.7976931348623157e308) ||
                      alpha == 0.0 || total >= maxit;
    if (stop) break;
    if (LEARNED) {
      NoAcc none;
      sellu_rows<__nv_bfloat16, U, true, TPB>(GT, r, GatherWeak{}, OpInnerStore{a.y}, none);
      if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
      Acc1 acc;
      sellu_rows<__nv_bfloat16, U, true, TPB>(G, a.y, GatherWeak{},
                                              PersistZ{r, a.C, a.z, a.eps}, acc);
      put_partial<TPB>(acc.a0, slot2);
      if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
    }
    const double rzn = sum_partials<TPB>(slot2);
    beta = rzn / rho;
    rho = rzn;
    direction_rows<TPB, false>(N, p, a.d, LEARNED ? a.z : nullptr, r, a.C, (float)alpha,
                               (float)beta);
    if (!(ok = grid_sync(a.sync, ++bar * nb))) break;
  }
  persist_publish(st, alpha, beta, rho, res, it, total, 0, ok);
}

}  // namespace cgx
