// Device-side helpers shared by every kernel of libcgb200: block reductions,
// the mbarrier / bulk-copy (TMA) primitives used to stage matrix tiles in
// shared memory, and the solver state that lives in device memory.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cgx {

constexpr int kThreads = 256;   // threads per CTA for every streaming kernel
constexpr int kWarps = kThreads / 32;
constexpr int kMaxGrid = 148 * 8;  // upper bound on persistent CTAs (partials)
constexpr int kPad = 8;  // elements of padding after every index/value array

// Error bits recorded in CgState::error by device code.
enum : int {
  kErrBarrierTimeout = 1,  // a bounded mbarrier wait gave up
};

// Iteration state of one solve, resident in device memory so that the loop
// needs no host round trip. Every field is written only by the last CTA of a
// kernel (the "finalize" step) or by the host before a launch.
struct CgState {
  double rho, rho_old, alpha, beta, pq, r2, nrm0, residual;
  double tol;
  int iteration, max_iter;
  int stop;       // set when converged or when the iteration limit is hit
  int converged;
  int finished;   // chunked loop: the final x update has been applied
  int error;      // kErr* bits
  unsigned counter[8];  // last-CTA-done tickets, one per kernel kind
  unsigned long long cond;  // cudaGraphConditionalHandle of the while node
  int use_cond;
  int body_count;  // loop bodies run; the graph loop guard caps it
  // Mixed-precision inner solve (FP32 vectors, FP64 scalars).
  double in_rho, in_alpha, in_beta, in_nrm0, in_tol, in_res;
  double bnorm;          // ||b|| of the refinement loop
  double inner_tol_min;  // floor of the inner relative tolerance
  int in_iter, in_stop, in_finished;
  int total_inner;
  int in_pslot;  // fused persistent inner solve: ping-pong buffer of the last p
};

// The inner FP32 iteration cannot make progress: a step length that is zero
// (<p,q> overflowed to infinity, as with values beyond the FP32 range) or not
// finite. The stop that follows hands the failed refinement step to the
// host, which restores x and finishes in FP64. A NaN residual stops the loop
// through the residual test itself (!(res > tol)).
__device__ __forceinline__ bool inner_broke_down(const CgState *st) {
  const double a = st->in_alpha;
  return !(fabs(a) <= 1.7976931348623157e308) || a == 0.0;
}

// --- reductions ------------------------------------------------------------

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic sum of one double per thread over a kThreads-thread CTA.
// The result is valid in thread 0. `sh` holds kWarps doubles.
__device__ __forceinline__ double block_sum(double v, double *sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < kWarps ? sh[lane] : 0.0;
    v = warp_sum(v);
  }
  return v;
}

// Writes this CTA's NACC partial sums, and lets the CTA that finishes last
// reduce all partials in a fixed order. Returns true in every thread of the
// last CTA; `out` then holds the grid-wide sums in thread 0.
template <int NACC>
__device__ __forceinline__ bool grid_reduce(const double (&acc)[NACC],
                                            double *partials, unsigned *ticket,
                                            double (&out)[NACC]) {
  __shared__ double sh[kWarps];
  __shared__ bool am_last;
#pragma unroll
  for (int a = 0; a < NACC; a++) {
    double s = block_sum(acc[a], sh);
    if (threadIdx.x == 0) partials[a * kMaxGrid + blockIdx.x] = s;
  }
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  // All of a thread's partials are loaded before the first addition (one L2
  // round trip instead of one per partial); they are added in the same order
  // as a plain loop would, so the sums do not change.
  constexpr int kPer = (kMaxGrid + kThreads - 1) / kThreads;
#pragma unroll
  for (int a = 0; a < NACC; a++) {
    double v[kPer];
#pragma unroll
    for (int k = 0; k < kPer; k++) {
      const int b = threadIdx.x + k * kThreads;
      v[k] = b < (int)gridDim.x ? __ldcg(&partials[a * kMaxGrid + b]) : 0.0;
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kPer; k++) s += v[k];
    out[a] = block_sum(s, sh);
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

// --- mbarrier + bulk async copy (TMA, 1-D) ------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar,
                                                      unsigned bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_addr(bar)),
      "r"(bytes)
      : "memory");
}

// Global -> shared bulk copy completing on `bar`. Both addresses must be
// 16-byte aligned and `bytes` a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src,
                                         unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after `limit` polls (each poll may itself suspend
// for a hardware-defined interval) and reports false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar,
                                                  unsigned parity,
                                                  unsigned limit = 1u << 22) {
  for (unsigned i = 0; i < limit; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

}  // namespace cgx
