// Row loops of the fused band inner iteration, for the persistent inner
// solve (persist.cuh).
//
// One inner PCG iteration on the symmetric band form (band.cuh) runs as
//   A  p = z + b p_old, d += a_old p_old, q = A p, <p,q> -> a
//   B  (learned) r = r_old - a q, y = G^T r, <r,r> -> residual test
//      (Jacobi)  r -= a q, z = C r, <r,r>, <r,z> -> residual test, b
//   C  (learned) z = G y + eps C r, <r,z> -> b
// The products read p and r of neighbouring rows; those values are formed
// from the previous iteration's vectors by every thread that needs them (the
// same single-rounding operations as the owner's, so the same bits), and the
// new vectors go to the other buffer of a ping-pong pair, because the old
// ones are still read by other rows' threads. The update of d lags one
// iteration (it needs p_old, which the next phase A reads anyway); the
// refinement step's epilogue applies the last one (k_outer_update_pending).
//
// The loops are those of the generic band kernels: one row per thread,
// grid-stride, the row-major band values (one 16-byte load of U, one 8-byte
// load of the factor's row), the same products added in the same order and
// the same masks. Vectors written inside a persistent launch are read
// through L2 (__ldcg): another CTA wrote them in an earlier phase of the same
// launch, so the read-only path could hold stale lines.
#pragma once

#include "band.cuh"
#include "kernels.cuh"

namespace cgx {

struct DirArgs {
  const float *z;     // preconditioned residual
  const float *pold;  // search direction of the last iteration
  float *pnew;        // the new search direction
  float *d;           // inner solution
  float *q;           // A p
};

// Phase A: this thread's partial sum of <p,q>.
__device__ __forceinline__ double band_dir_rows(const BandView<4> &B, const DirArgs &a,
                                                float al, float be) {
  const int N = B.N;
  const unsigned nmax = (unsigned)(N - 1);
  const float4 *__restrict__ U4 = reinterpret_cast<const float4 *>(B.U);
  const float *__restrict__ z = a.z;
  const float *__restrict__ po = a.pold;
  double acc = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N; i += gridDim.x * kThreads) {
    const float4 u = __ldg(U4 + i);
    const float po0 = __ldcg(po + i);
    const float p0 = fmaf(be, po0, __ldcg(z + i));
    float pu[4], lv[4], pl[4];
    pu[0] = p0;
#pragma unroll
    for (int k = 1; k < 4; k++) {
      const int ju = (int)min((unsigned)i + (unsigned)B.d[k], nmax);
      pu[k] = fmaf(be, __ldcg(po + ju), __ldcg(z + ju));
      const int j = i - B.d[k], jc = max(j, 0);
      lv[k] = __ldg(&B.U[(size_t)jc * 4 + k]);
      pl[k] = fmaf(be, __ldcg(po + jc), __ldcg(z + jc));
      lv[k] = j < 0 ? 0.f : lv[k];
    }
    float sum = fmaf(u.x, pu[0], 0.f);
    sum = fmaf(u.y, pu[1], sum);
    sum = fmaf(u.z, pu[2], sum);
    sum = fmaf(u.w, pu[3], sum);
#pragma unroll
    for (int k = 1; k < 4; k++) sum = fmaf(lv[k], pl[k], sum);
    a.d[i] = fmaf(al, po0, a.d[i]);
    a.pnew[i] = p0;
    a.q[i] = sum;
    acc = fma((double)p0, (double)sum, acc);
  }
  return acc;
}

struct ResArgs {
  const float *rold;  // residual of the last iteration
  const float *q;     // A p of this iteration
  float *rnew;        // the new residual
  float *y;           // G^T r
};

// Phase B (learned): this thread's partial sum of <r,r>.
__device__ __forceinline__ double gband_res_rows(const GBandView &B, const ResArgs &a,
                                                 float na) {
  const int N = B.N;
  const unsigned short *gv = reinterpret_cast<const unsigned short *>(B.val);
  const float *__restrict__ ro = a.rold;
  const float *__restrict__ qv = a.q;
  double rr = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N; i += gridDim.x * kThreads) {
    const float r0 = fmaf(na, __ldcg(qv + i), __ldcg(ro + i));
    float v[4], xv[4];
    v[0] = bf16_bits_to_float(__ldg(&gv[(size_t)i * 4]));
    xv[0] = r0;
#pragma unroll
    for (int k = 1; k < 4; k++) {
      const unsigned j = (unsigned)i + (unsigned)B.d[k];
      const int jc = (int)min(j, (unsigned)(N - 1));
      v[k] = bf16_bits_to_float(__ldg(&gv[(size_t)jc * 4 + k]));
      xv[k] = fmaf(na, __ldcg(qv + jc), __ldcg(ro + jc));
      v[k] = j < (unsigned)N ? v[k] : 0.f;
    }
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) sum = fmaf(v[k], xv[k], sum);
    a.rnew[i] = r0;
    a.y[i] = sum;
    rr = fma((double)r0, (double)r0, rr);
  }
  return rr;
}

struct GzArgs {
  const float *y, *r, *C;
  float *z;
  float eps;
};

// Phase C (learned): z = G y + eps C r; this thread's partial sum of <r,z>.
__device__ __forceinline__ double gband_z_rows(const GBandView &B, const GzArgs &a) {
  const int N = B.N;
  const float *__restrict__ y = a.y;
  double acc = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N; i += gridDim.x * kThreads) {
    const uint2 raw = __ldg(reinterpret_cast<const uint2 *>(B.val) + i);
    float v[4], xv[4];
    v[0] = __uint_as_float(raw.x << 16);
    v[1] = __uint_as_float(raw.x & 0xffff0000u);
    v[2] = __uint_as_float(raw.y << 16);
    v[3] = __uint_as_float(raw.y & 0xffff0000u);
#pragma unroll
    for (int k = 0; k < 4; k++) xv[k] = __ldcg(y + max(i - B.d[k], 0));
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) sum = fmaf(v[k], xv[k], sum);
    const float ri = __ldcg(a.r + i);
    const float zi = fmaf(a.eps * __ldg(a.C + i), ri, sum);
    a.z[i] = zi;
    acc = fma((double)ri, (double)zi, acc);
  }
  return acc;
}

}  // namespace cgx
