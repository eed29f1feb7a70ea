// Row loops of the persistent inner solves (persist.cuh).
//
// Fused phases. One inner PCG iteration on the symmetric band form
// (band.cuh) runs as
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
// Split phases: the kernels of the graph iteration as phases, one product
// or one update each (q = A p | r -= a q, d += a p | y = G^T r |
// z = G y + eps C r | p = z + b p), with the same arithmetic as those
// kernels, so the same bits.
//
// The loops are those of the generic band kernels: one row per thread (four
// consecutive elements for the streaming updates), grid-stride over TPB-wide
// CTAs, the row-major band values (one 16-byte load of U, one 8-byte load of
// the factor's row), the same products added in the same order and the same
// masks. The band values, the factor and C do not change during a launch and
// take the read-only path (__ldg). The vectors are written inside the launch
// and are read with weak loads that L1 may cache (ldv): every read of another
// CTA's value comes after a grid barrier whose GPU-scope acquire (grid_sync)
// makes that value visible to the weak loads that follow it, so L1 holds no
// line from before the barrier that is still read. Each vector element is
// written by the one thread that owns it, and no phase reads a value written
// in the same phase by another thread.
#pragma once

#include "band.cuh"
#include "kernels.cuh"

namespace cgx {

// (Reading them through L2 only, __ldcg, measured 1-2 % slower.)
__device__ __forceinline__ float ldv(const float *p) { return __ldca(p); }
__device__ __forceinline__ float4 ldv4(const float *v, int i) {
  return __ldca(reinterpret_cast<const float4 *>(v) + i);
}

// L2 prefetch of the read-only row values a thread reads PF grid-stride
// steps later (PF = 0: none): one lane per 128-byte line issues it. It keeps
// more of the band stream in flight than the warps' own loads (whose
// registers cap them at one row per thread), which bounds the products
// once the band no longer stays in L2 between iterations.
template <int BYTES_PER_ROW, int PF>
__device__ __forceinline__ void prefetch_row(const void *base, int i, int stride, int N) {
  constexpr int kRowsPerLine = 128 / BYTES_PER_ROW;
  const long long j = (long long)i + (long long)PF * stride;
  if (PF > 0 && (threadIdx.x & (kRowsPerLine - 1)) == 0 && j < N)
    asm volatile("prefetch.global.L2 [%0];"
                 :
                 : "l"((const char *)base + j * BYTES_PER_ROW));
}

struct DirArgs {
  const float *z;     // preconditioned residual
  const float *pold;  // search direction of the last iteration
  float *pnew;        // the new search direction
  float *d;           // inner solution
  float *q;           // A p
};

// Phase A: this thread's partial sum of <p,q>.
template <int TPB>
__device__ __forceinline__ double band_dir_rows(const BandView<4> &B, const DirArgs &a,
                                                float al, float be) {
  const int N = B.N;
  const unsigned nmax = (unsigned)(N - 1);
  const float4 *__restrict__ U4 = reinterpret_cast<const float4 *>(B.U);
  const float *z = a.z, *po = a.pold;
  double acc = 0.0;
  const int stride = gridDim.x * TPB;
  for (int i = blockIdx.x * TPB + threadIdx.x; i < N; i += stride) {
    prefetch_row<16, 0>(B.U, i, stride, N);
    const float4 u = __ldg(U4 + i);
    const float po0 = ldv(po + i);
    const float p0 = fmaf(be, po0, ldv(z + i));
    float pu[4], lv[4], pl[4];
    pu[0] = p0;
#pragma unroll
    for (int k = 1; k < 4; k++) {
      const int ju = (int)min((unsigned)i + (unsigned)B.d[k], nmax);
      pu[k] = fmaf(be, ldv(po + ju), ldv(z + ju));
      const int j = i - B.d[k], jc = max(j, 0);
      lv[k] = __ldg(&B.U[(size_t)jc * 4 + k]);
      pl[k] = fmaf(be, ldv(po + jc), ldv(z + jc));
      lv[k] = j < 0 ? 0.f : lv[k];
    }
    float sum = fmaf(u.x, pu[0], 0.f);
    sum = fmaf(u.y, pu[1], sum);
    sum = fmaf(u.z, pu[2], sum);
    sum = fmaf(u.w, pu[3], sum);
#pragma unroll
    for (int k = 1; k < 4; k++) sum = fmaf(lv[k], pl[k], sum);
    a.d[i] = fmaf(al, po0, ldv(a.d + i));
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
template <int TPB>
__device__ __forceinline__ double gband_res_rows(const GBandView &B, const ResArgs &a,
                                                 float na) {
  const int N = B.N;
  const unsigned short *gv = reinterpret_cast<const unsigned short *>(B.val);
  const float *ro = a.rold, *qv = a.q;
  double rr = 0.0;
  const int stride = gridDim.x * TPB;
  for (int i = blockIdx.x * TPB + threadIdx.x; i < N; i += stride) {
    prefetch_row<8, 0>(B.val, i, stride, N);
    const float r0 = fmaf(na, ldv(qv + i), ldv(ro + i));
    float v[4], xv[4];
    v[0] = bf16_bits_to_float(__ldg(&gv[(size_t)i * 4]));
    xv[0] = r0;
#pragma unroll
    for (int k = 1; k < 4; k++) {
      const unsigned j = (unsigned)i + (unsigned)B.d[k];
      const int jc = (int)min(j, (unsigned)(N - 1));
      v[k] = bf16_bits_to_float(__ldg(&gv[(size_t)jc * 4 + k]));
      xv[k] = fmaf(na, ldv(qv + jc), ldv(ro + jc));
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
template <int TPB, int PF = 0>
__device__ __forceinline__ double gband_z_rows(const GBandView &B, const GzArgs &a) {
  const int N = B.N;
  const float *y = a.y;
  double acc = 0.0;
  const int stride = gridDim.x * TPB;
  for (int i = blockIdx.x * TPB + threadIdx.x; i < N; i += stride) {
    prefetch_row<8, PF>(B.val, i, stride, N);
    const uint2 raw = __ldg(reinterpret_cast<const uint2 *>(B.val) + i);
    float v[4], xv[4];
    v[0] = __uint_as_float(raw.x << 16);
    v[1] = __uint_as_float(raw.x & 0xffff0000u);
    v[2] = __uint_as_float(raw.y << 16);
    v[3] = __uint_as_float(raw.y & 0xffff0000u);
#pragma unroll
    for (int k = 0; k < 4; k++) xv[k] = ldv(y + max(i - B.d[k], 0));
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) sum = fmaf(v[k], xv[k], sum);
    const float ri = ldv(a.r + i);
    const float zi = fmaf(a.eps * __ldg(a.C + i), ri, sum);
    a.z[i] = zi;
    acc = fma((double)ri, (double)zi, acc);
  }
  return acc;
}

// Four consecutive elements per thread (the streaming kernels' float4 loop)
// and the tail N mod 4 one per thread.
template <int TPB, typename F4, typename F1>
__device__ __forceinline__ void rows4(int N, F4 f4, F1 f1) {
  const int n4 = N >> 2;
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n4; i += gridDim.x * TPB) f4(i);
  for (int i = 4 * n4 + blockIdx.x * TPB + threadIdx.x; i < N; i += gridDim.x * TPB) f1(i);
}

// Phase B (Jacobi): r -= a q and z = C r (k_inner_update's arithmetic);
// this thread's partials of <r,r> and <r,z>.
template <int TPB>
__device__ __forceinline__ void jacobi_res_rows(int N, float *r, const float *q,
                                                const float *C, float *z, float na,
                                                double &rr, double &rz) {
  rr = 0.0;
  rz = 0.0;
  auto dots = [&](float ri, float zi) {
    rr = fma((double)ri, (double)ri, rr);
    rz = fma((double)ri, (double)zi, rz);
  };
  rows4<TPB>(
      N,
      [&](int i) {
        float4 rv = ldv4(r, i);
        const float4 qv = ldv4(q, i);
        const float4 cv = __ldg(reinterpret_cast<const float4 *>(C) + i);
        rv.x = fmaf(na, qv.x, rv.x);
        rv.y = fmaf(na, qv.y, rv.y);
        rv.z = fmaf(na, qv.z, rv.z);
        rv.w = fmaf(na, qv.w, rv.w);
        reinterpret_cast<float4 *>(r)[i] = rv;
        const float4 zv = make_float4(cv.x * rv.x, cv.y * rv.y, cv.z * rv.z, cv.w * rv.w);
        reinterpret_cast<float4 *>(z)[i] = zv;
        dots(rv.x, zv.x);
        dots(rv.y, zv.y);
        dots(rv.z, zv.z);
        dots(rv.w, zv.w);
      },
      [&](int i) {
        const float ri = fmaf(na, ldv(q + i), ldv(r + i));
        r[i] = ri;
        const float zi = __ldg(C + i) * ri;
        z[i] = zi;
        dots(ri, zi);
      });
}

// ---- Split phases ----------------------------------------------------------

// q = A p; this thread's partial of <p,q> (k_band with OpInnerQ).
template <int TPB, int PF = 0>
__device__ __forceinline__ double band_q_rows(const BandView<4> &B, const float *p,
                                              float *q) {
  const int N = B.N;
  const unsigned nmax = (unsigned)(N - 1);
  const float4 *__restrict__ U4 = reinterpret_cast<const float4 *>(B.U);
  double acc = 0.0;
  const int stride = gridDim.x * TPB;
  for (int i = blockIdx.x * TPB + threadIdx.x; i < N; i += stride) {
    prefetch_row<16, PF>(B.U, i, stride, N);
    const float4 u = __ldg(U4 + i);
    float xu[4], lv[4], xl[4];
#pragma unroll
    for (int k = 0; k < 4; k++) xu[k] = ldv(p + min((unsigned)i + (unsigned)B.d[k], nmax));
#pragma unroll
    for (int k = 1; k < 4; k++) {
      const int j = i - B.d[k], jc = max(j, 0);
      lv[k] = __ldg(&B.U[(size_t)jc * 4 + k]);
      xl[k] = ldv(p + jc);
      lv[k] = j < 0 ? 0.f : lv[k];
    }
    float sum = fmaf(u.x, xu[0], 0.f);
    sum = fmaf(u.y, xu[1], sum);
    sum = fmaf(u.z, xu[2], sum);
    sum = fmaf(u.w, xu[3], sum);
#pragma unroll
    for (int k = 1; k < 4; k++) sum = fmaf(lv[k], xl[k], sum);
    q[i] = sum;
    acc = fma((double)xu[0], (double)sum, acc);
  }
  return acc;
}

// y = G^T r (k_gband<true> with OpInnerStore).
template <int TPB, int PF = 0>
__device__ __forceinline__ void gband_t_rows(const GBandView &B, const float *r, float *y) {
  const int N = B.N;
  const unsigned short *gv = reinterpret_cast<const unsigned short *>(B.val);
  const int stride = gridDim.x * TPB;
  for (int i = blockIdx.x * TPB + threadIdx.x; i < N; i += stride) {
    prefetch_row<8, PF>(B.val, i, stride, N);
    float v[4], xv[4];
    v[0] = bf16_bits_to_float(__ldg(&gv[(size_t)i * 4]));
    xv[0] = ldv(r + i);
#pragma unroll
    for (int k = 1; k < 4; k++) {
      const unsigned j = (unsigned)i + (unsigned)B.d[k];
      const int jc = (int)min(j, (unsigned)(N - 1));
      v[k] = bf16_bits_to_float(__ldg(&gv[(size_t)jc * 4 + k]));
      xv[k] = ldv(r + jc);
      v[k] = j < (unsigned)N ? v[k] : 0.f;
    }
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) sum = fmaf(v[k], xv[k], sum);
    y[i] = sum;
  }
}

// r -= a q (k_inner_update_z / k_inner_update), and with D also d += a p
// (the d half of k_inner_direction; p does not change before the direction
// phase); this thread's partial of <r,r> and, with C (Jacobi), of <r,Cr>.
template <int TPB, bool D>
__device__ __forceinline__ void update_rows(int N, float *r, const float *q, float *d,
                                            const float *p, const float *C, float a,
                                            double &rr, double &rz) {
  const float na = -a;
  rr = 0.0;
  rz = 0.0;
  auto dots = [&](float ri, float ci) {
    rr = fma((double)ri, (double)ri, rr);
    if (C) rz = fma((double)ri, (double)(ci * ri), rz);
  };
  rows4<TPB>(
      N,
      [&](int i) {
        // Every load before the first store: the compiler cannot tell that
        // r, d and p do not overlap, so a load after a store would wait
        // for it.
        float4 rv = ldv4(r, i), dv = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 qv = ldv4(q, i);
        float4 pv = dv;
        if (D) {
          dv = ldv4(d, i);
          pv = ldv4(p, i);
        }
        rv.x = fmaf(na, qv.x, rv.x);
        rv.y = fmaf(na, qv.y, rv.y);
        rv.z = fmaf(na, qv.z, rv.z);
        rv.w = fmaf(na, qv.w, rv.w);
        dv.x = fmaf(a, pv.x, dv.x);
        dv.y = fmaf(a, pv.y, dv.y);
        dv.z = fmaf(a, pv.z, dv.z);
        dv.w = fmaf(a, pv.w, dv.w);
        reinterpret_cast<float4 *>(r)[i] = rv;
        if (D) reinterpret_cast<float4 *>(d)[i] = dv;
        const float4 cv =
            C ? __ldg(reinterpret_cast<const float4 *>(C) + i) : make_float4(0.f, 0.f, 0.f, 0.f);
        dots(rv.x, cv.x);
        dots(rv.y, cv.y);
        dots(rv.z, cv.z);
        dots(rv.w, cv.w);
      },
      [&](int i) {
        const float ri = fmaf(na, ldv(q + i), ldv(r + i));
        r[i] = ri;
        if (D) d[i] = fmaf(a, ldv(p + i), ldv(d + i));
        dots(ri, C ? __ldg(C + i) : 0.f);
      });
}

// p = z + b p (learned, k_inner_direction_z) or p = C r + b p (Jacobi,
// k_inner_direction: z = nullptr); with D first d += a p, p read once for
// both updates.
template <int TPB, bool D>
__device__ __forceinline__ void direction_rows(int N, float *p, float *d, const float *z,
                                               const float *r, const float *C, float a,
                                               float b) {
  rows4<TPB>(
      N,
      [&](int i) {
        const float4 pv = ldv4(p, i);
        float4 dv = D ? ldv4(d, i) : make_float4(0.f, 0.f, 0.f, 0.f);
        float4 zv;
        if (z) {
          zv = ldv4(z, i);
        } else {
          const float4 rv = ldv4(r, i), cv = __ldg(reinterpret_cast<const float4 *>(C) + i);
          zv = make_float4(cv.x * rv.x, cv.y * rv.y, cv.z * rv.z, cv.w * rv.w);
        }
        if (D) {
          dv.x = fmaf(a, pv.x, dv.x);
          dv.y = fmaf(a, pv.y, dv.y);
          dv.z = fmaf(a, pv.z, dv.z);
          dv.w = fmaf(a, pv.w, dv.w);
          reinterpret_cast<float4 *>(d)[i] = dv;
        }
        reinterpret_cast<float4 *>(p)[i] =
            make_float4(fmaf(b, pv.x, zv.x), fmaf(b, pv.y, zv.y), fmaf(b, pv.z, zv.z),
                        fmaf(b, pv.w, zv.w));
      },
      [&](int i) {
        const float pi = ldv(p + i);
        const float zi = z ? ldv(z + i) : __ldg(C + i) * ldv(r + i);
        if (D) d[i] = fmaf(a, pi, ldv(d + i));
        p[i] = fmaf(b, pi, zi);
      });
}

}  // namespace cgx
