// Device kernels of libcgb200.
//
// Sparse matrix-vector products (CRS and tile-major ELL, both staged by
// bulk copies; COO runs on its row-grouped CRS), each taking a row epilogue
// ("Op") so that the product is fused
// with whatever the conjugate-gradient step does with the row result: store
// it, form a dot product, form the residual, ... Ops with accumulators end
// with a deterministic grid-wide reduction whose last CTA runs the Op's
// finalize(), which updates the solver scalars in device memory.
//
// FP64 arithmetic that the reference performs as separate multiplies and adds
// (serial/SerialCG.cpp:79-174) is written with __dmul_rn / __dadd_rn so that
// the compiler does not contract it into FMAs: the SpMV rows, axpy, xpay and
// the Jacobi apply are then bit-identical to the reference's serial kernels.
// Only the dot products differ, by summation order.
#pragma once

#include "device.cuh"

namespace cgx {

// ---------------------------------------------------------------------------
// Matrix views (device pointers). Index/value arrays carry kPad elements of
// padding so that 16-byte-rounded bulk copies stay inside the allocation.

// CRS with value storage VT (double, float or half) and index storage IT:
// int holds the column itself, int16_t the column minus the row (used when
// every entry lies within 32767 of the diagonal, which halves index bytes).
template <typename VT, typename IT = int>
struct CrsView {
  const int *ptr;
  const IT *index;
  const VT *value;
  int N;
  int tile_cap;  // max nonzeros of a staged 256-row tile; 0 disables staging
  int warp_cap;  // > 0: 256-row tiles overflow tile_cap, and k_crs_warp stages
                 // 32-row tiles of up to warp_cap nonzeros instead
};

// Arithmetic type of a value storage type: half values are widened to FP32.
template <typename VT>
struct Comp {
  using T = VT;
};
template <>
struct Comp<__half> {
  using T = float;
};
template <>
struct Comp<__nv_bfloat16> {
  using T = float;
};

__device__ __forceinline__ int column(int, int stored) { return stored; }
__device__ __forceinline__ int column(int row, int16_t stored) {
  return row + (int)stored;
}

// ELL on the device, tile-major: rows are cut into 256-row tiles and tile t
// holds its slots one after another, each as 256 consecutive entries, so
// element (i, j) is at (t * width + j) * 256 + i % 256 with t = i / 256. The
// reference's column-major array (element (i, j) at j * N + i) is rearranged
// this way at upload. Within a slot, consecutive rows are adjacent, as in the
// column-major form, and a whole tile is one contiguous block. The last tile
// is allocated in full (its gap rows are zero).
template <typename VT>
struct EllView {
  const int *length;
  const int *index;
  const VT *data;
  int N;
  int width;
};

static_assert(kThreads == 256, "ELL tiles are the 256-row CTA tiles");
__host__ __device__ inline size_t ell_at(int i, int j, int width) {
  return ((size_t)(i >> 8) * (size_t)width + (size_t)j) * 256 + (size_t)(i & 255);
}
__host__ __device__ inline size_t ell_elems(int N, int width) {
  return (((size_t)N + 255) >> 8) * 256 * (size_t)width;
}

// Multiply-add of one matrix entry. FP64 keeps the reference's separate
// rounding; FP32 (the inner solve of the mixed path) uses an FMA.
__device__ __forceinline__ double madd(double acc, double v, double x) {
  return __dadd_rn(acc, __dmul_rn(v, x));
}
__device__ __forceinline__ float madd(float acc, float v, float x) {
  return fmaf(v, x, acc);
}
__device__ __forceinline__ float madd(float acc, __half v, float x) {
  return fmaf(__half2float(v), x, acc);
}
__device__ __forceinline__ float madd(float acc, __nv_bfloat16 v, float x) {
  return fmaf(__bfloat162float(v), x, acc);
}

template <typename VT>
__host__ __device__ constexpr int vals_per_16B() {
  return 16 / (int)sizeof(VT);
}

__host__ __device__ inline size_t align16(size_t b) {
  return (b + 15) & ~(size_t)15;
}

// Sum of row entries [j0, j1) in storage order: value(j) * x[col(j)]. The
// loads of a group of 8 entries are all issued before the first multiply-add,
// so up to 8 gathers of x are in flight per thread; the additions still run
// one after another in entry order, so the FP64 result is unchanged.
template <typename VT, int U = 8, typename ValF, typename ColF>
__device__ __forceinline__ VT row_sum(int j0, int j1, ValF val, ColF col,
                                      const VT *__restrict__ x) {
  VT sum = 0;
  for (int j = j0; j < j1; j += U) {
    VT v[U], xv[U];
#pragma unroll
    for (int k = 0; k < U; k++) {
      if (j + k < j1) {
        v[k] = val(j + k);
        xv[k] = __ldg(&x[col(j + k)]);
      }
    }
#pragma unroll
    for (int k = 0; k < U; k++)
      if (j + k < j1) sum = madd(sum, v[k], xv[k]);
  }
  return sum;
}

// Row sum from shared-memory staged values/indices: the U gathers of x of a
// group are issued first (only they occupy registers); the values are read
// from shared memory just before each multiply-add, in entry order.
template <typename VT, typename IT, int U, typename XT = typename Comp<VT>::T>
__device__ __forceinline__ XT row_sum_staged(int row, int j0, int j1,
                                             const VT *__restrict__ sv,
                                             const IT *__restrict__ si,
                                             const XT *__restrict__ x) {
  XT sum = 0;
  for (int j = j0; j < j1; j += U) {
    XT xv[U];
#pragma unroll
    for (int k = 0; k < U; k++)
      if (j + k < j1) xv[k] = __ldg(&x[column(row, si[j + k])]);
#pragma unroll
    for (int k = 0; k < U; k++)
      if (j + k < j1) sum = madd(sum, sv[j + k], xv[k]);
  }
  return sum;
}

// Plain sequential row sum (rare paths where ILP does not matter).
template <typename VT, typename ValF, typename ColF>
__device__ __forceinline__ VT row_sum_serial(int j0, int j1, ValF val,
                                             ColF col,
                                             const VT *__restrict__ x) {
  VT sum = 0;
  for (int j = j0; j < j1; j++) sum = madd(sum, val(j), __ldg(&x[col(j)]));
  return sum;
}

// Dynamic shared memory of the staged CRS kernel for a given tile capacity:
// two stages of cap + 16 values and indices (room for the 16-byte rounding
// of both ends of a tile's range).
template <typename VT, typename IT = int>
__host__ __device__ inline size_t crs_stage_bytes(int cap) {
  return align16((size_t)(cap + 16) * sizeof(VT)) +
         align16((size_t)(cap + 16) * sizeof(IT));
}
template <typename VT, typename IT = int>
__host__ __device__ inline size_t crs_smem_bytes(int cap) {
  return cap > 0 ? 16 + 2 * crs_stage_bytes<VT, IT>(cap) : 16;
}

// ---------------------------------------------------------------------------
// CRS SpMV, persistent: CTA b handles 256-row tiles b, b+grid, ... One thread
// owns one row and sums it sequentially in storage order (the reference's
// order). A tile's value/index range is brought into shared memory by two
// 1-D bulk copies (TMA) issued one tile ahead, double-buffered on two
// mbarriers; the x gathers go through the read-only path and mostly hit L2.
// Tiles whose range exceeds tile_cap are read straight from global memory.

template <typename VT, typename IT, typename Op,
          typename XT = typename Comp<VT>::T>
__global__ void __launch_bounds__(kThreads)
    k_crs(CrsView<VT, IT> A, const XT *__restrict__ x, Op op, CgState *st,
          double *partials) {
  if (op.skip(st)) return;
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int VPER = vals_per_16B<VT>();
  constexpr int IPER = vals_per_16B<IT>();
  const int cap = A.tile_cap;
  const int N = A.N;
  const int nTiles = (N + kThreads - 1) / kThreads;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  const size_t vbytes = align16((size_t)(cap + 16) * sizeof(VT));
  const size_t sbytes = crs_stage_bytes<VT, IT>(cap);
  VT *sval0 = reinterpret_cast<VT *>(smem + 16);
  IT *sidx0 = reinterpret_cast<IT *>(smem + 16 + vbytes);
  VT *sval1 = reinterpret_cast<VT *>(smem + 16 + sbytes);
  IT *sidx1 = reinterpret_cast<IT *>(smem + 16 + sbytes + vbytes);

  if (cap > 0 && threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncthreads();

  auto issue = [&](int t, int buf) {
    const int r0 = t * kThreads;
    const int r1 = min(N, r0 + kThreads);
    const int s = __ldg(&A.ptr[r0]), e = __ldg(&A.ptr[r1]);
    if (!(cap > 0 && e > s && e - s <= cap)) return;
    const int vs = s & ~(VPER - 1), ve = (e + VPER - 1) & ~(VPER - 1);
    const int is = s & ~(IPER - 1), ie = (e + IPER - 1) & ~(IPER - 1);
    const unsigned vb = (unsigned)(ve - vs) * (unsigned)sizeof(VT);
    const unsigned ib = (unsigned)(ie - is) * (unsigned)sizeof(IT);
    mbar_arrive_expect_tx(&bars[buf], vb + ib);
    bulk_g2s(buf ? sval1 : sval0, A.value + vs, vb, &bars[buf]);
    bulk_g2s(buf ? sidx1 : sidx0, A.index + is, ib, &bars[buf]);
  };

  typename Op::Acc acc;
  unsigned ph0 = 0, ph1 = 0;
  int k = 0;
  int t = blockIdx.x;
  if (threadIdx.x == 0 && t < nTiles) issue(t, 0);
  for (; t < nTiles; t += gridDim.x, k++) {
    const int buf = k & 1;
    const int tn = t + gridDim.x;
    if (threadIdx.x == 0 && tn < nTiles) issue(tn, buf ^ 1);
    const int r0 = t * kThreads;
    const int r1 = min(N, r0 + kThreads);
    const int s = __ldg(&A.ptr[r0]), e = __ldg(&A.ptr[r1]);
    const bool staged = cap > 0 && e > s && e - s <= cap;
    // The row bounds are loaded before the wait so that their latency
    // overlaps the bulk copy's.
    const int row = r0 + threadIdx.x;
    const int j0 = row < r1 ? __ldg(&A.ptr[row]) : 0;
    const int j1 = row < r1 ? __ldg(&A.ptr[row + 1]) : 0;
    bool ok = true;
    if (staged) {
      ok = mbar_wait_bounded(&bars[buf], buf ? ph1 : ph0);
      if (buf) ph1 ^= 1u; else ph0 ^= 1u;
      if (!ok && threadIdx.x == 0) atomicOr(&st->error, kErrBarrierTimeout);
    }
    if (row < r1) {
      XT sum = 0;
      if (staged) {
        if (ok) {
          const VT *sv = (buf ? sval1 : sval0) - (s & ~(VPER - 1));
          const IT *si = (buf ? sidx1 : sidx0) - (s & ~(IPER - 1));
          sum = row_sum_staged<VT, IT, 8>(row, j0, j1, sv, si, x);
        }
      } else {
        for (int j = j0; j < j1; j++)
          sum = madd(sum, A.value[j], __ldg(&x[column(row, A.index[j])]));
      }
      op.row(row, sum, acc);
    }
    __syncthreads();
  }
  op.finish(acc, st, partials);
}

// CRS SpMV for rows too long for k_crs's 256-row tiles (a tile above its
// capacity would take the direct path, whose per-thread row loads do not
// coalesce): each warp stages its own 32-row tiles (warp w of the grid takes
// tiles w, w + warps, ...). One lane issues the tile's two 1-D bulk copies
// into the warp's shared-memory slot (A.warp_cap nonzeros) on the warp's
// mbarrier, and every lane then sums its row from the slot in storage order,
// as k_crs does, so the FP64 result is the same. One stage per warp: the
// copies of the SM's other warps overlap a warp's summation.
template <typename VT, typename IT, typename Op,
          typename XT = typename Comp<VT>::T>
__global__ void __launch_bounds__(kThreads)
    k_crs_warp(CrsView<VT, IT> A, const XT *__restrict__ x, Op op, CgState *st,
               double *partials) {
  if (op.skip(st)) return;
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int VPER = vals_per_16B<VT>();
  constexpr int IPER = vals_per_16B<IT>();
  const int cap = A.warp_cap;
  const int N = A.N;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  const size_t vbytes = align16((size_t)(cap + 16) * sizeof(VT));
  const size_t sbytes = crs_stage_bytes<VT, IT>(cap);
  unsigned char *slot = smem + 16 * kWarps + (size_t)warp * sbytes;
  VT *sv = reinterpret_cast<VT *>(slot);
  IT *si = reinterpret_cast<IT *>(slot + vbytes);
  if (threadIdx.x == 0) {
    for (int w = 0; w < kWarps; w++) mbar_init(&bars[w], 1);
    mbar_fence_init();
  }
  __syncthreads();

  typename Op::Acc acc;
  unsigned phase = 0;
  const int ntiles = (N + 31) >> 5;
  const int nw = gridDim.x * kWarps;
  for (int t = blockIdx.x * kWarps + warp; t < ntiles; t += nw) {
    const int r0 = t << 5, r1 = min(N, r0 + 32);
    const int s = __ldg(&A.ptr[r0]), e = __ldg(&A.ptr[r1]);
    const bool staged = e > s && e - s <= cap;
    const int row = r0 + lane;
    const int j0 = row < r1 ? __ldg(&A.ptr[row]) : 0;
    const int j1 = row < r1 ? __ldg(&A.ptr[row + 1]) : 0;
    const int vs = s & ~(VPER - 1), is = s & ~(IPER - 1);
    bool ok = true;
    if (staged) {
      if (lane == 0) {
        const int ve = (e + VPER - 1) & ~(VPER - 1);
        const int ie = (e + IPER - 1) & ~(IPER - 1);
        const unsigned vb = (unsigned)(ve - vs) * (unsigned)sizeof(VT);
        const unsigned ib = (unsigned)(ie - is) * (unsigned)sizeof(IT);
        mbar_arrive_expect_tx(&bars[warp], vb + ib);
        bulk_g2s(sv, A.value + vs, vb, &bars[warp]);
        bulk_g2s(si, A.index + is, ib, &bars[warp]);
      }
      ok = mbar_wait_bounded(&bars[warp], phase);
      phase ^= 1u;
      if (!ok && lane == 0) atomicOr(&st->error, kErrBarrierTimeout);
    }
    if (row < r1) {
      XT sum = 0;
      if (staged) {
        if (ok) sum = row_sum_staged<VT, IT, 8>(row, j0, j1, sv - vs, si - is, x);
      } else {
        for (int j = j0; j < j1; j++)
          sum = madd(sum, A.value[j], __ldg(&x[column(row, A.index[j])]));
      }
      op.row(row, sum, acc);
    }
    __syncwarp();  // the slot is read before the warp's next copy lands
  }
  op.finish(acc, st, partials);
}

// Column indices as 16-bit offsets from the row (the compact CRS of the
// mixed and learned paths); sets *flag if an offset does not fit.
__global__ void __launch_bounds__(kThreads)
    k_delta16(int N, const int *__restrict__ ptr, const int *__restrict__ index,
              int16_t *__restrict__ out, int *flag) {
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads)
    for (int j = ptr[i]; j < ptr[i + 1]; j++) {
      const int d = index[j] - i;
      if (d < -32768 || d > 32767) {
        atomicOr(flag, 1);
        out[j] = 0;
      } else {
        out[j] = (int16_t)d;
      }
    }
}

// ---------------------------------------------------------------------------
// ELL SpMV. Rows stop at length[i] (the reference leaves padding slots
// uninitialised, Matrix.cpp:339-361), and each row is summed from 0 over its
// slots in order, so the FP64 result equals the reference's.
//
// k_ell_tma, persistent, for widths up to kEllStagedWidth: CTA b handles
// 256-row tiles b, b + grid, ... One thread brings a tile's values and
// indices (two contiguous blocks of the tile-major layout) into shared memory
// with two 1-D bulk copies (TMA) one tile ahead, double-buffered on two
// mbarriers, as k_crs does for a CRS tile. The x gathers go through the
// read-only path and mostly hit L2.

constexpr int kEllStagedWidth = 16;

template <typename VT>
__host__ __device__ inline size_t ell_stage_bytes(int width) {
  return (size_t)width * kThreads * (sizeof(VT) + sizeof(int));
}
template <typename VT>
__host__ __device__ inline size_t ell_smem_bytes(int width) {
  return 16 + 2 * ell_stage_bytes<VT>(width);
}

template <typename VT, typename Op>
__global__ void __launch_bounds__(kThreads)
    k_ell_tma(EllView<VT> A, const VT *__restrict__ x, Op op, CgState *st,
              double *partials) {
  if (op.skip(st)) return;
  extern __shared__ __align__(16) unsigned char smem[];
  const int W = A.width, N = A.N;
  const int nTiles = (N + kThreads - 1) / kThreads;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  const size_t sbytes = ell_stage_bytes<VT>(W);
  const size_t vbytes = (size_t)W * kThreads * sizeof(VT);
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncthreads();

  // A tile is two contiguous blocks (values, indices) of the tile-major
  // layout: one bulk copy each.
  auto issue = [&](int t, int buf) {
    unsigned char *stage = smem + 16 + (size_t)buf * sbytes;
    const size_t base = (size_t)t * W * kThreads;
    mbar_arrive_expect_tx(&bars[buf], (unsigned)sbytes);
    bulk_g2s(stage, A.data + base, (unsigned)vbytes, &bars[buf]);
    bulk_g2s(stage + vbytes, A.index + base, (unsigned)(sbytes - vbytes),
             &bars[buf]);
  };

  typename Op::Acc acc;
  unsigned ph0 = 0, ph1 = 0;
  int k = 0;
  int t = blockIdx.x;
  if (threadIdx.x == 0 && t < nTiles) issue(t, 0);
  for (; t < nTiles; t += gridDim.x, k++) {
    const int buf = k & 1;
    const int tn = t + gridDim.x;
    if (threadIdx.x == 0 && tn < nTiles) issue(tn, buf ^ 1);
    const int row = t * kThreads + threadIdx.x;
    const int len = row < N ? __ldg(&A.length[row]) : 0;
    const bool ok = mbar_wait_bounded(&bars[buf], buf ? ph1 : ph0);
    if (buf) ph1 ^= 1u; else ph0 ^= 1u;
    if (!ok && threadIdx.x == 0) atomicOr(&st->error, kErrBarrierTimeout);
    if (row < N) {
      VT sum = 0;
      if (ok) {
        const unsigned char *stage = smem + 16 + (size_t)buf * sbytes;
        const VT *sv = reinterpret_cast<const VT *>(stage) + threadIdx.x;
        const int *si =
            reinterpret_cast<const int *>(stage + vbytes) + threadIdx.x;
        for (int j0 = 0; j0 < len; j0 += 8) {
          VT xv[8];
#pragma unroll
          for (int u = 0; u < 8; u++)
            if (j0 + u < len) xv[u] = __ldg(&x[si[(j0 + u) * kThreads]]);
#pragma unroll
          for (int u = 0; u < 8; u++)
            if (j0 + u < len) sum = madd(sum, sv[(j0 + u) * kThreads], xv[u]);
        }
      }
      op.row(row, sum, acc);
    }
    __syncthreads();
  }
  op.finish(acc, st, partials);
}

// k_ell, for wider rows: one thread per row, loads straight from global
// memory; consecutive threads read consecutive rows, so every load of a
// column is coalesced.
template <typename VT, typename Op>
__global__ void __launch_bounds__(kThreads)
    k_ell(EllView<VT> A, const VT *__restrict__ x, Op op, CgState *st,
          double *partials) {
  if (op.skip(st)) return;
  typename Op::Acc acc;
  const int N = A.N;
  for (int row = blockIdx.x * kThreads + threadIdx.x; row < N;
       row += gridDim.x * kThreads) {
    const int len = __ldg(&A.length[row]);
    const size_t o = ell_at(row, 0, A.width);
    const VT *dat = A.data + o;
    const int *idx = A.index + o;
    const VT sum = row_sum<VT, 4>(
        0, len, [&](int j) { return __ldg(&dat[j * kThreads]); },
        [&](int j) { return __ldg(&idx[j * kThreads]); }, x);
    op.row(row, sum, acc);
  }
  op.finish(acc, st, partials);
}

// ---------------------------------------------------------------------------
// Row epilogues.

struct NoAcc {};
struct Acc1 {
  double a0 = 0.0;
};
struct Acc2 {
  double a0 = 0.0, a1 = 0.0;
};

// y = A x (CG::matvecKernel). Never skipped.
template <typename VT>
struct OpStore {
  using Acc = NoAcc;
  VT *y;
  __device__ bool skip(const CgState *) const { return false; }
  __device__ void row(int i, VT s, Acc &) const { y[i] = s; }
  __device__ void finish(Acc &, CgState *, double *) const {}
};

// Solve set-up (CG.cpp:293-318): r = k - A x, p = C r (or r), then
// r2 = <r,r>, nrm2_0 = sqrt(r2), rho = <p,r> (or r2).
template <bool JACOBI>
struct OpSetup {
  using Acc = Acc2;
  const double *k;
  double *r, *p;
  const double *C;
  unsigned *ticket;
  __device__ bool skip(const CgState *) const { return false; }
  __device__ void row(int i, double s, Acc &a) const {
    const double ri = __dadd_rn(__ldg(&k[i]), __dmul_rn(-1.0, s));
    const double pi = JACOBI ? __dmul_rn(__ldg(&C[i]), ri) : ri;
    r[i] = ri;
    p[i] = pi;
    a.a0 = fma(ri, ri, a.a0);
    a.a1 = fma(pi, ri, a.a1);
  }
  __device__ void finish(Acc &a, CgState *st, double *partials) const {
    double in[2] = {a.a0, a.a1}, out[2];
    if (grid_reduce<2>(in, partials, ticket, out) && threadIdx.x == 0) {
      st->r2 = out[0];
      st->nrm0 = sqrt(out[0]);
      st->rho = JACOBI ? out[1] : out[0];
      st->iteration = 0;
      st->converged = 0;
      st->finished = 0;
      st->stop = st->max_iter <= 0;
      st->residual = 0.0;
      if (st->use_cond)
        cudaGraphSetConditional((cudaGraphConditionalHandle)st->cond,
                                st->stop ? 0u : 1u);
    }
  }
};

// q = A p fused with <p,q>; finalize a = rho / <p,q> (CG.cpp:324-334).
struct OpPcgQ {
  using Acc = Acc1;
  const double *p;
  double *q;
  unsigned *ticket;
  __device__ bool skip(CgState *st) const {
    if (st->stop) {
      if (blockIdx.x == 0 && threadIdx.x == 0) st->finished = 1;
      return true;
    }
    return false;
  }
  __device__ void row(int i, double s, Acc &a) const {
    q[i] = s;
    a.a0 = fma(__ldg(&p[i]), s, a.a0);
  }
  __device__ void finish(Acc &a, CgState *st, double *partials) const {
    double in[1] = {a.a0}, out[1];
    if (grid_reduce<1>(in, partials, ticket, out) && threadIdx.x == 0) {
      st->pq = out[0];
      st->alpha = st->rho / out[0];
    }
  }
};

// FP64 true residual of the refinement loop: r = b - A x, <r,r>.
struct OpTrueResidual {
  using Acc = Acc1;
  const double *b;
  double *r;
  unsigned *ticket;
  __device__ bool skip(const CgState *) const { return false; }
  __device__ void row(int i, double s, Acc &a) const {
    const double ri = __ldg(&b[i]) - s;
    r[i] = ri;
    a.a0 = fma(ri, ri, a.a0);
  }
  __device__ void finish(Acc &a, CgState *st, double *partials) const {
    double in[1] = {a.a0}, out[1];
    if (grid_reduce<1>(in, partials, ticket, out) && threadIdx.x == 0)
      st->r2 = out[0];
  }
};

// Inner FP32 solve: q = A p fused with <p,q> (FP64 accumulation).
struct OpInnerQ {
  using Acc = Acc1;
  const float *p;
  float *q;
  unsigned *ticket;
  __device__ bool skip(CgState *st) const {
    if (st->in_stop) {
      if (blockIdx.x == 0 && threadIdx.x == 0) st->in_finished = 1;
      return true;
    }
    return false;
  }
  __device__ void row(int i, float s, Acc &a) const {
    q[i] = s;
    a.a0 = fma((double)__ldg(&p[i]), (double)s, a.a0);
  }
  struct Pre {
    float p;
  };
  __device__ Pre prefetch(int i) const { return Pre{__ldg(&p[i])}; }
  __device__ void row(int i, float s, Acc &a, const Pre &pr) const {
    q[i] = s;
    a.a0 = fma((double)pr.p, (double)s, a.a0);
  }
  __device__ void finish(Acc &a, CgState *st, double *partials) const {
    double in[1] = {a.a0}, out[1];
    if (grid_reduce<1>(in, partials, ticket, out) && threadIdx.x == 0)
      st->in_alpha = st->in_rho / out[0];
  }
};

// ---------------------------------------------------------------------------
// Fused vector steps of one PCG iteration (CG.cpp:339-381). The update of x
// is deferred from step 2 to step 3, where p is read anyway; the result is
// the same x because x(i+1) = x(i) + a p(i) only needs p(i), which step 3
// reads before overwriting it.

// Step 2: r -= a q; z = C r (not stored); partials of <r,r> and <r,z>;
// finalize: residual test, rho, b, stop flag, conditional-node value.
template <bool JACOBI>
__global__ void __launch_bounds__(kThreads)
    k_pcg_update(int N, double *__restrict__ r, const double *__restrict__ q,
                 const double *__restrict__ C, CgState *st, double *partials,
                 unsigned *ticket) {
  if (st->stop) return;
  const double na = -st->alpha;
  double rr = 0.0, rz = 0.0;
  const int n2 = N >> 1;
  double2 *r2p = reinterpret_cast<double2 *>(r);
  const double2 *q2p = reinterpret_cast<const double2 *>(q);
  const double2 *c2p = reinterpret_cast<const double2 *>(C);
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n2;
       i += gridDim.x * kThreads) {
    double2 rv = r2p[i];
    const double2 qv = __ldg(&q2p[i]);
    rv.x = __dadd_rn(rv.x, __dmul_rn(na, qv.x));
    rv.y = __dadd_rn(rv.y, __dmul_rn(na, qv.y));
    r2p[i] = rv;
    rr = fma(rv.x, rv.x, rr);
    rr = fma(rv.y, rv.y, rr);
    if (JACOBI) {
      const double2 cv = __ldg(&c2p[i]);
      rz = fma(rv.x, __dmul_rn(cv.x, rv.x), rz);
      rz = fma(rv.y, __dmul_rn(cv.y, rv.y), rz);
    }
  }
  if ((N & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const int i = N - 1;
    const double ri = __dadd_rn(r[i], __dmul_rn(na, q[i]));
    r[i] = ri;
    rr = fma(ri, ri, rr);
    if (JACOBI) rz = fma(ri, __dmul_rn(C[i], ri), rz);
  }
  double in[2] = {rr, rz}, out[2];
  if (grid_reduce<2>(in, partials, ticket, out) && threadIdx.x == 0) {
    st->r2 = out[0];
    const double res = sqrt(out[0]) / st->nrm0;
    st->residual = res;
    st->iteration += 1;
    if (res <= st->tol) {
      st->converged = 1;
      st->stop = 1;
    } else {
      st->rho_old = st->rho;
      st->rho = JACOBI ? out[1] : out[0];
      st->beta = st->rho / st->rho_old;
      if (st->iteration >= st->max_iter) st->stop = 1;
    }
    if (st->use_cond)
      cudaGraphSetConditional((cudaGraphConditionalHandle)st->cond,
                              st->stop ? 0u : 1u);
  }
}

// Step 3: x += a p(i); unless stopping, p = z + b p(i) with z = C r.
template <bool JACOBI>
__global__ void __launch_bounds__(kThreads)
    k_pcg_direction(int N, double *__restrict__ x, double *__restrict__ p,
                    const double *__restrict__ r, const double *__restrict__ C,
                    CgState *st) {
  if (st->finished) return;
  const double a = st->alpha, b = st->beta;
  const bool upd = !st->stop;
  const int n2 = N >> 1;
  double2 *x2 = reinterpret_cast<double2 *>(x);
  double2 *p2 = reinterpret_cast<double2 *>(p);
  const double2 *r2 = reinterpret_cast<const double2 *>(r);
  const double2 *c2 = reinterpret_cast<const double2 *>(C);
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n2;
       i += gridDim.x * kThreads) {
    const double2 pv = p2[i];
    double2 xv = x2[i];
    xv.x = __dadd_rn(xv.x, __dmul_rn(a, pv.x));
    xv.y = __dadd_rn(xv.y, __dmul_rn(a, pv.y));
    x2[i] = xv;
    if (upd) {
      double2 zv = __ldg(&r2[i]);
      if (JACOBI) {
        const double2 cv = __ldg(&c2[i]);
        zv.x = __dmul_rn(cv.x, zv.x);
        zv.y = __dmul_rn(cv.y, zv.y);
      }
      double2 pn;
      pn.x = __dadd_rn(zv.x, __dmul_rn(b, pv.x));
      pn.y = __dadd_rn(zv.y, __dmul_rn(b, pv.y));
      p2[i] = pn;
    }
  }
  if ((N & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const int i = N - 1;
    const double pv = p[i];
    x[i] = __dadd_rn(x[i], __dmul_rn(a, pv));
    if (upd) {
      const double zv = JACOBI ? __dmul_rn(C[i], r[i]) : r[i];
      p[i] = __dadd_rn(zv, __dmul_rn(b, pv));
    }
  }
}

// ---------------------------------------------------------------------------
// Single-purpose kernels behind the reference's per-kernel interface
// (CG.h:224-237), used when CG::solve drives the device one call at a time.

__global__ void __launch_bounds__(kThreads)
    k_axpy(int N, double a, const double *__restrict__ x,
           double *__restrict__ y) {
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads)
    y[i] = __dadd_rn(y[i], __dmul_rn(a, x[i]));
}

__global__ void __launch_bounds__(kThreads)
    k_xpay(int N, const double *__restrict__ x, double a,
           double *__restrict__ y) {
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads)
    y[i] = __dadd_rn(x[i], __dmul_rn(a, y[i]));
}

__global__ void __launch_bounds__(kThreads)
    k_jacobi(int N, const double *__restrict__ C, const double *__restrict__ x,
             double *__restrict__ y) {
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads)
    y[i] = __dmul_rn(C[i], x[i]);
}

// <a,b> into *out (device), deterministic two-level reduction.
__global__ void __launch_bounds__(kThreads)
    k_dot(int N, const double *__restrict__ a, const double *__restrict__ b,
          double *out, double *partials, unsigned *ticket) {
  double s = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads)
    s = fma(a[i], b[i], s);
  double in[1] = {s}, res[1];
  if (grid_reduce<1>(in, partials, ticket, res) && threadIdx.x == 0)
    *out = res[0];
}

// C[i] = 1 / (last diagonal entry of row i in storage order), 0 if none:
// Jacobi::init (Preconditioner.cpp:13-23) on the CRS arrays, whose rows keep
// file order (Matrix.cpp:203-228).
__global__ void __launch_bounds__(kThreads)
    k_jacobi_from_crs(int N, const int *__restrict__ ptr,
                      const int *__restrict__ index,
                      const double *__restrict__ value, double *C) {
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads) {
    double c = 0.0;
    for (int j = ptr[i]; j < ptr[i + 1]; j++)
      if (index[j] == i) c = 1 / value[j];
    C[i] = c;
  }
}

__global__ void __launch_bounds__(kThreads)
    k_to_f32(size_t n, const double *__restrict__ a, float *__restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < n;
       i += (size_t)gridDim.x * kThreads)
    b[i] = (float)a[i];
}

__global__ void __launch_bounds__(kThreads)
    k_fill(size_t n, double v, double *__restrict__ a) {
  for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < n;
       i += (size_t)gridDim.x * kThreads)
    a[i] = v;
}

// ---------------------------------------------------------------------------
// Mixed-precision inner solve: FP32 Jacobi-PCG on A d = r / ||r|| with FP64
// scalars, inside an FP64 refinement loop driven by the host.

// Start: r32 = r64 / ||r64||, d = 0, p = C r32 (and z = p when z is given,
// for the fused persistent inner solve); <r,p>, <r,r>; a = b = 0, so that
// its first iteration forms p = z and leaves d at 0.
__global__ void __launch_bounds__(kThreads)
    k_inner_start(int N, const double *__restrict__ r64, float *__restrict__ r,
                  float *__restrict__ d, float *__restrict__ p,
                  const float *__restrict__ C, CgState *st, double *partials,
                  unsigned *ticket, float *__restrict__ z = nullptr) {
  const double inv = 1.0 / sqrt(st->r2);
  double rp = 0.0, rr = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads) {
    const float ri = (float)(r64[i] * inv);
    const float pi = C[i] * ri;
    r[i] = ri;
    d[i] = 0.0f;
    p[i] = pi;
    if (z) z[i] = pi;
    rp = fma((double)ri, (double)pi, rp);
    rr = fma((double)ri, (double)ri, rr);
  }
  double in[2] = {rp, rr}, out[2];
  if (grid_reduce<2>(in, partials, ticket, out) && threadIdx.x == 0) {
    st->in_rho = out[0];
    st->in_nrm0 = sqrt(out[1]);
    st->in_alpha = 0.0;
    st->in_beta = 0.0;
    st->in_iter = 0;
    st->in_stop = 0;
    st->in_finished = 0;
    if (st->use_cond)
      cudaGraphSetConditional((cudaGraphConditionalHandle)st->cond, 1u);
  }
}

// Inner step 2: r -= a q; partial <r,r>, <r,Cr>; finalize residual test and b.
__global__ void __launch_bounds__(kThreads)
    k_inner_update(int N, float *__restrict__ r, const float *__restrict__ q,
                   const float *__restrict__ C, CgState *st, double *partials,
                   unsigned *ticket) {
  if (st->in_stop) return;
  const float na = (float)(-st->in_alpha);
  double rr = 0.0, rz = 0.0;
  const int n4 = N >> 2;
  float4 *r4 = reinterpret_cast<float4 *>(r);
  const float4 *q4 = reinterpret_cast<const float4 *>(q);
  const float4 *c4 = reinterpret_cast<const float4 *>(C);
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n4;
       i += gridDim.x * kThreads) {
    float4 rv = r4[i];
    const float4 qv = __ldg(&q4[i]);
    const float4 cv = __ldg(&c4[i]);
    rv.x = fmaf(na, qv.x, rv.x);
    rv.y = fmaf(na, qv.y, rv.y);
    rv.z = fmaf(na, qv.z, rv.z);
    rv.w = fmaf(na, qv.w, rv.w);
    r4[i] = rv;
    const float4 zv = make_float4(cv.x * rv.x, cv.y * rv.y, cv.z * rv.z, cv.w * rv.w);
    rr = fma((double)rv.x, (double)rv.x, rr);
    rr = fma((double)rv.y, (double)rv.y, rr);
    rr = fma((double)rv.z, (double)rv.z, rr);
    rr = fma((double)rv.w, (double)rv.w, rr);
    rz = fma((double)rv.x, (double)zv.x, rz);
    rz = fma((double)rv.y, (double)zv.y, rz);
    rz = fma((double)rv.z, (double)zv.z, rz);
    rz = fma((double)rv.w, (double)zv.w, rz);
  }
  for (int i = 4 * n4 + blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads) {
    const float ri = fmaf(na, q[i], r[i]);
    r[i] = ri;
    const float zi = C[i] * ri;
    rr = fma((double)ri, (double)ri, rr);
    rz = fma((double)ri, (double)zi, rz);
  }
  double in[2] = {rr, rz}, out[2];
  if (grid_reduce<2>(in, partials, ticket, out) && threadIdx.x == 0) {
    st->in_iter += 1;
    st->total_inner += 1;
    const double res = sqrt(out[0]) / st->in_nrm0;
    st->in_res = res;
    if (!(res > st->in_tol) || inner_broke_down(st) ||
        st->total_inner >= st->max_iter) {
      st->in_stop = 1;
    } else {
      const double rho = out[1];
      st->in_beta = rho / st->in_rho;
      st->in_rho = rho;
    }
    if (st->use_cond)
      cudaGraphSetConditional((cudaGraphConditionalHandle)st->cond,
                              st->in_stop ? 0u : 1u);
  }
}

// Inner step 3: d += a p; unless stopping, p = C r + b p. It also runs in the
// iteration whose step 2 stopped the loop (that d update must not be lost);
// in a chunked loop the next step-1 launch then sets in_finished.
__global__ void __launch_bounds__(kThreads)
    k_inner_direction(int N, float *__restrict__ d, float *__restrict__ p,
                      const float *__restrict__ r, const float *__restrict__ C,
                      CgState *st) {
  if (st->in_finished) return;
  const float a = (float)st->in_alpha, b = (float)st->in_beta;
  const bool upd = !st->in_stop;
  const int n4 = N >> 2;
  float4 *d4 = reinterpret_cast<float4 *>(d);
  float4 *p4 = reinterpret_cast<float4 *>(p);
  const float4 *r4 = reinterpret_cast<const float4 *>(r);
  const float4 *c4 = reinterpret_cast<const float4 *>(C);
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n4;
       i += gridDim.x * kThreads) {
    const float4 pv = p4[i];
    float4 dv = d4[i];
    dv.x = fmaf(a, pv.x, dv.x);
    dv.y = fmaf(a, pv.y, dv.y);
    dv.z = fmaf(a, pv.z, dv.z);
    dv.w = fmaf(a, pv.w, dv.w);
    d4[i] = dv;
    if (upd) {
      const float4 rv = __ldg(&r4[i]);
      const float4 cv = __ldg(&c4[i]);
      float4 pn;
      pn.x = fmaf(b, pv.x, cv.x * rv.x);
      pn.y = fmaf(b, pv.y, cv.y * rv.y);
      pn.z = fmaf(b, pv.z, cv.z * rv.z);
      pn.w = fmaf(b, pv.w, cv.w * rv.w);
      p4[i] = pn;
    }
  }
  for (int i = 4 * n4 + blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads) {
    const float pv = p[i];
    d[i] = fmaf(a, pv, d[i]);
    if (upd) p[i] = fmaf(b, pv, C[i] * r[i]);
  }
}

// ---------------------------------------------------------------------------
// Inner FP32 PCG with an explicit preconditioned residual z = M^-1 r (the
// learned factor: z = G (G^T r) + eps C r, two SpMVs with a global
// dependency between them, so z is stored).

// Start: r32 = r64 / ||r64||, d = 0, ||r32||; the first z and p = z come from
// the apply that follows (OpLearnedZ in start mode).
__global__ void __launch_bounds__(kThreads)
    k_inner_start_z(int N, const double *__restrict__ r64,
                    float *__restrict__ r, float *__restrict__ d, CgState *st,
                    double *partials, unsigned *ticket) {
  const double inv = 1.0 / sqrt(st->r2);
  double rr = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads) {
    const float ri = (float)(r64[i] * inv);
    r[i] = ri;
    d[i] = 0.0f;
    rr = fma((double)ri, (double)ri, rr);
  }
  double in[1] = {rr}, out[1];
  if (grid_reduce<1>(in, partials, ticket, out) && threadIdx.x == 0) {
    st->in_nrm0 = sqrt(out[0]);
    st->in_iter = 0;
    st->in_stop = 0;
    st->in_finished = 0;
    if (st->use_cond)
      cudaGraphSetConditional((cudaGraphConditionalHandle)st->cond, 1u);
  }
}

// y = M r for the first factor of the apply; skipped once the loop stopped.
struct OpInnerStore {
  using Acc = NoAcc;
  struct Pre {};
  float *y;
  __device__ bool skip(const CgState *st) const { return st->in_stop != 0; }
  __device__ void row(int i, float s, Acc &) const { y[i] = s; }
  __device__ Pre prefetch(int) const { return Pre{}; }
  __device__ void row(int i, float s, Acc &, const Pre &) const { y[i] = s; }
  __device__ void finish(Acc &, CgState *, double *) const {}
};

// z = s + eps C r (s = row of G y), <r,z>; in start mode also p = z and
// rho = <r,z>, otherwise b = <r,z> / rho_old.
struct OpLearnedZ {
  using Acc = Acc1;
  const float *r, *C;
  float *z, *p;
  float eps;
  int start;
  unsigned *ticket;
  __device__ bool skip(const CgState *st) const { return st->in_stop != 0; }
  __device__ void row(int i, float s, Acc &a) const {
    row(i, s, a, prefetch(i));
  }
  struct Pre {
    float r, c;
  };
  __device__ Pre prefetch(int i) const { return Pre{__ldg(&r[i]), __ldg(&C[i])}; }
  __device__ void row(int i, float s, Acc &a, const Pre &pr) const {
    const float zi = fmaf(eps * pr.c, pr.r, s);
    z[i] = zi;
    if (start) p[i] = zi;
    a.a0 = fma((double)pr.r, (double)zi, a.a0);
  }
  __device__ void finish(Acc &a, CgState *st, double *partials) const {
    double in[1] = {a.a0}, out[1];
    if (grid_reduce<1>(in, partials, ticket, out) && threadIdx.x == 0) {
      if (start) {
        st->in_rho = out[0];
        st->in_alpha = 0.0;  // a fused first iteration: p = z, d stays 0
        st->in_beta = 0.0;
      } else {
        st->in_beta = out[0] / st->in_rho;
        st->in_rho = out[0];
      }
    }
  }
};

// r -= a q; <r,r>; residual test (z and b follow from the apply).
__global__ void __launch_bounds__(kThreads)
    k_inner_update_z(int N, float *__restrict__ r, const float *__restrict__ q,
                     CgState *st, double *partials, unsigned *ticket) {
  if (st->in_stop) return;
  const float na = (float)(-st->in_alpha);
  double rr = 0.0;
  const int n4 = N >> 2;
  float4 *r4 = reinterpret_cast<float4 *>(r);
  const float4 *q4 = reinterpret_cast<const float4 *>(q);
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n4;
       i += gridDim.x * kThreads) {
    float4 rv = r4[i];
    const float4 qv = __ldg(&q4[i]);
    rv.x = fmaf(na, qv.x, rv.x);
    rv.y = fmaf(na, qv.y, rv.y);
    rv.z = fmaf(na, qv.z, rv.z);
    rv.w = fmaf(na, qv.w, rv.w);
    r4[i] = rv;
    rr = fma((double)rv.x, (double)rv.x, rr);
    rr = fma((double)rv.y, (double)rv.y, rr);
    rr = fma((double)rv.z, (double)rv.z, rr);
    rr = fma((double)rv.w, (double)rv.w, rr);
  }
  for (int i = 4 * n4 + blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads) {
    const float ri = fmaf(na, q[i], r[i]);
    r[i] = ri;
    rr = fma((double)ri, (double)ri, rr);
  }
  double in[1] = {rr}, out[1];
  if (grid_reduce<1>(in, partials, ticket, out) && threadIdx.x == 0) {
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

// d += a p; unless stopping, p = z + b p.
__global__ void __launch_bounds__(kThreads)
    k_inner_direction_z(int N, float *__restrict__ d, float *__restrict__ p,
                        const float *__restrict__ z, CgState *st) {
  if (st->in_finished) return;
  const float a = (float)st->in_alpha, b = (float)st->in_beta;
  const bool upd = !st->in_stop;
  const int n4 = N >> 2;
  float4 *d4 = reinterpret_cast<float4 *>(d);
  float4 *p4 = reinterpret_cast<float4 *>(p);
  const float4 *z4 = reinterpret_cast<const float4 *>(z);
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n4;
       i += gridDim.x * kThreads) {
    const float4 pv = p4[i];
    float4 dv = d4[i];
    dv.x = fmaf(a, pv.x, dv.x);
    dv.y = fmaf(a, pv.y, dv.y);
    dv.z = fmaf(a, pv.z, dv.z);
    dv.w = fmaf(a, pv.w, dv.w);
    d4[i] = dv;
    if (upd) {
      const float4 zv = __ldg(&z4[i]);
      p4[i] = make_float4(fmaf(b, pv.x, zv.x), fmaf(b, pv.y, zv.y),
                          fmaf(b, pv.z, zv.z), fmaf(b, pv.w, zv.w));
    }
  }
  for (int i = 4 * n4 + blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads) {
    const float pv = p[i];
    d[i] = fmaf(a, pv, d[i]);
    if (upd) p[i] = fmaf(b, pv, __ldg(&z[i]));
  }
}

// x += ||r64|| d (FP64).
__global__ void __launch_bounds__(kThreads)
    k_outer_update(int N, double *__restrict__ x, const float *__restrict__ d,
                   const CgState *st) {
  const double s = sqrt(st->r2);
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads)
    x[i] = fma(s, (double)d[i], x[i]);
}

// The same after a fused band inner solve, whose last update of d is still
// pending: x += ||r64|| (d + a p), with p the buffer of the pair that the
// last iteration wrote and d + a p rounded as the unfused update rounds it.
__global__ void __launch_bounds__(kThreads)
    k_outer_update_pending(int N, double *__restrict__ x,
                           const float *__restrict__ d,
                           const float *__restrict__ p0,
                           const float *__restrict__ p1, const CgState *st) {
  const double s = sqrt(st->r2);
  const float a = (float)st->in_alpha;
  const float *__restrict__ p = st->in_pslot ? p1 : p0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N;
       i += gridDim.x * kThreads)
    x[i] = fma(s, (double)fmaf(a, p[i], d[i]), x[i]);
}

}  // namespace cgx
