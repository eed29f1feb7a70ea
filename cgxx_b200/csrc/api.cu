// libcgb200: C ABI (include/cgx.h) over the sm_100a kernels in kernels.cuh.
//
// One handle owns one matrix and the six solver vectors of the reference
// (CG::Vector, CG.h:22-35) in device memory, a CUDA stream, the solver state
// (CgState) and cached CUDA graphs of the solve loop. The device solve keeps
// every scalar on the device: the iteration is three fused kernels
//   1. q = A p      + partials of <p,q>; last CTA: a = rho / <p,q>
//   2. r -= a q     + partials of <r,r>, <r,Cr>; last CTA: residual test,
//                     rho, b, stop flag, value of the graph's while condition
//   3. x += a p; p = C r + b p
// captured once into a graph whose while node repeats them until step 2
// clears the condition.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <map>
#include <unordered_map>
#include <vector>

#include "cgx.h"
#include "band.cuh"
#include "ingest.cuh"
#include "kernels.cuh"
#include "learned.cuh"
#include "persist.cuh"
#include "sell.cuh"

using namespace cgx;

// ---------------------------------------------------------------------------
// Errors

static thread_local std::string g_err;

static cgx_status fail(cgx_status s, const std::string &msg) {
  g_err = msg;
  return s;
}

void cgx_internal_set_error(const std::string &msg) { g_err = msg; }

static cgx_status cuda_fail(cudaError_t e, const char *what) {
  cgx_status s = (e == cudaErrorMemoryAllocation) ? CGX_ERROR_OUT_OF_MEMORY
                                                  : CGX_ERROR_CUDA;
  return fail(s, std::string("CUDA error: ") + cudaGetErrorString(e) + " (" +
                     what + ")");
}

#define CUDA_TRY(call)                                  \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

#define CGX_TRY(call)                    \
  do {                                   \
    cgx_status s_ = (call);              \
    if (s_ != CGX_SUCCESS) return s_;    \
  } while (0)

// Makes the handle's device current for the scope and restores the caller's.
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// ---------------------------------------------------------------------------
// Handle

namespace {

enum : int {
  kTicketSetup = 0,
  kTicketQ = 1,
  kTicketUpdate = 2,
  kTicketDot = 3,
  kTicketTrue = 4,
  kTicketInnerStart = 5,
  kTicketInnerQ = 6,
  kTicketInnerUpdate = 7,
};

struct GraphEntry {
  int key = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long cond = 0;
};

constexpr int kChunk = 16;  // iterations per launch of the chunked loop

size_t round_up(size_t b, size_t a) { return (b + a - 1) / a * a; }

// Bump allocator over one device allocation; every piece 256-byte aligned.
struct Carver {
  size_t off = 0;
  template <typename T>
  size_t take(size_t count) {
    size_t o = off;
    off = round_up(off + count * sizeof(T), 256);
    return o;
  }
};

}  // namespace

// SELL-U layout of a CRS pattern (sell.cuh): slice meta, offsets and the
// value slot of every CRS entry (map); `slots` values including padding.
struct SellU {
  void *mem = nullptr;
  int4 *meta = nullptr;
  int *off = nullptr;
  int *map = nullptr;
  size_t slots = 0;
  long long uniform = 0;  // slices with uniform offsets
  int max_width = 0;      // largest slot count of a slice
  bool ok = false;
};

struct cgx_handle;
static cudaError_t dev_alloc(cgx_handle *h, void **p, size_t bytes);
static void dev_free(cgx_handle *h, void *p);

static void sellu_free(cgx_handle *h, SellU &S) {
  if (S.mem) dev_free(h, S.mem);
  S = SellU{};
}

// Symmetric band copy of A's FP32 values (band.cuh). K > 0: the offsets of
// A fit the layout (planned once per pattern); ok: the values of the last
// refresh passed the symmetry check and U holds them.
struct Band {
  float *U = nullptr;  // N x kBandMaxK, row-major
  int K = 0;
  int d[kBandMaxK] = {};
  bool ok = false;
};

static void band_free(cgx_handle *h, Band &B) {
  if (B.U) dev_free(h, B.U);
  B = Band{};
}

// Releases U after a refresh whose values failed the symmetry check, keeping
// the planned offsets: a later refresh with symmetric values fills U again.
static void band_drop_values(cgx_handle *h, Band &B) {
  if (B.U) dev_free(h, B.U);
  B.U = nullptr;
  B.ok = false;
}

struct cgx_handle {
  int device = 0;
  // Device blocks of replaced matrices, kept for the next upload
  // (dev_alloc / dev_free): size -> block, and the size of every block the
  // handle owns.
  std::multimap<size_t, void *> spare;
  std::unordered_map<void *, size_t> block_size;
  int num_sms = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;

  // Matrix.
  int format = -1;
  int N = 0;
  int nz = 0;
  void *mat_mem = nullptr;
  int *ptr = nullptr, *index = nullptr;  // CRS, and COO grouped by row
  double *value = nullptr;
  int tile_cap = 0;
  int warp_cap = 0;  // k_crs_warp's tile capacity when 256-row tiles overflow
  int *ell_length = nullptr, *ell_index = nullptr;  // ELL
  void *rows_mem = nullptr;  // ELL: the row layout (ptr, index, value), built on first use
  double *ell_data = nullptr;
  int ell_width = 0;

  // Vectors K X P Q R Z and Jacobi C.
  void *vec_mem = nullptr;
  double *vec[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  double *C = nullptr;
  double *tmp = nullptr;  // FP64 scratch vector (true residual)
  bool c_valid = false;

  // FP32 mirror and inner vectors of the mixed path (allocated on demand).
  void *f32_mem = nullptr;
  float *value32 = nullptr, *C32 = nullptr;
  // Column indices as 16-bit offsets from the row, when they all fit
  // (compact16): the mixed and learned paths read 6 instead of 8 bytes per
  // FP32 entry.
  int16_t *idx16 = nullptr;
  bool compact16 = false;
  float *d32 = nullptr, *r32 = nullptr, *p32 = nullptr, *q32 = nullptr;
  // Second buffers of the ping-pong pairs (p, r) and z of the persistent
  // inner solves (persist.cuh).
  float *p32b = nullptr, *r32b = nullptr, *z32 = nullptr;
  // Partial sums and the barrier counter of the persistent inner solves.
  double *persist_part = nullptr;
  unsigned long long *persist_sync = nullptr;
  double *r64 = nullptr;
  bool f32_valid = false;
  // What the captured inner-solve graphs took from the FP32 copy (its
  // buffers, index form and band / SELL-U layout) when they were built.
  std::array<uintptr_t, 10> f32_key{};
  // SELL-U copy of A's FP32 values for the inner SpMV (built with the FP32
  // mirror; sa.ok when the layout's indices fit in int).
  SellU sa;
  float *sa_val = nullptr;
  bool sa_tried = false;
  // Symmetric band copy, preferred over SELL-U when A fits it.
  Band band;
  bool band_tried = false;

  // Scratch: state, partial sums, dot result, validation flag.
  void *scratch = nullptr;
  CgState *st = nullptr;
  double *partials = nullptr;
  double *dot_out = nullptr;
  int *flag = nullptr;
  CgState *host_st = nullptr;  // pinned mirror
  double *host_scalar = nullptr;  // pinned

  std::vector<GraphEntry> graphs;
  cudaEvent_t ev[8] = {};
  // Per-kernel timing mode: 4 events for each of kChunk iterations that are
  // enqueued before the host waits (created on first use).
  std::vector<cudaEvent_t> evpool;

  // Learned preconditioner (cgx_learned_setup / cgx_learned_factor).
  struct Learned *L = nullptr;
};

// Device buffers of the learned preconditioner for one matrix.
struct Learned {
  int N = 0, nnz = 0, nnzL = 0, nblocks = 0;
  void *mem = nullptr;    // graph, factor, activations, inner vectors
  void *train = nullptr;  // training buffers (allocated on first use)
  double *dis = nullptr;
  float *ahat = nullptr, *feat = nullptr;
  int *nlow = nullptr, *nup = nullptr, *sums = nullptr, *flag = nullptr;
  int *gptr = nullptr, *gcol = nullptr, *grow = nullptr, *g2a = nullptr;
  int *tptr = nullptr, *tcol = nullptr, *t2g = nullptr, *g2t = nullptr;
  float *ghat = nullptr, *gs = nullptr, *gts = nullptr;
  // SELL-U copies of G and G^T for the apply (BF16 values), used when both
  // layouts were built (sell_ok); their maps take the values from k_assemble.
  SellU sg, st;
  void *sell_val = nullptr;
  __nv_bfloat16 *sg_val = nullptr, *st_val = nullptr;
  bool sell_ok = false;
  // Band copy of G (band.cuh) when A's offsets fit the band: preferred over
  // the SELL-U copies, which are then not built.
  void *gb_mem = nullptr;
  __nv_bfloat16 *gb_val = nullptr;
  int *g2b = nullptr;
  int gb_d[kBandMaxK] = {};
  bool gb_ok = false;
  __nv_bfloat16 *h[4] = {};
  __nv_bfloat16 *agg[3] = {};
  float *pre[4] = {};
  float *o = nullptr;
  float *y32 = nullptr, *z32 = nullptr;
  // training
  float *V = nullptr, *T1 = nullptr, *T2 = nullptr, *rho = nullptr;
  float *dT2 = nullptr, *dT1 = nullptr, *dg = nullptr, *dO = nullptr;
  float *dh = nullptr, *dh2 = nullptr, *dself = nullptr, *dagg = nullptr,
        *dpre = nullptr;
  float *partial = nullptr, *grad = nullptr, *loss = nullptr;
  float *gtmp = nullptr;  // two reduced [W*W | W] blocks of a layer gradient
  float *snap = nullptr;  // residual snapshots (probe columns), N x S
  double *snap_scale = nullptr;
  unsigned snap_valid = 0;  // bit c: column c holds a snapshot of this matrix
  bool has_factor = false;
  float eps = 0.f;
};

struct cgx_gnn {
  int device = 0;
  float *params = nullptr, *m = nullptr, *v = nullptr;
  int step = 0;
  // Probe recipe (cgx_gnn_set_probes).
  int smooth_steps = 0, smooth_cols = 0, residual_cols = 0;
  float smooth_scale = 1.f;
};

// Device memory of a handle. A block released by dev_free stays with the
// handle, and dev_alloc hands it out again for a request it fits (at most a
// quarter plus 1 MiB larger): re-uploading a matrix of the same size, as a
// time-stepping caller does every step, then allocates nothing, where
// cudaMalloc and cudaFree of the same gigabytes took 8 to 180 ms per upload.
// All of a handle's work is ordered on its stream (cgx_set_stream first
// drains the old one), so a block is never reused while a kernel still
// reads it. On an allocation failure the spare blocks are released and the
// allocation is retried; cgx_destroy releases everything.
static void release_spare(cgx_handle *h) {
  for (auto &kv : h->spare) {
    h->block_size.erase(kv.second);
    cudaFree(kv.second);
  }
  h->spare.clear();
}

static cudaError_t dev_alloc(cgx_handle *h, void **p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 1;
  auto it = h->spare.lower_bound(bytes);
  if (it != h->spare.end() && it->first <= bytes + bytes / 4 + (1u << 20)) {
    *p = it->second;
    h->spare.erase(it);
    return cudaSuccess;
  }
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation && !h->spare.empty()) {
    cudaGetLastError();
    release_spare(h);
    e = cudaMalloc(p, bytes);
  }
  if (e != cudaSuccess) {
    *p = nullptr;
    return e;
  }
  h->block_size[*p] = bytes;
  return cudaSuccess;
}

static void dev_free(cgx_handle *h, void *p) {
  if (!p) return;
  auto it = h->block_size.find(p);
  if (it == h->block_size.end()) return;
  h->spare.emplace(it->second, p);
}

static void drop_graphs(cgx_handle *h) {
  for (auto &g : h->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
  }
  h->graphs.clear();
}

static void free_learned(cgx_handle *h) {
  if (!h->L) return;
  if (h->L->mem) dev_free(h, h->L->mem);
  if (h->L->train) dev_free(h, h->L->train);
  sellu_free(h, h->L->sg);
  sellu_free(h, h->L->st);
  if (h->L->sell_val) dev_free(h, h->L->sell_val);
  if (h->L->gb_mem) dev_free(h, h->L->gb_mem);
  delete h->L;
  h->L = nullptr;
}

static void free_matrix(cgx_handle *h) {
  drop_graphs(h);
  free_learned(h);
  if (h->mat_mem) dev_free(h, h->mat_mem);
  if (h->rows_mem) dev_free(h, h->rows_mem);
  h->rows_mem = nullptr;
  if (h->vec_mem) dev_free(h, h->vec_mem);
  if (h->f32_mem) dev_free(h, h->f32_mem);
  h->mat_mem = h->vec_mem = h->f32_mem = nullptr;
  sellu_free(h, h->sa);
  if (h->sa_val) dev_free(h, h->sa_val);
  h->sa_val = nullptr;
  h->sa_tried = false;
  band_free(h, h->band);
  h->band_tried = false;
  h->format = -1;
  h->N = h->nz = 0;
  h->ptr = h->index = nullptr;
  h->value = nullptr;
  h->ell_length = h->ell_index = nullptr;
  h->ell_data = nullptr;
  for (auto &v : h->vec) v = nullptr;
  h->C = nullptr;
  h->tmp = nullptr;
  h->c_valid = false;
  h->value32 = h->C32 = h->d32 = h->r32 = h->p32 = h->q32 = nullptr;
  h->p32b = h->r32b = h->z32 = nullptr;
  h->persist_part = nullptr;
  h->persist_sync = nullptr;
  h->r64 = nullptr;
  h->idx16 = nullptr;
  h->compact16 = false;
  h->f32_valid = false;
}

// Grid of the streaming (vector) kernels: a few CTAs per SM, enough bytes in
// flight to saturate HBM, never more CTAs than there is work.
static int grid_stream(const cgx_handle *h, size_t work_items) {
  size_t need = (work_items + kThreads - 1) / kThreads;
  size_t g = std::min<size_t>((size_t)h->num_sms * 8, need);
  g = std::min<size_t>(g, kMaxGrid);
  return (int)std::max<size_t>(g, 1);
}

// ---------------------------------------------------------------------------
// Validation kernels for uploaded matrices (invalid data is an error, not
// undefined behaviour as in the reference).

__global__ void k_validate_crs(int N, int nz, const int *ptr, const int *index,
                               int *flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x)
    if (ptr[i] > ptr[i + 1]) atomicOr(flag, 1);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nz;
       j += gridDim.x * blockDim.x) {
    int c = index[j];
    if (c < 0 || c >= N) atomicOr(flag, 2);
  }
}

// Column-major (element (i, j) at j * N + i) to the tile-major device layout.
__global__ void k_ell_tiles(int N, int width, const int *__restrict__ ci,
                            const double *__restrict__ cd, int *__restrict__ ti,
                            double *__restrict__ td) {
  const size_t total = (size_t)N * (size_t)width;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / (size_t)N), i = (int)(e - (size_t)j * N);
    const size_t o = ell_at(i, j, width);
    ti[o] = ci[e];
    td[o] = cd[e];
  }
}

// Tile-major ELL to the row layout: row i's slots j < length[i] in order.
__global__ void k_ell_to_rows(int N, int width, const int *__restrict__ length,
                              const int *__restrict__ eidx,
                              const double *__restrict__ edat,
                              const int *__restrict__ ptr, int *__restrict__ index,
                              double *__restrict__ value) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x) {
    const int len = length[i], o = ptr[i];
    for (int j = 0; j < len; j++) {
      index[o + j] = eidx[ell_at(i, j, width)];
      value[o + j] = edat[ell_at(i, j, width)];
    }
  }
}

__global__ void k_validate_ell(int N, int width, const int *length,
                               const int *index, int *flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += gridDim.x * blockDim.x) {
    int len = length[i];
    if (len < 0 || len > width) {
      atomicOr(flag, 1);
      continue;
    }
    for (int j = 0; j < len; j++) {
      int c = index[ell_at(i, j, width)];
      if (c < 0 || c >= N) atomicOr(flag, 2);
    }
  }
}

// Runaway guard of a graph while loop: whatever happens to the reductions,
// the condition is cleared after max_iter + 2 bodies.
__global__ void k_loop_guard(CgState *st) {
  if (++st->body_count > st->max_iter + 1) {
    st->error |= 2;
    st->stop = 1;
    st->in_stop = 1;
    if (st->use_cond)
      cudaGraphSetConditional((cudaGraphConditionalHandle)st->cond, 0u);
  }
}

// ---------------------------------------------------------------------------
// Launch helpers

// Staged CRS SpMV over any CRS view (A itself, or the learned factor's G and
// G^T, whose rows are subsets of A's rows so A's tile capacity bounds them).
template <typename VT, typename IT, typename Op>
static cudaError_t launch_crs_view(cgx_handle *h, CrsView<VT, IT> A,
                                   const typename Comp<VT>::T *x, Op op) {
  if (A.warp_cap > 0) {
    const size_t smem = 16 * kWarps + kWarps * crs_stage_bytes<VT, IT>(A.warp_cap);
    auto kern = k_crs_warp<VT, IT, Op>;
    cudaError_t e;
    if (smem > 48 * 1024 &&
        (e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem)) != cudaSuccess)
      return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
    if (e != cudaSuccess) return e;
    const int wtiles = (h->N + 31) / 32;
    const int grid = std::max(1, std::min(std::min(h->num_sms * std::max(1, per_sm), kMaxGrid),
                                          (wtiles + kWarps - 1) / kWarps));
    kern<<<grid, kThreads, smem, h->stream>>>(A, x, op, h->st, h->partials);
    return cudaGetLastError();
  }
  const int cap = A.tile_cap;
  const size_t smem = crs_smem_bytes<VT, IT>(cap);
  auto kern = k_crs<VT, IT, Op>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, kern, kThreads, smem);
  if (e != cudaSuccess) return e;
  per_sm = std::max(1, per_sm);
  const int tiles = (h->N + kThreads - 1) / kThreads;
  int grid = std::min(std::min(h->num_sms * per_sm, kMaxGrid), tiles);
  grid = std::max(grid, 1);
  kern<<<grid, kThreads, smem, h->stream>>>(A, x, op, h->st, h->partials);
  return cudaGetLastError();
}

template <typename VT, typename Op>
static cudaError_t launch_crs(cgx_handle *h, const VT *value, int cap,
                              const VT *x, Op op) {
  return launch_crs_view<VT, int, Op>(
      h, CrsView<VT, int>{h->ptr, h->index, value, h->N, cap, h->warp_cap}, x, op);
}

template <typename Op>
static cudaError_t launch_spmv(cgx_handle *h, const double *x, Op op) {
  switch (h->format) {
  case CGX_FORMAT_CRS:
  case CGX_FORMAT_COO:  // held in the row-grouped layout (cgx_upload_coo)
    return launch_crs<double, Op>(h, h->value, h->tile_cap, x, op);
  case CGX_FORMAT_ELL: {
    EllView<double> A{h->ell_length, h->ell_index, h->ell_data, h->N,
                      h->ell_width};
    if (h->ell_width >= 1 && h->ell_width <= kEllStagedWidth) {
      const size_t smem = ell_smem_bytes<double>(h->ell_width);
      auto kern = k_ell_tma<double, Op>;
      cudaError_t e;
      if (smem > 48 * 1024 &&
          (e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem)) != cudaSuccess)
        return e;
      int per_sm = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
      if (e != cudaSuccess) return e;
      const int tiles = (h->N + kThreads - 1) / kThreads;
      const int grid = std::max(1, std::min(std::min(h->num_sms * std::max(1, per_sm),
                                                     kMaxGrid), tiles));
      kern<<<grid, kThreads, smem, h->stream>>>(A, x, op, h->st, h->partials);
    } else {
      k_ell<double, Op><<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(
          A, x, op, h->st, h->partials);
    }
    return cudaGetLastError();
  }
  }
  return cudaErrorInvalidValue;
}

static unsigned *ticket(cgx_handle *h, int which) {
  return &h->st->counter[which];
}

// One PCG iteration's three kernels (FP64).
static cudaError_t launch_pcg_iteration(cgx_handle *h, bool jacobi,
                                        cudaEvent_t *evs = nullptr) {
  double *x = h->vec[CGX_VECTOR_X], *p = h->vec[CGX_VECTOR_P];
  double *q = h->vec[CGX_VECTOR_Q], *r = h->vec[CGX_VECTOR_R];
  cudaError_t e;
  if (evs) cudaEventRecord(evs[0], h->stream);
  e = launch_spmv(h, p, OpPcgQ{p, q, ticket(h, kTicketQ)});
  if (e != cudaSuccess) return e;
  if (evs) cudaEventRecord(evs[1], h->stream);
  const int g = grid_stream(h, (size_t)(h->N + 1) / 2);
  if (jacobi)
    k_pcg_update<true><<<g, kThreads, 0, h->stream>>>(
        h->N, r, q, h->C, h->st, h->partials, ticket(h, kTicketUpdate));
  else
    k_pcg_update<false><<<g, kThreads, 0, h->stream>>>(
        h->N, r, q, h->C, h->st, h->partials, ticket(h, kTicketUpdate));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (evs) cudaEventRecord(evs[2], h->stream);
  if (jacobi)
    k_pcg_direction<true><<<g, kThreads, 0, h->stream>>>(h->N, x, p, r, h->C,
                                                          h->st);
  else
    k_pcg_direction<false><<<g, kThreads, 0, h->stream>>>(h->N, x, p, r, h->C,
                                                           h->st);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (evs) cudaEventRecord(evs[3], h->stream);
  return cudaSuccess;
}

static cudaError_t launch_pcg_setup(cgx_handle *h, bool jacobi) {
  double *k = h->vec[CGX_VECTOR_K], *x = h->vec[CGX_VECTOR_X];
  double *p = h->vec[CGX_VECTOR_P], *r = h->vec[CGX_VECTOR_R];
  if (jacobi)
    return launch_spmv(h, x,
                       OpSetup<true>{k, r, p, h->C, ticket(h, kTicketSetup)});
  return launch_spmv(h, x,
                     OpSetup<false>{k, r, p, h->C, ticket(h, kTicketSetup)});
}

// q = A p in FP32 with <p,q> (inner solves), compact indices when they fit.
// k_sellu over one wave of CTAs (as many as fit on the SMs at once), fewer
// when the warp steps run out; chunks of 4 slots when no slice is wider,
// and the uniform-only kernel when every slice is uniform.
template <typename VT, int U, bool ALL_UNIFORM, typename Op>
static cudaError_t launch_sellu_u(cgx_handle *h, SellUView<VT> A, const float *x,
                                  Op op) {
  auto kern = k_sellu<VT, U, ALL_UNIFORM, Op>;
  int per_sm = 0;
  cudaError_t e =
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, 0);
  if (e != cudaSuccess) return e;
  // Warp steps: slice pairs on a uniform layout, single slices otherwise.
  const int slices = (h->N + 31) / 32;
  const int steps = ALL_UNIFORM ? (slices + 1) / 2 : slices;
  const int grid = std::max(1, std::min(h->num_sms * std::max(1, per_sm),
                                        (steps + kWarps - 1) / kWarps));
  kern<<<grid, kThreads, 0, h->stream>>>(A, x, op, h->st, h->partials);
  return cudaGetLastError();
}

template <typename VT, typename Op>
static cudaError_t launch_sellu(cgx_handle *h, const SellU &S, const VT *val,
                                const float *x, Op op) {
  const SellUView<VT> A{S.meta, S.off, val, h->N};
  const bool all = S.uniform == (long long)((h->N + 31) / 32);
  if (S.max_width <= 4)
    return all ? launch_sellu_u<VT, 4, true>(h, A, x, op)
               : launch_sellu_u<VT, 4, false>(h, A, x, op);
  return all ? launch_sellu_u<VT, 8, true>(h, A, x, op)
             : launch_sellu_u<VT, 8, false>(h, A, x, op);
}

// Persistent kernel over `rows` rows: as many CTAs as fit on the SMs at
// once, fewer when the 256-row tiles run out.
template <typename Kern, typename... Args>
static cudaError_t launch_rows(cgx_handle *h, Kern kern, size_t rows, Args... args) {
  int per_sm = 0;
  cudaError_t e =
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, 0);
  if (e != cudaSuccess) return e;
  const size_t tiles = (rows + kThreads - 1) / kThreads;
  const int grid = (int)std::max<size_t>(
      1, std::min<size_t>(std::min(h->num_sms * std::max(1, per_sm), kMaxGrid), tiles));
  kern<<<grid, kThreads, 0, h->stream>>>(args...);
  return cudaGetLastError();
}

static BandView<4> band_view(const cgx_handle *h) {
  BandView<4> B;
  B.U = h->band.U;
  B.N = h->N;
  for (int k = 0; k < 4; k++) B.d[k] = k < h->band.K ? h->band.d[k] : 0;
  return B;
}

template <typename Op>
static cudaError_t launch_band(cgx_handle *h, const float *x, Op op) {
  return launch_rows(h, k_band<4, Op>, h->N, band_view(h), x, op, h->st, h->partials);
}

static cudaError_t launch_inner_q(cgx_handle *h) {
  OpInnerQ op{h->p32, h->q32, ticket(h, kTicketInnerQ)};
  if (h->band.ok) return launch_band(h, h->p32, op);
  if (h->sa.ok)
    return launch_sellu(h, h->sa, h->sa_val, h->p32, op);
  if (h->compact16)
    return launch_crs_view(
        h, CrsView<float, int16_t>{h->ptr, h->idx16, h->value32, h->N, h->tile_cap,
                                   h->warp_cap},
        h->p32, op);
  return launch_crs_view(
      h, CrsView<float, int>{h->ptr, h->index, h->value32, h->N, h->tile_cap,
                             h->warp_cap},
      h->p32, op);
}

// Inner FP32 PCG iteration of the mixed path: three kernels, whose
// kernel-mode segments are (q = A p | r update | p update).
static cudaError_t launch_inner_iteration(cgx_handle *h, cudaEvent_t *evs = nullptr) {
  cudaError_t e;
  const int g = grid_stream(h, (size_t)(h->N + 3) / 4);
  if (evs) cudaEventRecord(evs[0], h->stream);
  e = launch_inner_q(h);
  if (e != cudaSuccess) return e;
  if (evs) cudaEventRecord(evs[1], h->stream);
  k_inner_update<<<g, kThreads, 0, h->stream>>>(
      h->N, h->r32, h->q32, h->C32, h->st, h->partials,
      ticket(h, kTicketInnerUpdate));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (evs) cudaEventRecord(evs[2], h->stream);
  k_inner_direction<<<g, kThreads, 0, h->stream>>>(h->N, h->d32, h->p32,
                                                   h->r32, h->C32, h->st);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (evs) cudaEventRecord(evs[3], h->stream);
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// Graph construction: `prologue` is captured into the top-level graph, then
// a while node whose body is `body`, then `epilogue` after it.

template <typename Pro, typename Body, typename Epi>
static cgx_status build_while_graph(cgx_handle *h, int key, Pro prologue,
                                    Body body, Epi epilogue, GraphEntry **out) {
  for (auto &g : h->graphs)
    if (g.key == key) {
      *out = &g;
      return CGX_SUCCESS;
    }
  GraphEntry ge;
  ge.key = key;
  CUDA_TRY(cudaGraphCreate(&ge.graph, 0));
  cudaGraphConditionalHandle cond;
  CUDA_TRY(cudaGraphConditionalHandleCreate(&cond, ge.graph, 1,
                                            cudaGraphCondAssignDefault));
  ge.cond = (unsigned long long)cond;

  // Prologue.
  CUDA_TRY(cudaStreamBeginCaptureToGraph(h->stream, ge.graph, nullptr, nullptr,
                                         0, cudaStreamCaptureModeThreadLocal));
  cudaError_t le = prologue();
  cudaGraph_t captured = nullptr;
  cudaError_t ce = cudaStreamEndCapture(h->stream, &captured);
  if (le != cudaSuccess) return cuda_fail(le, "graph prologue");
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
  size_t n = 0;
  CUDA_TRY(cudaGraphGetNodes(ge.graph, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  CUDA_TRY(cudaGraphGetNodes(ge.graph, nodes.data(), &n));
  // The prologue is a chain; its leaf is the node without dependents.
  cudaGraphNode_t leaf = nullptr;
  for (auto nd : nodes) {
    size_t nd_out = 0;
    CUDA_TRY(cudaGraphNodeGetDependentNodes(nd, nullptr, &nd_out));
    if (nd_out == 0) leaf = nd;
  }

  // The struct's union has no default constructor in C++: zeroed storage.
  alignas(cudaGraphNodeParams) unsigned char cpbuf[sizeof(cudaGraphNodeParams)];
  std::memset(cpbuf, 0, sizeof(cpbuf));
  cudaGraphNodeParams &cp = *reinterpret_cast<cudaGraphNodeParams *>(cpbuf);
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  CUDA_TRY(cudaGraphAddNode(&cnode, ge.graph, leaf ? &leaf : nullptr,
                            leaf ? 1 : 0, &cp));
  cudaGraph_t bodyGraph = cp.conditional.phGraph_out[0];

  CUDA_TRY(cudaStreamBeginCaptureToGraph(h->stream, bodyGraph, nullptr,
                                         nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal));
  le = body();
  ce = cudaStreamEndCapture(h->stream, &captured);
  if (le != cudaSuccess) return cuda_fail(le, "graph body");
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");

  CUDA_TRY(cudaStreamBeginCaptureToGraph(h->stream, ge.graph, &cnode, nullptr,
                                         1, cudaStreamCaptureModeThreadLocal));
  le = epilogue();
  ce = cudaStreamEndCapture(h->stream, &captured);
  if (le != cudaSuccess) return cuda_fail(le, "graph epilogue");
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");

  CUDA_TRY(cudaGraphInstantiate(&ge.exec, ge.graph, 0));
  h->graphs.push_back(ge);
  *out = &h->graphs.back();
  return CGX_SUCCESS;
}

// Graph of a fixed number of iterations for the chunked loop.
template <typename Body>
static cgx_status build_chunk_graph(cgx_handle *h, int key, Body body,
                                    GraphEntry **out) {
  for (auto &g : h->graphs)
    if (g.key == key) {
      *out = &g;
      return CGX_SUCCESS;
    }
  GraphEntry ge;
  ge.key = key;
  CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t le = cudaSuccess;
  for (int i = 0; i < kChunk && le == cudaSuccess; i++) le = body();
  cudaError_t ce = cudaStreamEndCapture(h->stream, &ge.graph);
  if (le != cudaSuccess) return cuda_fail(le, "chunk body");
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
  CUDA_TRY(cudaGraphInstantiate(&ge.exec, ge.graph, 0));
  h->graphs.push_back(ge);
  *out = &h->graphs.back();
  return CGX_SUCCESS;
}

// ---------------------------------------------------------------------------
// State transfer

static cgx_status push_state(cgx_handle *h) {
  CUDA_TRY(cudaMemcpyAsync(h->st, h->host_st, sizeof(CgState),
                           cudaMemcpyHostToDevice, h->stream));
  return CGX_SUCCESS;
}

static cgx_status pull_state(cgx_handle *h) {
  CUDA_TRY(cudaMemcpyAsync(h->host_st, h->st, sizeof(CgState),
                           cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CGX_SUCCESS;
}

static void reset_host_state(cgx_handle *h, int max_iter, double tol,
                             bool use_cond, unsigned long long cond) {
  CgState &s = *h->host_st;
  std::memset(&s, 0, sizeof(s));
  s.max_iter = max_iter;
  s.tol = tol;
  s.use_cond = use_cond ? 1 : 0;
  s.cond = cond;
}

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

void cgx_version(int *major, int *minor) {
  if (major) *major = CGX_VERSION_MAJOR;
  if (minor) *minor = CGX_VERSION_MINOR;
}

const char *cgx_status_string(cgx_status s) {
  switch (s) {
  case CGX_SUCCESS: return "success";
  case CGX_ERROR_INVALID_ARGUMENT: return "invalid argument";
  case CGX_ERROR_INVALID_STATE: return "invalid state";
  case CGX_ERROR_UNSUPPORTED: return "unsupported";
  case CGX_ERROR_CUDA: return "CUDA error";
  case CGX_ERROR_OUT_OF_MEMORY: return "out of device memory";
  case CGX_ERROR_DEVICE: return "device-side check failed";
  case CGX_ERROR_IO: return "I/O error";
  case CGX_ERROR_NUMERICAL: return "numerical breakdown";
  }
  return "unknown status";
}

const char *cgx_last_error(void) { return g_err.c_str(); }

cgx_status cgx_device_count(int *count) {
  if (!count) return fail(CGX_ERROR_INVALID_ARGUMENT, "count is NULL");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  *count = n;
  return CGX_SUCCESS;
}

cgx_status cgx_default_options(cgx_options *o) {
  if (!o) return fail(CGX_ERROR_INVALID_ARGUMENT, "options is NULL");
  std::memset(o, 0, sizeof(*o));
  o->max_iterations = 1000;
  o->tolerance = 1e-9;
  o->preconditioner = CGX_PRECONDITIONER_JACOBI;
  o->precision = CGX_PRECISION_FP64;
  o->loop = CGX_LOOP_GRAPH;
  o->inner_tolerance = 3e-6;
  o->max_outer = 30;
  o->compute_true_residual = 0;
  return CGX_SUCCESS;
}

cgx_status cgx_create(cgx_handle **out, int device) {
  if (!out) return fail(CGX_ERROR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  int n = 0;
  cgx_device_count(&n);
  if (device < 0 || device >= n)
    return fail(CGX_ERROR_INVALID_ARGUMENT,
                "no CUDA device " + std::to_string(device) + " (found " +
                    std::to_string(n) + ")");
  DeviceGuard guard(device);
  if (!guard.ok) return fail(CGX_ERROR_CUDA, "cudaSetDevice failed");
  cgx_handle *h = new cgx_handle();
  h->device = device;
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    delete h;
    return cuda_fail(e, "cudaGetDeviceProperties");
  }
  h->num_sms = prop.multiProcessorCount;
  if (prop.major < 10) {
    delete h;
    return fail(CGX_ERROR_UNSUPPORTED,
                std::string("libcgb200 is built for sm_100a; device is ") +
                    prop.name);
  }
  Carver c;
  size_t o_st = c.take<CgState>(1);
  size_t o_part = c.take<double>(2 * (size_t)kMaxGrid);
  size_t o_dot = c.take<double>(4);
  size_t o_flag = c.take<int>(4);
  if ((e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking)) !=
          cudaSuccess ||
      (e = cudaMalloc(&h->scratch, c.off)) != cudaSuccess ||
      (e = cudaMallocHost((void **)&h->host_st, sizeof(CgState))) !=
          cudaSuccess ||
      (e = cudaMallocHost((void **)&h->host_scalar, 64)) != cudaSuccess) {
    cgx_destroy(h);
    return cuda_fail(e, "cgx_create allocation");
  }
  for (auto &ev : h->ev)
    if ((e = cudaEventCreate(&ev)) != cudaSuccess) {
      cgx_destroy(h);
      return cuda_fail(e, "cudaEventCreate");
    }
  h->stream = h->own_stream;
  char *base = (char *)h->scratch;
  h->st = (CgState *)(base + o_st);
  h->partials = (double *)(base + o_part);
  h->dot_out = (double *)(base + o_dot);
  h->flag = (int *)(base + o_flag);
  e = cudaMemsetAsync(h->scratch, 0, c.off, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    cgx_destroy(h);
    return cuda_fail(e, "scratch init");
  }
  *out = h;
  return CGX_SUCCESS;
}

cgx_status cgx_destroy(cgx_handle *h) {
  if (!h) return CGX_SUCCESS;
  DeviceGuard guard(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_matrix(h);
  release_spare(h);
  for (auto &ev : h->ev)
    if (ev) cudaEventDestroy(ev);
  for (auto &ev : h->evpool) cudaEventDestroy(ev);
  if (h->scratch) cudaFree(h->scratch);
  if (h->host_st) cudaFreeHost(h->host_st);
  if (h->host_scalar) cudaFreeHost(h->host_scalar);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return CGX_SUCCESS;
}

cgx_status cgx_set_stream(cgx_handle *h, void *stream) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  cudaStream_t s = stream ? (cudaStream_t)stream : h->own_stream;
  if (s != h->stream) {
    DeviceGuard guard(h->device);
    // Blocks the handle reuses were last used on the old stream.
    if (h->stream) CUDA_TRY(cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    h->stream = s;
  }
  return CGX_SUCCESS;
}

cgx_status cgx_synchronize(cgx_handle *h) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  DeviceGuard guard(h->device);
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CGX_SUCCESS;
}

cgx_status cgx_host_alloc(void **p, size_t bytes) {
  if (!p) return fail(CGX_ERROR_INVALID_ARGUMENT, "p is NULL");
  *p = nullptr;
  CUDA_TRY(cudaMallocHost(p, bytes > 0 ? bytes : 1));
  return CGX_SUCCESS;
}

cgx_status cgx_host_free(void *p) {
  if (p) CUDA_TRY(cudaFreeHost(p));
  return CGX_SUCCESS;
}

cgx_status cgx_inner_layout(cgx_handle *h, long long *value_slots,
                            long long *uniform_slices, long long *slices) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  const bool ok = h->sa.ok;
  if (value_slots) *value_slots = ok ? (long long)h->sa.slots : 0;
  if (uniform_slices) *uniform_slices = ok ? h->sa.uniform : 0;
  if (slices) *slices = ok ? (h->N + 31) / 32 : 0;
  return CGX_SUCCESS;
}

cgx_status cgx_inner_band(cgx_handle *h, int *stored_offsets, int *offsets) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  const int K = h->band.ok ? h->band.K : 0;
  if (stored_offsets) *stored_offsets = K;
  if (offsets)
    for (int k = 0; k < K; k++) offsets[k] = h->band.d[k];
  return CGX_SUCCESS;
}

cgx_status cgx_matrix_info(cgx_handle *h, int *N, int *nz, int *format) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  if (N) *N = h->N;
  if (nz) *nz = h->nz;
  if (format) *format = h->format;
  return CGX_SUCCESS;
}

}  // extern "C"

// Allocates the vector block (K X P Q R Z, C, scratch) for N rows and zeroes
// it.
static cgx_status alloc_vectors(cgx_handle *h, int N) {
  Carver c;
  size_t o[8];
  for (int i = 0; i < 8; i++) o[i] = c.take<double>((size_t)N + kPad);
  CUDA_TRY(dev_alloc(h, (void **)&h->vec_mem, c.off));
  char *base = (char *)h->vec_mem;
  for (int i = 0; i < 6; i++) h->vec[i] = (double *)(base + o[i]);
  h->C = (double *)(base + o[6]);
  h->tmp = (double *)(base + o[7]);
  CUDA_TRY(cudaMemsetAsync(h->vec_mem, 0, c.off, h->stream));
  return CGX_SUCCESS;
}

static cgx_status check_flag(cgx_handle *h, const char *what) {
  CUDA_TRY(cudaMemcpyAsync(h->host_scalar, h->flag, sizeof(int),
                           cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  int f = *(int *)h->host_scalar;
  if (f) {
    std::string m = std::string("invalid ") + what + " matrix:";
    if (f & 1) m += " row pointers/lengths out of order or range;";
    if (f & 2) m += " column index outside [0, N);";
    free_matrix(h);
    return fail(CGX_ERROR_INVALID_ARGUMENT, m);
  }
  return CGX_SUCCESS;
}

extern "C" {

// Tile capacity of the staged CRS SpMV: the largest nonzero count of a
// 256-row tile, bounded so that two stages fit next to each other with
// several CTAs per SM; larger tiles fall back to direct loads. Rows too long
// for those tiles: 32-row tiles staged per warp (k_crs_warp) when they hold
// at most 2048 nonzeros.
static void set_tile_caps(cgx_handle *h, const int *ptr, int N) {
  int maxTile = 0;
  for (int r0 = 0; r0 < N; r0 += kThreads)
    maxTile = std::max(maxTile, ptr[std::min(N, r0 + kThreads)] - ptr[r0]);
  h->tile_cap = std::min(maxTile, 4096);
  h->warp_cap = 0;
  if (maxTile > 4096) {
    int maxWarp = 0;
    for (int r0 = 0; r0 < N; r0 += 32)
      maxWarp = std::max(maxWarp, ptr[std::min(N, r0 + 32)] - ptr[r0]);
    if (maxWarp <= 2048) h->warp_cap = maxWarp;
  }
}

// Row-grouped device layout shared by CRS and COO: row pointers, column
// indices and values in storage order, validated on the device.
static cgx_status upload_rows(cgx_handle *h, int N, int nz, const int *ptr,
                              const int *index, const double *value,
                              int format, const char *what) {
  DeviceGuard guard(h->device);
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  free_matrix(h);
  set_tile_caps(h, ptr, N);

  Carver c;
  size_t o_ptr = c.take<int>((size_t)N + 1 + kPad);
  size_t o_idx = c.take<int>((size_t)nz + kPad);
  size_t o_val = c.take<double>((size_t)nz + kPad);
  CUDA_TRY(dev_alloc(h, (void **)&h->mat_mem, c.off));
  char *base = (char *)h->mat_mem;
  h->ptr = (int *)(base + o_ptr);
  h->index = (int *)(base + o_idx);
  h->value = (double *)(base + o_val);
  CUDA_TRY(cudaMemsetAsync(h->mat_mem, 0, c.off, h->stream));
  CUDA_TRY(cudaMemcpyAsync(h->ptr, ptr, sizeof(int) * ((size_t)N + 1),
                           cudaMemcpyHostToDevice, h->stream));
  if (nz > 0) {
    CUDA_TRY(cudaMemcpyAsync(h->index, index, sizeof(int) * (size_t)nz,
                             cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(h->value, value, sizeof(double) * (size_t)nz,
                             cudaMemcpyHostToDevice, h->stream));
  }
  h->N = N;
  h->nz = nz;
  h->format = format;
  CGX_TRY(alloc_vectors(h, N));
  CUDA_TRY(cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream));
  k_validate_crs<<<grid_stream(h, std::max(N, nz)), kThreads, 0, h->stream>>>(
      N, nz, h->ptr, h->index, h->flag);
  CUDA_TRY(cudaGetLastError());
  return check_flag(h, what);
}

cgx_status cgx_upload_crs(cgx_handle *h, int N, int nz, const int *ptr,
                          const int *index, const double *value) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  if (N <= 0 || nz < 0 || !ptr || (nz > 0 && (!index || !value)))
    return fail(CGX_ERROR_INVALID_ARGUMENT, "bad CRS sizes or pointers");
  if (ptr[0] != 0 || ptr[N] != nz)
    return fail(CGX_ERROR_INVALID_ARGUMENT,
                "CRS ptr must start at 0 and end at nz");
  return upload_rows(h, N, nz, ptr, index, value, CGX_FORMAT_CRS, "CRS");
}

cgx_status cgx_upload_ell(cgx_handle *h, int N, int nz, int maxNz,
                          const int *length, const int *index,
                          const double *data) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  if (N <= 0 || nz < 0 || maxNz < 0 || !length ||
      ((size_t)maxNz * N > 0 && (!index || !data)))
    return fail(CGX_ERROR_INVALID_ARGUMENT, "bad ELL sizes or pointers");
  // nz sizes the row-layout copies of the mixed and learned paths, so it must
  // be the number of entries the lengths describe (a well-formed ELL matrix
  // has it by construction).
  {
    long long sum = 0;
    for (int i = 0; i < N; i++)
      if (length[i] < 0 || length[i] > maxNz)
        return fail(CGX_ERROR_INVALID_ARGUMENT,
                    "invalid ELL matrix: row pointers/lengths out of order or range;");
      else
        sum += length[i];
    if (sum != nz)
      return fail(CGX_ERROR_INVALID_ARGUMENT,
                  "invalid ELL matrix: nz differs from the sum of the row lengths");
  }
  DeviceGuard guard(h->device);
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  free_matrix(h);
  // The caller's column-major arrays go through a temporary device copy into
  // the tile-major layout (ell_at).
  const size_t elems = ell_elems(N, maxNz);
  const size_t celems = (size_t)maxNz * (size_t)N;
  Carver c;
  size_t o_len = c.take<int>((size_t)N + kPad);
  size_t o_idx = c.take<int>(elems + kPad);
  size_t o_dat = c.take<double>(elems + kPad);
  CUDA_TRY(dev_alloc(h, (void **)&h->mat_mem, c.off));
  char *base = (char *)h->mat_mem;
  h->ell_length = (int *)(base + o_len);
  h->ell_index = (int *)(base + o_idx);
  h->ell_data = (double *)(base + o_dat);
  h->ell_width = maxNz;
  CUDA_TRY(cudaMemsetAsync(h->mat_mem, 0, c.off, h->stream));
  CUDA_TRY(cudaMemcpyAsync(h->ell_length, length, sizeof(int) * (size_t)N,
                           cudaMemcpyHostToDevice, h->stream));
  if (celems > 0) {
    void *tmp = nullptr;
    Carver t;
    const size_t o_ti = t.take<int>(celems), o_td = t.take<double>(celems);
    CUDA_TRY(dev_alloc(h, (void **)&tmp, t.off));
    int *ci = (int *)((char *)tmp + o_ti);
    double *cd = (double *)((char *)tmp + o_td);
    cudaError_t e = cudaMemcpyAsync(ci, index, sizeof(int) * celems,
                                    cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(cd, data, sizeof(double) * celems,
                          cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
      k_ell_tiles<<<grid_stream(h, celems), kThreads, 0, h->stream>>>(
          N, maxNz, ci, cd, h->ell_index, h->ell_data);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    dev_free(h, tmp);
    CUDA_TRY(e);
  }
  h->N = N;
  h->nz = nz;
  h->format = CGX_FORMAT_ELL;
  CGX_TRY(alloc_vectors(h, N));
  CUDA_TRY(cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream));
  k_validate_ell<<<grid_stream(h, N), kThreads, 0, h->stream>>>(
      N, maxNz, h->ell_length, h->ell_index, h->flag);
  CUDA_TRY(cudaGetLastError());
  return check_flag(h, "ELL");
}

static cgx_status need_matrix(cgx_handle *h);
static cgx_status ensure_rows(cgx_handle *h);
namespace {
cudaError_t scan(cgx_handle *h, int n, const int *in, int *out, int *sums);
}

// COO entries from the host into the row layout on the device (ingest.cuh):
// validated, stable-sorted by row, so each row keeps its entries in entry
// order -- the order in which serial/SerialCG.cpp:79-85 adds a row's
// products and in which DataMatrix<CRS>::convert and DataMatrix<ELL>::convert
// (Matrix.cpp:203-228, 339-361) lay them out. `format` CRS or COO: the rows
// become the matrix itself; ELL: the rows are kept as the row layout of the
// mixed paths and the tile-major ELL of the SpMV is built from them.
static cgx_status upload_coo_device(cgx_handle *h, int N, int nz, const int *I,
                                    const int *J, const double *V, int format) {
  DeviceGuard guard(h->device);
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  free_matrix(h);
  const char *what = format == CGX_FORMAT_ELL ? "ELL" : format == CGX_FORMAT_CRS ? "CRS" : "COO";

  // The row layout (ptr, index, value), laid out as the CRS upload does.
  Carver c;
  const size_t o_ptr = c.take<int>((size_t)N + 1 + kPad);
  const size_t o_idx = c.take<int>((size_t)nz + kPad);
  const size_t o_val = c.take<double>((size_t)nz + kPad);
  void *rows = nullptr;
  CUDA_TRY(dev_alloc(h, &rows, c.off));
  int *ptr = (int *)((char *)rows + o_ptr);
  int *index = (int *)((char *)rows + o_idx);
  double *value = (double *)((char *)rows + o_val);
  if (format == CGX_FORMAT_ELL) h->rows_mem = rows;
  else h->mat_mem = rows;
  CUDA_TRY(cudaMemsetAsync(rows, 0, c.off, h->stream));

  // Scratch: the entries, two (row, entry) buffers, the per-tile digit
  // counts and their scan.
  const int ntiles = std::max(1, (nz + kSortTile - 1) / kSortTile);
  const int ncount = kRadix * ntiles;
  const int nsums = (ncount + cgx::learned::kScanBlock - 1) / cgx::learned::kScanBlock;
  Carver t;
  const size_t t_i = t.take<int>((size_t)nz + kPad), t_j = t.take<int>((size_t)nz + kPad);
  const size_t t_v = t.take<double>((size_t)nz + kPad);
  const size_t t_k0 = t.take<int>((size_t)nz + kPad), t_v0 = t.take<int>((size_t)nz + kPad);
  const size_t t_k1 = t.take<int>((size_t)nz + kPad), t_v1 = t.take<int>((size_t)nz + kPad);
  const size_t t_h = t.take<int>((size_t)ncount), t_o = t.take<int>((size_t)ncount + 1);
  const size_t t_s = t.take<int>((size_t)nsums);
  void *tmp = nullptr;
  CUDA_TRY(dev_alloc(h, &tmp, t.off));
  char *tb = (char *)tmp;
  int *dI = (int *)(tb + t_i), *dJ = (int *)(tb + t_j);
  double *dV = (double *)(tb + t_v);
  int *kbuf[2] = {(int *)(tb + t_k0), (int *)(tb + t_k1)};
  int *vbuf[2] = {(int *)(tb + t_v0), (int *)(tb + t_v1)};
  int *hist = (int *)(tb + t_h), *offs = (int *)(tb + t_o), *sums = (int *)(tb + t_s);

  cudaError_t e = cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream);
  if (e == cudaSuccess && nz > 0) {
    e = cudaMemcpyAsync(dI, I, sizeof(int) * (size_t)nz, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(dJ, J, sizeof(int) * (size_t)nz, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(dV, V, sizeof(double) * (size_t)nz, cudaMemcpyHostToDevice,
                          h->stream);
    if (e == cudaSuccess) {
      k_coo_validate<<<grid_stream(h, nz), kThreads, 0, h->stream>>>(N, nz, dI, dJ, h->flag);
      e = cudaGetLastError();
    }
  }
  int flag = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&flag, h->flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess && flag) {
    dev_free(h, tmp);
    free_matrix(h);
    std::string m = std::string("invalid ") + what + " matrix:";
    if (flag & 1) m += " row index outside [0, N);";
    if (flag & 2) m += " column index outside [0, N);";
    return fail(CGX_ERROR_INVALID_ARGUMENT, m);
  }
  // The sort: as many 8-bit passes as N - 1 has significant bits (one at
  // least); pass p sorts stably by bits 8p .. 8p + 7 of the row.
  const int* keys = dI;
  const int* order = nullptr;
  if (e == cudaSuccess && nz > 0) {
    int bits = 0;
    while (bits < 31 && ((unsigned)(N - 1) >> bits) != 0u) bits++;
    const int passes = std::max(1, (bits + 7) / 8);
    for (int pass = 0; pass < passes && e == cudaSuccess; pass++) {
      const int shift = 8 * pass;
      k_sort_hist<<<ntiles, kThreads, 0, h->stream>>>(nz, keys, shift, ntiles, hist);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = scan(h, ncount, hist, offs, sums);
      if (e == cudaSuccess) {
        k_sort_scatter<<<ntiles, kThreads, 0, h->stream>>>(
            nz, keys, order, shift, ntiles, offs, kbuf[pass & 1], vbuf[pass & 1]);
        e = cudaGetLastError();
      }
      keys = kbuf[pass & 1];
      order = vbuf[pass & 1];
    }
  }
  if (e == cudaSuccess) {
    k_rows_ptr<<<grid_stream(h, (size_t)nz + 1), kThreads, 0, h->stream>>>(
        N, nz, nz > 0 ? keys : dI, ptr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && nz > 0) {
    k_rows_gather<<<grid_stream(h, nz), kThreads, 0, h->stream>>>(nz, order, dJ, dV,
                                                                  index, value);
    e = cudaGetLastError();
  }
  std::vector<int> hptr((size_t)N + 1);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hptr.data(), ptr, sizeof(int) * ((size_t)N + 1),
                        cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  dev_free(h, tmp);
  CUDA_TRY(e);
  h->ptr = ptr;
  h->index = index;
  h->value = value;
  set_tile_caps(h, hptr.data(), N);

  if (format == CGX_FORMAT_ELL) {
    // Width = the longest row (MatrixDataELL's maxNz, Matrix.cpp:339-361).
    CUDA_TRY(cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream));
    k_row_len_max<<<grid_stream(h, N), kThreads, 0, h->stream>>>(N, ptr, h->flag);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(h->host_scalar, h->flag, sizeof(int),
                             cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    const int width = *(int *)h->host_scalar;
    const size_t elems = ell_elems(N, width);
    Carver m;
    const size_t m_len = m.take<int>((size_t)N + kPad);
    const size_t m_idx = m.take<int>(elems + kPad);
    const size_t m_dat = m.take<double>(elems + kPad);
    CUDA_TRY(dev_alloc(h, (void **)&h->mat_mem, m.off));
    char *base = (char *)h->mat_mem;
    h->ell_length = (int *)(base + m_len);
    h->ell_index = (int *)(base + m_idx);
    h->ell_data = (double *)(base + m_dat);
    h->ell_width = width;
    CUDA_TRY(cudaMemsetAsync(h->mat_mem, 0, m.off, h->stream));
    k_rows_to_ell<<<grid_stream(h, N), kThreads, 0, h->stream>>>(
        N, width, ptr, index, value, h->ell_length, h->ell_index, h->ell_data);
    CUDA_TRY(cudaGetLastError());
  }
  h->N = N;
  h->nz = nz;
  h->format = format;
  CGX_TRY(alloc_vectors(h, N));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CGX_SUCCESS;
}

cgx_status cgx_upload_coo_as(cgx_handle *h, int N, int nz, const int *I,
                             const int *J, const double *V, int format) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  if (N <= 0 || nz < 0 || (nz > 0 && (!I || !J || !V)))
    return fail(CGX_ERROR_INVALID_ARGUMENT, "bad COO sizes or pointers");
  if (format != CGX_FORMAT_COO && format != CGX_FORMAT_CRS && format != CGX_FORMAT_ELL)
    return fail(CGX_ERROR_INVALID_ARGUMENT, "unknown matrix format");
  return upload_coo_device(h, N, nz, I, J, V, format);
}

cgx_status cgx_upload_coo(cgx_handle *h, int N, int nz, const int *I,
                          const int *J, const double *V) {
  return cgx_upload_coo_as(h, N, nz, I, J, V, CGX_FORMAT_COO);
}

cgx_status cgx_download_crs(cgx_handle *h, int *ptr, int *index, double *value) {
  CGX_TRY(need_matrix(h));
  DeviceGuard guard(h->device);
  CGX_TRY(ensure_rows(h));
  if (ptr)
    CUDA_TRY(cudaMemcpyAsync(ptr, h->ptr, sizeof(int) * ((size_t)h->N + 1),
                             cudaMemcpyDeviceToHost, h->stream));
  if (index && h->nz > 0)
    CUDA_TRY(cudaMemcpyAsync(index, h->index, sizeof(int) * (size_t)h->nz,
                             cudaMemcpyDeviceToHost, h->stream));
  if (value && h->nz > 0)
    CUDA_TRY(cudaMemcpyAsync(value, h->value, sizeof(double) * (size_t)h->nz,
                             cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CGX_SUCCESS;
}

cgx_status cgx_download_ell(cgx_handle *h, int *max_nz, int *length, int *index,
                            double *data) {
  CGX_TRY(need_matrix(h));
  if (h->format != CGX_FORMAT_ELL)
    return fail(CGX_ERROR_INVALID_STATE, "the uploaded matrix is not ELL");
  DeviceGuard guard(h->device);
  const int N = h->N, W = h->ell_width;
  if (max_nz) *max_nz = W;
  if (length)
    CUDA_TRY(cudaMemcpyAsync(length, h->ell_length, sizeof(int) * (size_t)N,
                             cudaMemcpyDeviceToHost, h->stream));
  const size_t celems = (size_t)N * (size_t)W;
  if ((index || data) && celems > 0) {
    Carver t;
    const size_t o_i = t.take<int>(celems), o_d = t.take<double>(celems);
    void *tmp = nullptr;
    CUDA_TRY(dev_alloc(h, &tmp, t.off));
    int *ci = (int *)((char *)tmp + o_i);
    double *cd = (double *)((char *)tmp + o_d);
    k_ell_columns<<<grid_stream(h, celems), kThreads, 0, h->stream>>>(
        N, W, h->ell_length, h->ell_index, h->ell_data, ci, cd);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && index)
      e = cudaMemcpyAsync(index, ci, sizeof(int) * celems, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && data)
      e = cudaMemcpyAsync(data, cd, sizeof(double) * celems, cudaMemcpyDeviceToHost,
                          h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    dev_free(h, tmp);
    CUDA_TRY(e);
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CGX_SUCCESS;
}

// The row layout (ptr, index, value) that the Jacobi set-up, the FP32 copies
// and the learned set-up read: CRS and COO hold it from the upload; for ELL
// it is built on first use (ensure_rows).
static cgx_status ensure_rows(cgx_handle *h);

static cgx_status need_matrix(cgx_handle *h) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  if (h->format < 0)
    return fail(CGX_ERROR_INVALID_STATE, "no matrix has been uploaded");
  return CGX_SUCCESS;
}

static cgx_status vec_arg(cgx_handle *h, int v, double **out) {
  if (v < CGX_VECTOR_K || v > CGX_VECTOR_Z)
    return fail(CGX_ERROR_INVALID_ARGUMENT, "invalid cgx_vector");
  *out = h->vec[v];
  return CGX_SUCCESS;
}

cgx_status cgx_upload_jacobi(cgx_handle *h, const double *C) {
  CGX_TRY(need_matrix(h));
  if (!C) return fail(CGX_ERROR_INVALID_ARGUMENT, "C is NULL");
  DeviceGuard guard(h->device);
  CUDA_TRY(cudaMemcpyAsync(h->C, C, sizeof(double) * h->N,
                           cudaMemcpyHostToDevice, h->stream));
  h->c_valid = true;
  h->f32_valid = false;
  return CGX_SUCCESS;
}

cgx_status cgx_jacobi_from_matrix(cgx_handle *h) {
  CGX_TRY(need_matrix(h));
  DeviceGuard guard(h->device);
  CGX_TRY(ensure_rows(h));
  k_jacobi_from_crs<<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(
      h->N, h->ptr, h->index, h->value, h->C);
  CUDA_TRY(cudaGetLastError());
  h->c_valid = true;
  h->f32_valid = false;
  return CGX_SUCCESS;
}

cgx_status cgx_set_vector(cgx_handle *h, cgx_vector v, const double *host) {
  CGX_TRY(need_matrix(h));
  double *d;
  CGX_TRY(vec_arg(h, v, &d));
  if (!host) return fail(CGX_ERROR_INVALID_ARGUMENT, "host is NULL");
  DeviceGuard guard(h->device);
  CUDA_TRY(cudaMemcpyAsync(d, host, sizeof(double) * h->N,
                           cudaMemcpyHostToDevice, h->stream));
  return CGX_SUCCESS;
}

cgx_status cgx_get_vector(cgx_handle *h, cgx_vector v, double *host) {
  CGX_TRY(need_matrix(h));
  double *d;
  CGX_TRY(vec_arg(h, v, &d));
  if (!host) return fail(CGX_ERROR_INVALID_ARGUMENT, "host is NULL");
  DeviceGuard guard(h->device);
  CUDA_TRY(cudaMemcpyAsync(host, d, sizeof(double) * h->N,
                           cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CGX_SUCCESS;
}

cgx_status cgx_fill_vector(cgx_handle *h, cgx_vector v, double value) {
  CGX_TRY(need_matrix(h));
  double *d;
  CGX_TRY(vec_arg(h, v, &d));
  DeviceGuard guard(h->device);
  k_fill<<<grid_stream(h, h->N), kThreads, 0, h->stream>>>((size_t)h->N,
                                                           value, d);
  CUDA_TRY(cudaGetLastError());
  return CGX_SUCCESS;
}

// --- per-kernel interface -----------------------------------------------------

cgx_status cgx_copy(cgx_handle *h, cgx_vector dst, cgx_vector src) {
  CGX_TRY(need_matrix(h));
  double *d, *s;
  CGX_TRY(vec_arg(h, dst, &d));
  CGX_TRY(vec_arg(h, src, &s));
  DeviceGuard guard(h->device);
  if (d != s)
    CUDA_TRY(cudaMemcpyAsync(d, s, sizeof(double) * h->N,
                             cudaMemcpyDeviceToDevice, h->stream));
  return CGX_SUCCESS;
}

cgx_status cgx_matvec(cgx_handle *h, cgx_vector x, cgx_vector y) {
  CGX_TRY(need_matrix(h));
  double *dx, *dy;
  CGX_TRY(vec_arg(h, x, &dx));
  CGX_TRY(vec_arg(h, y, &dy));
  if (dx == dy)
    return fail(CGX_ERROR_INVALID_ARGUMENT, "matvec input and output alias");
  DeviceGuard guard(h->device);
  CUDA_TRY(launch_spmv(h, dx, OpStore<double>{dy}));
  return CGX_SUCCESS;
}

cgx_status cgx_axpy(cgx_handle *h, double a, cgx_vector x, cgx_vector y) {
  CGX_TRY(need_matrix(h));
  double *dx, *dy;
  CGX_TRY(vec_arg(h, x, &dx));
  CGX_TRY(vec_arg(h, y, &dy));
  DeviceGuard guard(h->device);
  k_axpy<<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(h->N, a, dx, dy);
  CUDA_TRY(cudaGetLastError());
  return CGX_SUCCESS;
}

cgx_status cgx_xpay(cgx_handle *h, cgx_vector x, double a, cgx_vector y) {
  CGX_TRY(need_matrix(h));
  double *dx, *dy;
  CGX_TRY(vec_arg(h, x, &dx));
  CGX_TRY(vec_arg(h, y, &dy));
  DeviceGuard guard(h->device);
  k_xpay<<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(h->N, dx, a, dy);
  CUDA_TRY(cudaGetLastError());
  return CGX_SUCCESS;
}

cgx_status cgx_dot(cgx_handle *h, cgx_vector a, cgx_vector b, double *result) {
  CGX_TRY(need_matrix(h));
  double *da, *db;
  CGX_TRY(vec_arg(h, a, &da));
  CGX_TRY(vec_arg(h, b, &db));
  if (!result) return fail(CGX_ERROR_INVALID_ARGUMENT, "result is NULL");
  DeviceGuard guard(h->device);
  k_dot<<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(
      h->N, da, db, h->dot_out, h->partials, ticket(h, kTicketDot));
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(h->host_scalar, h->dot_out, sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  *result = h->host_scalar[0];
  return CGX_SUCCESS;
}

cgx_status cgx_apply_jacobi(cgx_handle *h, cgx_vector x, cgx_vector y) {
  CGX_TRY(need_matrix(h));
  double *dx, *dy;
  CGX_TRY(vec_arg(h, x, &dx));
  CGX_TRY(vec_arg(h, y, &dy));
  if (!h->c_valid)
    return fail(CGX_ERROR_INVALID_STATE, "Jacobi preconditioner not set");
  DeviceGuard guard(h->device);
  k_jacobi<<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(h->N, h->C, dx,
                                                             dy);
  CUDA_TRY(cudaGetLastError());
  return CGX_SUCCESS;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Solve

static cgx_status device_errors(cgx_handle *h) {
  if (h->host_st->error & 1)
    return fail(CGX_ERROR_DEVICE,
                "a bulk-copy wait in the SpMV timed out; results are invalid");
  if (h->host_st->error & 2)
    return fail(CGX_ERROR_DEVICE,
                "the device loop guard stopped a loop that did not terminate");
  if (h->host_st->error & kErrGridSync)
    return fail(CGX_ERROR_DEVICE,
                "a grid barrier of the persistent inner solve timed out; results are invalid");

  return CGX_SUCCESS;
}

// Event pool of the per-kernel timing mode.
static cgx_status ensure_event_pool(cgx_handle *h) {
  while ((int)h->evpool.size() < 4 * kChunk) {
    cudaEvent_t e;
    CUDA_TRY(cudaEventCreate(&e));
    h->evpool.push_back(e);
  }
  return CGX_SUCCESS;
}

// Adds the three segments (SpMV | update | direction) of the first `ran`
// iterations of the last chunk; iterations enqueued after the stop ran no
// kernel work and are not counted.
static cudaError_t add_segments(cgx_handle *h, int ran, double &t_spmv,
                                double &t_upd, double &t_dir) {
  for (int j = 0; j < std::min(ran, kChunk); j++) {
    float a = 0, b = 0, c = 0;
    cudaError_t e;
    if ((e = cudaEventElapsedTime(&a, h->evpool[4 * j], h->evpool[4 * j + 1])) != cudaSuccess ||
        (e = cudaEventElapsedTime(&b, h->evpool[4 * j + 1], h->evpool[4 * j + 2])) != cudaSuccess ||
        (e = cudaEventElapsedTime(&c, h->evpool[4 * j + 2], h->evpool[4 * j + 3])) != cudaSuccess)
      return e;
    t_spmv += a;
    t_upd += b;
    t_dir += c;
  }
  return cudaSuccess;
}

static cgx_status solve_fp64(cgx_handle *h, const cgx_options &o,
                             cgx_result &res) {
  const bool jacobi = o.preconditioner == CGX_PRECONDITIONER_JACOBI;
  if (jacobi && !h->c_valid)
    return fail(CGX_ERROR_INVALID_STATE, "Jacobi preconditioner not set");
  cudaStream_t s = h->stream;
  // The persistent mode is an inner-solve mode of the mixed paths.
  const int loop =
      o.loop == CGX_LOOP_PERSISTENT || o.loop == CGX_LOOP_PERSISTENT_SPLIT ? CGX_LOOP_GRAPH
                                                                           : o.loop;

  if (loop == CGX_LOOP_GRAPH) {
    GraphEntry *ge = nullptr;
    const int key = 100 + (jacobi ? 1 : 0);
    CGX_TRY(build_while_graph(
        h, key, [&] { return launch_pcg_setup(h, jacobi); },
        [&] {
          cudaError_t e = launch_pcg_iteration(h, jacobi);
          if (e != cudaSuccess) return e;
          k_loop_guard<<<1, 1, 0, h->stream>>>(h->st);
          return cudaGetLastError();
        },
        [&] { return cudaSuccess; }, &ge));
    reset_host_state(h, o.max_iterations, o.tolerance, true, ge->cond);
    CGX_TRY(push_state(h));
    CUDA_TRY(cudaEventRecord(h->ev[0], s));
    CUDA_TRY(cudaGraphLaunch(ge->exec, s));
    CUDA_TRY(cudaEventRecord(h->ev[1], s));
    CGX_TRY(pull_state(h));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
    res.solve_ms = ms;
  } else if (loop == CGX_LOOP_CHUNKED) {
    GraphEntry *ge = nullptr;
    const int key = 200 + (jacobi ? 1 : 0);
    CGX_TRY(build_chunk_graph(
        h, key, [&] { return launch_pcg_iteration(h, jacobi); }, &ge));
    reset_host_state(h, o.max_iterations, o.tolerance, false, 0);
    CGX_TRY(push_state(h));
    CUDA_TRY(cudaEventRecord(h->ev[0], s));
    CUDA_TRY(launch_pcg_setup(h, jacobi));
    const int maxLaunches = o.max_iterations / kChunk + 2;
    for (int l = 0; l < maxLaunches; l++) {
      CUDA_TRY(cudaGraphLaunch(ge->exec, s));
      CUDA_TRY(cudaMemcpyAsync(h->host_scalar, &h->st->stop, sizeof(int),
                               cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaStreamSynchronize(s));
      if (*(int *)h->host_scalar) break;
    }
    CUDA_TRY(cudaEventRecord(h->ev[1], s));
    CGX_TRY(pull_state(h));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
    res.solve_ms = ms;
  } else {
    reset_host_state(h, o.max_iterations, o.tolerance, false, 0);
    CGX_TRY(push_state(h));
    CUDA_TRY(cudaEventRecord(h->ev[4], s));
    CUDA_TRY(launch_pcg_setup(h, jacobi));
    double t_spmv = 0, t_upd = 0, t_dir = 0;
    int it = 0;
    CGX_TRY(ensure_event_pool(h));
    const int maxChunks = o.max_iterations / kChunk + 2;
    for (int c = 0; c < maxChunks; c++) {
      for (int j = 0; j < kChunk; j++)
        CUDA_TRY(launch_pcg_iteration(h, jacobi, &h->evpool[4 * j]));
      CGX_TRY(pull_state(h));
      const int now = h->host_st->iteration;
      CUDA_TRY(add_segments(h, now - it, t_spmv, t_upd, t_dir));
      it = now;
      if (h->host_st->stop) break;
    }
    CUDA_TRY(cudaEventRecord(h->ev[5], s));
    CGX_TRY(pull_state(h));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, h->ev[4], h->ev[5]));
    res.solve_ms = ms;
    res.spmv_ms = t_spmv;
    res.update_ms = t_upd;
    res.direction_ms = t_dir;
    res.spmv_launches = res.update_launches = res.direction_launches = it;
  }
  CGX_TRY(device_errors(h));
  res.iterations = h->host_st->iteration;
  res.residual = h->host_st->residual;
  res.converged = h->host_st->converged;
  return CGX_SUCCESS;
}

namespace {
cgx_status build_sellu(cgx_handle *h, const int *ptr, const int *col,
                       size_t nnz, SellU &S);
}

// The offsets of A (k_band_offsets): B.K = 0 unless they form a symmetric
// set with at most kBandMaxK non-negative members.
static cgx_status band_plan(cgx_handle *h, Band &B) {
  B = Band{};
  const int N = h->N;
  int *table = nullptr;
  CUDA_TRY(dev_alloc(h, (void **)&table, sizeof(int) * kBandTable));
  std::vector<int> host(kBandTable, kBandEmpty);
  int flag = 0;
  cudaError_t e = cudaMemcpyAsync(table, host.data(), sizeof(int) * kBandTable,
                                  cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream);
  if (e == cudaSuccess) {
    k_band_offsets<<<grid_stream(h, N), kThreads, 0, h->stream>>>(
        N, h->ptr, h->index, table, h->flag);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(host.data(), table, sizeof(int) * kBandTable,
                        cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&flag, h->flag, sizeof(int), cudaMemcpyDeviceToHost,
                        h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  dev_free(h, table);
  CUDA_TRY(e);
  if (flag) return CGX_SUCCESS;
  std::vector<int> D;
  for (int v : host)
    if (v != kBandEmpty) D.push_back(v);
  std::sort(D.begin(), D.end());
  std::vector<int> up{0};
  // |d| < N, so -d cannot overflow.
  for (int d : D) {
    if (!std::binary_search(D.begin(), D.end(), -d)) return CGX_SUCCESS;
    if (d > 0) up.push_back(d);
  }
  if ((int)up.size() > kBandMaxK) return CGX_SUCCESS;
  B.K = (int)up.size();
  for (int k = 0; k < B.K; k++) B.d[k] = up[k];
  return CGX_SUCCESS;
}

// U from A's current values and the symmetry check; B.ok if it passed.
static cgx_status band_fill(cgx_handle *h, Band &B) {
  const int N = h->N;
  B.ok = false;
  const size_t bytes = sizeof(float) * (size_t)N * kBandMaxK;
  if (!B.U) CUDA_TRY(dev_alloc(h, (void **)&B.U, bytes));
  unsigned long long *counts = nullptr;
  CUDA_TRY(dev_alloc(h, (void **)&counts, 2 * sizeof(unsigned long long)));
  BandOffsets o{};
  o.K = B.K;
  for (int k = 0; k < B.K; k++) o.d[k] = B.d[k];
  unsigned long long hc[2] = {0, 0};
  int flag = 0;
  cudaError_t e = cudaMemsetAsync(B.U, 0, bytes, h->stream);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream);
  if (e == cudaSuccess) {
    k_band_fill<<<grid_stream(h, N), kThreads, 0, h->stream>>>(
        N, h->ptr, h->index, h->value, o, B.U, counts, h->flag);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_band_check<<<grid_stream(h, N), kThreads, 0, h->stream>>>(
        N, h->ptr, h->index, h->value, o, B.U, counts, h->flag);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hc, counts, sizeof(hc), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&flag, h->flag, sizeof(int), cudaMemcpyDeviceToHost,
                        h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  dev_free(h, counts);
  CUDA_TRY(e);
  B.ok = flag == 0 && hc[0] == hc[1];
  return CGX_SUCCESS;
}

static cgx_status ensure_f32(cgx_handle *h) {
  if (h->f32_valid) return CGX_SUCCESS;
  const int N = h->N;
  if (!h->f32_mem) {
    Carver c;
    size_t o_v = c.take<float>((size_t)h->nz + kPad);
    size_t o_c = c.take<float>((size_t)N + kPad);
    size_t o_d = c.take<float>((size_t)N + kPad);
    size_t o_r = c.take<float>((size_t)N + kPad);
    size_t o_p = c.take<float>((size_t)N + kPad);
    size_t o_q = c.take<float>((size_t)N + kPad);
    size_t o_pb = c.take<float>((size_t)N + kPad);
    size_t o_rb = c.take<float>((size_t)N + kPad);
    size_t o_z = c.take<float>((size_t)N + kPad);
    size_t o_r64 = c.take<double>((size_t)N + kPad);
    size_t o_pp = c.take<double>((size_t)kPersistSlots * kMaxGrid);
    size_t o_ps = c.take<unsigned long long>(1);
    size_t o_i16 = c.take<int16_t>((size_t)h->nz + kPad);
    CUDA_TRY(dev_alloc(h, (void **)&h->f32_mem, c.off));
    CUDA_TRY(cudaMemsetAsync(h->f32_mem, 0, c.off, h->stream));
    char *base = (char *)h->f32_mem;
    h->value32 = (float *)(base + o_v);
    h->C32 = (float *)(base + o_c);
    h->d32 = (float *)(base + o_d);
    h->r32 = (float *)(base + o_r);
    h->p32 = (float *)(base + o_p);
    h->q32 = (float *)(base + o_q);
    h->p32b = (float *)(base + o_pb);
    h->r32b = (float *)(base + o_rb);
    h->z32 = (float *)(base + o_z);
    h->r64 = (double *)(base + o_r64);
    h->persist_part = (double *)(base + o_pp);
    h->persist_sync = (unsigned long long *)(base + o_ps);
    h->idx16 = (int16_t *)(base + o_i16);
  }
  k_to_f32<<<grid_stream(h, h->nz), kThreads, 0, h->stream>>>(
      (size_t)h->nz, h->value, h->value32);
  CUDA_TRY(cudaGetLastError());
  k_to_f32<<<grid_stream(h, N), kThreads, 0, h->stream>>>((size_t)N, h->C,
                                                          h->C32);
  CUDA_TRY(cudaGetLastError());
  // Symmetric band copy of A when it fits (planned once per pattern, filled
  // and checked on every refresh); otherwise the SELL-U copy: the pattern
  // once per matrix, the value array once it exists, the values on every
  // refresh.
  if (!h->band_tried) {
    h->band_tried = true;
    CGX_TRY(band_plan(h, h->band));
  }
  if (h->band.K > 0) {
    CGX_TRY(band_fill(h, h->band));
    if (!h->band.ok) band_drop_values(h, h->band);
  }
  if (!h->band.ok && !h->sa_tried) {
    h->sa_tried = true;
    CGX_TRY(build_sellu(h, h->ptr, h->index, (size_t)h->nz, h->sa));
    // Mostly per-row slices (an irregular matrix) pad every row of a slice
    // to its longest one; A's FP32 CRS is faster there (measured on the 2M
    // point geometric graph: 64 against 71 us per product).
    if (h->sa.ok && 2 * h->sa.uniform < (long long)((h->N + 31) / 32))
      sellu_free(h, h->sa);
  }
  if (h->sa.ok && !h->sa_val) {
    CUDA_TRY(dev_alloc(h, (void **)&h->sa_val, sizeof(float) * (h->sa.slots + kPad)));
    CUDA_TRY(cudaMemsetAsync(h->sa_val, 0, sizeof(float) * (h->sa.slots + kPad),
                             h->stream));
  }
  if (h->sa.ok) {
    k_sellu_scatter<double, float><<<grid_stream(h, h->nz), kThreads, 0, h->stream>>>(
        (size_t)h->nz, h->sa.map, h->value, h->sa_val);
    CUDA_TRY(cudaGetLastError());
  }
  CUDA_TRY(cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream));
  k_delta16<<<grid_stream(h, N), kThreads, 0, h->stream>>>(N, h->ptr, h->index,
                                                           h->idx16, h->flag);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(h->host_scalar, h->flag, sizeof(int),
                           cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->compact16 = *(int *)h->host_scalar == 0;
  // The graphs hold pointers and layout choices, not values: a refresh that
  // keeps them keeps the graphs. (Destroying the executable graphs on every
  // refresh cost the first solve after it up to 40 ms of host time now and
  // then.)
  const std::array<uintptr_t, 10> key = {
      (uintptr_t)h->value32, (uintptr_t)h->idx16,  (uintptr_t)h->compact16,
      (uintptr_t)h->band.U,  (uintptr_t)h->band.K, (uintptr_t)h->band.ok,
      (uintptr_t)h->sa.meta, (uintptr_t)h->sa_val, (uintptr_t)h->sa.ok,
      (uintptr_t)h->C32};
  if (key != h->f32_key) {
    drop_graphs(h);
    h->f32_key = key;
  }
  h->f32_valid = true;
  return CGX_SUCCESS;
}

static cgx_status true_residual_r2(cgx_handle *h, double *r2) {
  CUDA_TRY(launch_spmv(h, h->vec[CGX_VECTOR_X],
                       OpTrueResidual{h->vec[CGX_VECTOR_K],
                                      h->r64 ? h->r64 : h->tmp,
                                      ticket(h, kTicketTrue)}));
  CUDA_TRY(cudaMemcpyAsync(h->host_scalar, &h->st->r2, sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  *r2 = h->host_scalar[0];
  return CGX_SUCCESS;
}

static GBandView gband_view(const cgx_handle *h) {
  GBandView B;
  B.val = h->L->gb_val;
  B.N = h->N;
  for (int k = 0; k < kBandMaxK; k++) B.d[k] = h->L->gb_d[k];
  return B;
}

template <bool TRANS, typename Op>
static cudaError_t launch_gband(cgx_handle *h, const float *x, Op op) {
  return launch_rows(h, k_gband<TRANS, Op>, h->N, gband_view(h), x, op, h->st,
                     h->partials);
}

// z = G (G^T r) + eps C r with <r,z> (start: also p = z and rho).
static cudaError_t launch_learned_apply(cgx_handle *h, bool start) {
  Learned *L = h->L;
  const OpLearnedZ zop{h->r32, h->C32, L->z32, h->p32, L->eps, start ? 1 : 0,
                       ticket(h, kTicketInnerStart)};
  cudaError_t e;
  if (L->gb_ok) {
    e = launch_gband<true>(h, h->r32, OpInnerStore{L->y32});
    if (e != cudaSuccess) return e;
    return launch_gband<false>(h, L->y32, zop);
  }
  if (L->sell_ok) {
    e = launch_sellu(h, L->st, L->st_val, h->r32, OpInnerStore{L->y32});
    if (e != cudaSuccess) return e;
    return launch_sellu(h, L->sg, L->sg_val, L->y32, zop);
  }
  CrsView<float, int> GT{L->tptr, L->tcol, L->gts, h->N, h->tile_cap};
  CrsView<float, int> Gv{L->gptr, L->gcol, L->gs, h->N, h->tile_cap};
  e = launch_crs_view(h, GT, h->r32, OpInnerStore{L->y32});
  if (e != cudaSuccess) return e;
  return launch_crs_view(h, Gv, L->y32, zop);
}

// One inner solve as a persistent cooperative launch (persist.cuh), after
// the path's start kernel(s). The grid is what the SMs hold at once, as a
// cooperative launch requires (and no more CTAs than 256-row tiles or
// partial-sum slots).
enum class InnerForm { kGraph, kFused, kSplit, kSell };

static cudaError_t launch_inner_persist(cgx_handle *h, bool learned, InnerForm form) {
  PersistArgs a;
  a.p[0] = h->p32;
  a.p[1] = h->p32b;
  a.r[0] = h->r32;
  a.r[1] = h->r32b;
  a.z = learned ? h->L->z32 : h->z32;
  a.d = h->d32;
  a.q = h->q32;
  a.y = learned ? h->L->y32 : nullptr;
  a.C = h->C32;
  a.eps = learned ? h->L->eps : 0.f;
  a.part = h->persist_part;
  a.sync = h->persist_sync;
  CgState *st = h->st;
  // The grid: as many CTAs as the SMs hold, at most one per T-row tile.
  auto grid_for = [&](const void *kern, int T, int *grid) {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, T, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    const long long tiles = ((long long)h->N + T - 1) / T;
    *grid = (int)std::max<long long>(
        1, std::min<long long>({(long long)h->num_sms * per_sm, kMaxGrid, tiles}));
    return cudaMemsetAsync(a.sync, 0, sizeof(unsigned long long), h->stream);
  };
  int grid = 0;
  cudaError_t e;
  if (form == InnerForm::kSell) {
    constexpr int T = kPersistSellThreads, B = kPersistSellMinB;
    const SellUView<float> A{h->sa.meta, h->sa.off, h->sa_val, h->N};
    SellUView<__nv_bfloat16> G{}, GT{};
    if (learned) {
      G = SellUView<__nv_bfloat16>{h->L->sg.meta, h->L->sg.off, h->L->sg_val, h->N};
      GT = SellUView<__nv_bfloat16>{h->L->st.meta, h->L->st.off, h->L->st_val, h->N};
    }
    const void *kern = learned ? (const void *)k_inner_persist_sell<true, T, B>
                               : (const void *)k_inner_persist_sell<false, T, B>;
    if ((e = grid_for(kern, T, &grid)) != cudaSuccess) return e;
    void *args[] = {(void *)&A, &G, &GT, &a, &st};
    return cudaLaunchCooperativeKernel(kern, grid, T, args, 0, h->stream);
  }
  BandView<4> A = band_view(h);
  GBandView G{};
  if (learned) G = gband_view(h);
  constexpr int T = kPersistThreads, F = kPersistFusedMinB;
  constexpr int SL = kPersistSplitMinB[1], SJ = kPersistSplitMinB[0];
  constexpr int PF = kPersistPrefetchRows;
  const bool split = form == InnerForm::kSplit;
  const bool pf = h->N >= kPersistPrefetchMinRows;
  const void *kern =
      split ? (learned ? (pf ? (const void *)k_inner_persist_split<true, T, SL, PF>
                             : (const void *)k_inner_persist_split<true, T, SL, 0>)
                       : (pf ? (const void *)k_inner_persist_split<false, T, SJ, PF>
                             : (const void *)k_inner_persist_split<false, T, SJ, 0>))
            : (learned ? (const void *)k_inner_persist<true, T, F>
                       : (const void *)k_inner_persist<false, T, F>);
  if ((e = grid_for(kern, T, &grid)) != cudaSuccess) return e;
  void *args[] = {&A, &G, &a, &st};
  return cudaLaunchCooperativeKernel(kern, grid, T, args, 0, h->stream);
}

// The SELL-U form of the persistent inner solve needs A's inner product on
// SELL-U with every slice uniform, and for the learned path G and G^T the
// same.
static bool sell_fits(const cgx_handle *h, bool learned) {
  const long long slices = ((long long)h->N + 31) / 32;
  if (h->band.ok || !h->sa.ok || !h->sa_val || h->sa.uniform != slices)
    return false;
  if (!learned) return true;
  const Learned *L = h->L;
  return L && !L->gb_ok && L->sell_ok && L->sg.uniform == slices && L->st.uniform == slices;
}

// The band forms need A on the band form (offsets 0 < d1 < d2 < d3, at most
// four), and for the learned path the factor on the band with the same
// offsets.
static bool persist_fits(const cgx_handle *h, bool learned) {
  if (!h->band.ok || h->band.K > 4) return false;
  if (!learned) return true;
  if (!(h->L && h->L->gb_ok)) return false;
  for (int k = 0; k < kBandMaxK; k++)
    if (h->L->gb_d[k] != (k < h->band.K ? h->band.d[k] : 0)) return false;
  return true;
}

// Which inner solve a mixed solve runs: the graph of per-iteration kernels,
// or a persistent launch per inner solve, fused (systems up to
// kPersistFusedMaxRows rows) or split (larger ones). CGX_LOOP_PERSISTENT and
// CGX_LOOP_PERSISTENT_SPLIT force their form on the band; the default
// CGX_LOOP_GRAPH takes the persistent form that measured fastest.
static InnerForm inner_form(const cgx_handle *h, const cgx_options &o, bool learned) {
  if (sell_fits(h, learned) &&
      (o.loop == CGX_LOOP_GRAPH || o.loop == CGX_LOOP_PERSISTENT_SPLIT))
    return InnerForm::kSell;
  if (!persist_fits(h, learned)) return InnerForm::kGraph;
  if (o.loop == CGX_LOOP_PERSISTENT) return InnerForm::kFused;
  if (o.loop == CGX_LOOP_PERSISTENT_SPLIT) return InnerForm::kSplit;
  if (o.loop != CGX_LOOP_GRAPH) return InnerForm::kGraph;
  return h->N <= kPersistFusedMaxRows ? InnerForm::kFused : InnerForm::kSplit;
}

static cudaError_t launch_learned_start(cgx_handle *h) {
  k_inner_start_z<<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(
      h->N, h->r64, h->r32, h->d32, h->st, h->partials,
      ticket(h, kTicketInnerStart));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_learned_apply(h, true);
}

// One learned inner iteration: five kernels, whose kernel-mode segments are
// (q = A p | r update and the apply | p update).
static cudaError_t launch_learned_iteration(cgx_handle *h, cudaEvent_t *evs = nullptr) {
  cudaError_t e;
  if (evs) cudaEventRecord(evs[0], h->stream);
  e = launch_inner_q(h);
  if (e != cudaSuccess) return e;
  if (evs) cudaEventRecord(evs[1], h->stream);
  const int g = grid_stream(h, h->N);
  k_inner_update_z<<<g, kThreads, 0, h->stream>>>(
      h->N, h->r32, h->q32, h->st, h->partials, ticket(h, kTicketInnerUpdate));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = launch_learned_apply(h, false)) != cudaSuccess) return e;
  if (evs) cudaEventRecord(evs[2], h->stream);
  k_inner_direction_z<<<g, kThreads, 0, h->stream>>>(h->N, h->d32, h->p32,
                                                     h->L->z32, h->st);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (evs) cudaEventRecord(evs[3], h->stream);
  return cudaSuccess;
}

// FP32-inner / FP64-refinement solve. The inner preconditioner is Jacobi or
// the learned factor. An outer step whose FP64 true residual is NaN/Inf or
// shrinks by less than half (the FP32 inner solve broke down or stalled:
// values beyond the FP32 range, a matrix too ill-conditioned for FP32, a
// corrupt factor) is undone, x is restored to where the step started, and
// the solve finishes with plain FP64 Jacobi-CG from there
// (result.fell_back = 1), the reference's algorithm, with its own budget of
// max_iterations.
static cgx_status solve_mixed(cgx_handle *h, const cgx_options &o,
                              cgx_result &res) {
  CGX_TRY(ensure_rows(h));
  const bool want_learned = o.preconditioner == CGX_PRECONDITIONER_LEARNED;
  if (o.preconditioner != CGX_PRECONDITIONER_JACOBI && !want_learned)
    return fail(CGX_ERROR_UNSUPPORTED,
                "mixed precision supports the Jacobi and learned preconditioners");
  if (!h->c_valid)
    return fail(CGX_ERROR_INVALID_STATE, "Jacobi preconditioner not set");
  if (want_learned && !(h->L && h->L->has_factor))
    return fail(CGX_ERROR_INVALID_STATE,
                "learned factor not set (cgx_learned_setup + cgx_learned_factor)");
  cudaStream_t s = h->stream;
  CUDA_TRY(cudaEventRecord(h->ev[6], s));
  CGX_TRY(ensure_f32(h));

  // The persistent inner solves (persist.cuh): the fused form, and the split
  // one where persist_defers_d, leave d's last update pending; the fused
  // form's start also stores z.
  const InnerForm form = inner_form(h, o, want_learned);
  const bool persist = form != InnerForm::kGraph;
  const bool pending =
      form == InnerForm::kFused ||
      (form == InnerForm::kSplit &&
       persist_defers_d(want_learned,
                        h->N >= kPersistPrefetchMinRows ? kPersistPrefetchRows : 0));
  // PERSISTENT on a matrix without the band form runs as GRAPH.
  const bool graph_loop =
      (o.loop == CGX_LOOP_GRAPH || o.loop == CGX_LOOP_PERSISTENT ||
       o.loop == CGX_LOOP_PERSISTENT_SPLIT) &&
      !persist;
  auto outer_update = [&] {
    if (pending)
      k_outer_update_pending<<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(
          h->N, h->vec[CGX_VECTOR_X], h->d32, h->p32, h->p32b, h->st);
    else
      k_outer_update<<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(
          h->N, h->vec[CGX_VECTOR_X], h->d32, h->st);
    return cudaGetLastError();
  };
  auto guard = [&] {
    k_loop_guard<<<1, 1, 0, h->stream>>>(h->st);
    return cudaGetLastError();
  };
  auto jacobi_start = [&] {
    k_inner_start<<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(
        h->N, h->r64, h->r32, h->d32, h->p32, h->C32, h->st, h->partials,
        ticket(h, kTicketInnerStart), form == InnerForm::kFused ? h->z32 : nullptr);
    return cudaGetLastError();
  };
  GraphEntry *gj = nullptr, *gl = nullptr;
  if (graph_loop) {
    CGX_TRY(build_while_graph(
        h, 300, jacobi_start,
        [&] {
          cudaError_t e = launch_inner_iteration(h);
          return e != cudaSuccess ? e : guard();
        },
        outer_update, &gj));
    if (want_learned)
      CGX_TRY(build_while_graph(
          h, 500, [&] { return launch_learned_start(h); },
          [&] {
            cudaError_t e = launch_learned_iteration(h);
            return e != cudaSuccess ? e : guard();
          },
          outer_update, &gl));
  } else if (o.loop == CGX_LOOP_CHUNKED) {
    CGX_TRY(build_chunk_graph(h, 400, [&] { return launch_inner_iteration(h); }, &gj));
  }
  const unsigned long long cond_j = gj && graph_loop ? gj->cond : 0;
  const unsigned long long cond_l = gl ? gl->cond : 0;

  // ||b||.
  double bnorm = 0;
  {
    k_dot<<<grid_stream(h, h->N), kThreads, 0, s>>>(
        h->N, h->vec[CGX_VECTOR_K], h->vec[CGX_VECTOR_K], h->dot_out,
        h->partials, ticket(h, kTicketDot));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(h->host_scalar, h->dot_out, sizeof(double),
                             cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    bnorm = std::sqrt(h->host_scalar[0]);
  }
  reset_host_state(h, o.max_iterations, o.tolerance, graph_loop, cond_j);
  h->host_st->bnorm = bnorm;
  h->host_st->inner_tol_min = o.inner_tolerance;
  CGX_TRY(push_state(h));

  const bool learned = want_learned;
  double *x = h->vec[CGX_VECTOR_X];
  double *xbak = h->tmp;  // x at the start of the current outer step
  double rel = 0, prev = -1;
  bool failed = false;
  int outer = 0;
  double t_spmv = 0, t_upd = 0, t_dir = 0, t_inner = 0;
  int launches = 0, inner_launches = 0;
  bool timed = false;  // ev[2], ev[3] bracket a persistent launch not yet read
  for (;;) {
    double r2;
    CGX_TRY(true_residual_r2(h, &r2));
    if (timed) {
      float ms = 0;
      CUDA_TRY(cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]));
      t_inner += ms;
      timed = false;
    }
    rel = bnorm > 0 ? std::sqrt(r2) / bnorm : std::sqrt(r2);
    if (outer > 0 && (!std::isfinite(rel) || rel > 0.5 * prev)) {
      // The step failed: undo it; plain FP64 finishes below.
      CUDA_TRY(cudaMemcpyAsync(x, xbak, sizeof(double) * h->N,
                               cudaMemcpyDeviceToDevice, s));
      failed = true;
      rel = prev;
      break;
    }
    if (!(rel > o.tolerance)) break;  // converged (or NaN before any step: stop)
    if (outer >= o.max_outer) break;
    CGX_TRY(pull_state(h));
    if (h->host_st->total_inner >= o.max_iterations) break;
    outer++;
    prev = rel;
    CUDA_TRY(cudaMemcpyAsync(xbak, x, sizeof(double) * h->N,
                             cudaMemcpyDeviceToDevice, s));
    const double tin = std::max(o.inner_tolerance, 0.5 * o.tolerance / rel);
    // Inner tolerance, graph condition and a fresh loop-guard count.
    h->host_st->in_tol = tin;
    h->host_st->body_count = 0;
    h->host_st->cond = learned ? cond_l : cond_j;
    CUDA_TRY(cudaMemcpyAsync(&h->st->in_tol, &h->host_st->in_tol,
                             sizeof(double), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(&h->st->body_count, &h->host_st->body_count,
                             sizeof(int), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(&h->st->cond, &h->host_st->cond,
                             sizeof(unsigned long long), cudaMemcpyHostToDevice, s));
    if (persist) {
      CUDA_TRY(learned ? launch_learned_start(h) : jacobi_start());
      CUDA_TRY(cudaEventRecord(h->ev[2], s));
      CUDA_TRY(launch_inner_persist(h, learned, form));
      CUDA_TRY(cudaEventRecord(h->ev[3], s));
      timed = true;
      inner_launches++;
      CUDA_TRY(outer_update());
    } else if (graph_loop) {
      CUDA_TRY(cudaGraphLaunch(learned ? gl->exec : gj->exec, s));
    } else {
      if (learned) {
        CUDA_TRY(launch_learned_start(h));
      } else {
        CUDA_TRY(jacobi_start());
      }
      if (o.loop == CGX_LOOP_KERNELS) {
        // kChunk iterations per host wait; their kernels skip once the
        // inner loop stopped.
        CGX_TRY(ensure_event_pool(h));
        int counted = h->host_st->total_inner;
        const int maxChunks = o.max_iterations / kChunk + 2;
        for (int c = 0; c < maxChunks; c++) {
          for (int j = 0; j < kChunk; j++) {
            if (learned)
              CUDA_TRY(launch_learned_iteration(h, &h->evpool[4 * j]));
            else
              CUDA_TRY(launch_inner_iteration(h, &h->evpool[4 * j]));
          }
          CGX_TRY(pull_state(h));
          const int now = h->host_st->total_inner;
          CUDA_TRY(add_segments(h, now - counted, t_spmv, t_upd, t_dir));
          launches += now - counted;
          counted = now;
          if (h->host_st->in_stop) break;
        }
      } else {
        const int maxLaunches = o.max_iterations + 2;
        for (int l = 0; l < maxLaunches; l++) {
          if (learned)
            CUDA_TRY(launch_learned_iteration(h, nullptr));
          else
            CUDA_TRY(cudaGraphLaunch(gj->exec, s));
          CUDA_TRY(cudaMemcpyAsync(h->host_scalar, &h->st->in_stop, sizeof(int),
                                   cudaMemcpyDeviceToHost, s));
          CUDA_TRY(cudaStreamSynchronize(s));
          if (*(int *)h->host_scalar) break;
        }
      }
      CUDA_TRY(outer_update());
    }
  }
  CUDA_TRY(cudaEventRecord(h->ev[7], s));
  CGX_TRY(pull_state(h));
  CGX_TRY(device_errors(h));
  float ms = 0;
  CUDA_TRY(cudaEventElapsedTime(&ms, h->ev[6], h->ev[7]));
  res.solve_ms = ms;
  res.iterations = h->host_st->total_inner;
  if (failed) {
    // Plain FP64 Jacobi-CG from the restored x. Its tolerance is relative to
    // the residual it starts from (rel = ||b - A x|| / ||b|| there), with a
    // factor 2 of margin for the drift between its recurrence residual and
    // the true one; the FP64 true residual is taken again afterwards.
    cgx_options fo = o;
    fo.precision = CGX_PRECISION_FP64;
    fo.preconditioner = CGX_PRECONDITIONER_JACOBI;
    fo.tolerance = 0.5 * o.tolerance / rel;
    cgx_result fr;
    std::memset(&fr, 0, sizeof(fr));
    CGX_TRY(solve_fp64(h, fo, fr));
    double r2;
    CGX_TRY(true_residual_r2(h, &r2));
    rel = bnorm > 0 ? std::sqrt(r2) / bnorm : std::sqrt(r2);
    res.fell_back = 1;
    res.iterations += fr.iterations;
    res.solve_ms += fr.solve_ms;
  }
  res.outer_iterations = outer;
  res.residual = rel;
  res.true_residual = rel;
  res.converged = rel <= o.tolerance;
  res.spmv_ms = t_spmv;
  res.update_ms = t_upd;
  res.direction_ms = t_dir;
  res.spmv_launches = res.update_launches = res.direction_launches = launches;
  res.inner_form = form == InnerForm::kFused ? 1
                   : form == InnerForm::kSplit ? 2
                   : form == InnerForm::kSell  ? 3
                                               : 0;
  res.inner_launches = inner_launches;
  res.inner_ms = t_inner;
  return CGX_SUCCESS;
}

// ---------------------------------------------------------------------------
// Learned preconditioner

namespace {

using namespace cgx::learned;

template <typename T>
size_t take_n(Carver &c, size_t n) {
  return c.take<T>(n + kPad);
}

int grid_for(const cgx_handle *h, size_t work) { return grid_stream(h, work); }

// Exclusive scan of in[0..n) into out[0..n] (out[n] = total).
cudaError_t scan(cgx_handle *h, int n, const int *in, int *out, int *sums) {
  const int nb = (n + kScanBlock - 1) / kScanBlock;
  k_scan_blocks<<<nb, kScanBlock, 0, h->stream>>>(n, in, out, sums);
  k_scan_sums<<<1, kScanBlock, 0, h->stream>>>(nb, sums);
  k_scan_add<<<nb, kScanBlock, 0, h->stream>>>(n, out, sums);
  return cudaGetLastError();
}

cgx_status learned_alloc(cgx_handle *h, int nnzL) {
  Learned *L = h->L;
  const int N = h->N;
  Carver c;
  size_t o_dis = take_n<double>(c, N), o_ahat = take_n<float>(c, h->nz);
  size_t o_feat = take_n<float>(c, (size_t)N * NIN);
  size_t o_nlow = take_n<int>(c, N), o_nup = take_n<int>(c, N);
  size_t o_sums = take_n<int>(c, L->nblocks), o_flag = take_n<int>(c, 4);
  size_t o_gptr = take_n<int>(c, N + 1), o_tptr = take_n<int>(c, N + 1);
  size_t o_gcol = take_n<int>(c, nnzL), o_grow = take_n<int>(c, nnzL);
  size_t o_g2a = take_n<int>(c, nnzL), o_tcol = take_n<int>(c, nnzL);
  size_t o_t2g = take_n<int>(c, nnzL), o_g2t = take_n<int>(c, nnzL);
  size_t o_ghat = take_n<float>(c, nnzL), o_gs = take_n<float>(c, nnzL);
  size_t o_gts = take_n<float>(c, nnzL);
  size_t o_h[4];
  for (int k = 0; k < 4; k++) o_h[k] = take_n<__nv_bfloat16>(c, (size_t)N * W);
  size_t o_o = take_n<float>(c, (size_t)N * NOUT);
  size_t o_y = take_n<float>(c, N), o_z = take_n<float>(c, N);
  CUDA_TRY(dev_alloc(h, (void **)&L->mem, c.off));
  CUDA_TRY(cudaMemsetAsync(L->mem, 0, c.off, h->stream));
  char *b = (char *)L->mem;
  L->dis = (double *)(b + o_dis);
  L->ahat = (float *)(b + o_ahat);
  L->feat = (float *)(b + o_feat);
  L->nlow = (int *)(b + o_nlow);
  L->nup = (int *)(b + o_nup);
  L->sums = (int *)(b + o_sums);
  L->flag = (int *)(b + o_flag);
  L->gptr = (int *)(b + o_gptr);
  L->tptr = (int *)(b + o_tptr);
  L->gcol = (int *)(b + o_gcol);
  L->grow = (int *)(b + o_grow);
  L->g2a = (int *)(b + o_g2a);
  L->tcol = (int *)(b + o_tcol);
  L->t2g = (int *)(b + o_t2g);
  L->g2t = (int *)(b + o_g2t);
  L->ghat = (float *)(b + o_ghat);
  L->gs = (float *)(b + o_gs);
  L->gts = (float *)(b + o_gts);
  for (int k = 0; k < 4; k++) L->h[k] = (__nv_bfloat16 *)(b + o_h[k]);
  L->o = (float *)(b + o_o);
  L->y32 = (float *)(b + o_y);
  L->z32 = (float *)(b + o_z);
  return CGX_SUCCESS;
}

cgx_status learned_train_alloc(cgx_handle *h) {
  Learned *L = h->L;
  if (L->train) return CGX_SUCCESS;
  const int N = h->N;
  Carver c;
  size_t o[20];
  int k = 0;
  for (int q = 0; q < 7; q++) o[k++] = take_n<float>(c, (size_t)N * S);
  o[k++] = take_n<float>(c, L->nnzL);                 // dg
  o[k++] = take_n<float>(c, (size_t)N * NOUT);        // dO
  for (int q = 0; q < 5; q++) o[k++] = take_n<float>(c, (size_t)N * W);
  o[k++] = take_n<float>(c, (size_t)kMaxGrid * (W * 2 * W + W));  // partial
  o[k++] = take_n<float>(c, NPARAMS);                 // grad
  o[k++] = take_n<float>(c, 4);                       // loss
  o[k++] = take_n<float>(c, 2 * (W * W + W));         // gtmp
  o[k++] = take_n<double>(c, 1);                      // snap_scale
  size_t o_agg[3], o_pre[4];
  for (int q = 0; q < 3; q++) o_agg[q] = take_n<__nv_bfloat16>(c, (size_t)N * W);
  for (int q = 0; q < 4; q++) o_pre[q] = take_n<float>(c, (size_t)N * W);
  CUDA_TRY(dev_alloc(h, (void **)&L->train, c.off));
  CUDA_TRY(cudaMemsetAsync(L->train, 0, c.off, h->stream));
  char *b = (char *)L->train;
  k = 0;
  L->V = (float *)(b + o[k++]);
  L->T1 = (float *)(b + o[k++]);
  L->T2 = (float *)(b + o[k++]);
  L->rho = (float *)(b + o[k++]);
  L->dT2 = (float *)(b + o[k++]);
  L->dT1 = (float *)(b + o[k++]);
  L->snap = (float *)(b + o[k++]);
  L->dg = (float *)(b + o[k++]);
  L->dO = (float *)(b + o[k++]);
  L->dh = (float *)(b + o[k++]);
  L->dh2 = (float *)(b + o[k++]);
  L->dself = (float *)(b + o[k++]);
  L->dagg = (float *)(b + o[k++]);
  L->dpre = (float *)(b + o[k++]);
  L->partial = (float *)(b + o[k++]);
  L->grad = (float *)(b + o[k++]);
  L->loss = (float *)(b + o[k++]);
  L->gtmp = (float *)(b + o[k++]);
  L->snap_scale = (double *)(b + o[k++]);
  for (int q = 0; q < 3; q++) L->agg[q] = (__nv_bfloat16 *)(b + o_agg[q]);
  for (int q = 0; q < 4; q++) L->pre[q] = (float *)(b + o_pre[q]);
  return CGX_SUCCESS;
}

// SELL-U layout of the CRS pattern (ptr, col) with nnz entries into S
// (sell.cuh). S.ok stays false when its value slots or offsets would not fit
// in int; the callers then keep their CRS kernels.
cgx_status build_sellu(cgx_handle *h, const int *ptr, const int *col,
                       size_t nnz, SellU &S) {
  sellu_free(h, S);
  const int N = h->N;
  const int nsl = (N + 31) / 32;
  cudaStream_t s = h->stream;
  Carver c;
  size_t o_wd = take_n<int>(c, nsl);
  size_t o_vc = take_n<int>(c, nsl), o_oc = take_n<int>(c, nsl);
  size_t o_un = take_n<int>(c, nsl), o_vb = take_n<int>(c, nsl + 1);
  size_t o_ob = take_n<int>(c, nsl + 1);
  size_t o_sm = take_n<int>(c, nsl / kScanBlock + 1);
  size_t o_tot = take_n<unsigned long long>(c, 4);
  void *tmp = nullptr;
  CUDA_TRY(dev_alloc(h, (void **)&tmp, c.off));
  char *t = (char *)tmp;
  int *wd = (int *)(t + o_wd);
  int *vc = (int *)(t + o_vc), *oc = (int *)(t + o_oc), *un = (int *)(t + o_un);
  int *vb = (int *)(t + o_vb), *ob = (int *)(t + o_ob), *sm = (int *)(t + o_sm);
  unsigned long long *tot = (unsigned long long *)(t + o_tot);
  auto fail_free = [&](cudaError_t e) {
    dev_free(h, tmp);
    return fail(CGX_ERROR_CUDA, cudaGetErrorString(e));
  };
  cudaError_t e = cudaMemsetAsync(tot, 0, 4 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return fail_free(e);
  const int wgrid = grid_stream(h, (size_t)nsl * 32);
  k_sellu_plan<<<wgrid, kThreads, 0, s>>>(N, ptr, col, wd, vc, oc, un, tot);
  unsigned long long ht[4] = {0, 0, 0, 0};
  if ((e = cudaGetLastError()) != cudaSuccess ||
      (e = cudaMemcpyAsync(ht, tot, sizeof(ht), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return fail_free(e);
  // Value slots: 128 per group.
  if (128 * ht[0] + 128 >= (unsigned long long)INT_MAX || ht[1] >= (unsigned long long)INT_MAX) {
    dev_free(h, tmp);
    return CGX_SUCCESS;
  }
  Carver d;
  size_t o_meta = take_n<int4>(d, nsl), o_off = take_n<int>(d, ht[1]);
  size_t o_map = take_n<int>(d, nnz);
  if ((e = scan(h, nsl, vc, vb, sm)) != cudaSuccess ||
      (e = scan(h, nsl, oc, ob, sm)) != cudaSuccess ||
      (e = dev_alloc(h, (void **)&S.mem, d.off)) != cudaSuccess ||
      (e = cudaMemsetAsync(S.mem, 0, d.off, s)) != cudaSuccess)
    return fail_free(e);
  char *b = (char *)S.mem;
  S.meta = (int4 *)(b + o_meta);
  S.off = (int *)(b + o_off);
  S.map = (int *)(b + o_map);
  k_sellu_fill<<<wgrid, kThreads, 0, s>>>(N, ptr, col, vb, ob, wd, un, S.meta,
                                          S.off, S.map);
  if ((e = cudaGetLastError()) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return fail_free(e);
  dev_free(h, tmp);
  S.max_width = (int)ht[3];
  S.slots = 128 * (size_t)ht[0];
  S.uniform = (long long)ht[2];
  S.ok = true;
  return CGX_SUCCESS;
}

// SELL-U layouts of G and G^T with their BF16 value arrays (zero padding;
// k_assemble writes the values through the maps).
cgx_status build_sell(cgx_handle *h) {
  Learned *L = h->L;
  L->sell_ok = false;
  L->gb_ok = false;
  if (L->gb_mem) dev_free(h, L->gb_mem);
  L->gb_mem = nullptr;
  // The band copy when A's offsets fit it.
  Band plan;
  CGX_TRY(band_plan(h, plan));
  // The slot map holds 4 i + k in an int.
  if (plan.K > 0 && (size_t)h->N * kBandMaxK <= (size_t)INT_MAX) {
    const int N = h->N;
    Carver c;
    size_t o_v = take_n<__nv_bfloat16>(c, (size_t)N * kBandMaxK);
    size_t o_m = take_n<int>(c, (size_t)L->nnzL);
    CUDA_TRY(dev_alloc(h, (void **)&L->gb_mem, c.off));
    L->gb_val = (__nv_bfloat16 *)((char *)L->gb_mem + o_v);
    L->g2b = (int *)((char *)L->gb_mem + o_m);
    BandOffsets o{};
    o.K = plan.K;
    for (int k = 0; k < kBandMaxK; k++) {
      o.d[k] = plan.d[k];
      L->gb_d[k] = k < plan.K ? plan.d[k] : 0;
    }
    CUDA_TRY(cudaMemsetAsync(L->gb_mem, 0, c.off, h->stream));
    CUDA_TRY(cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream));
    k_gband_map<<<grid_stream(h, L->nnzL), kThreads, 0, h->stream>>>(
        L->nnzL, L->grow, L->gcol, o, L->g2b, h->flag);
    CUDA_TRY(cudaGetLastError());
    int flag = 0;
    CUDA_TRY(cudaMemcpyAsync(&flag, h->flag, sizeof(int), cudaMemcpyDeviceToHost,
                             h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (flag == 0) {
      L->gb_ok = true;
      return CGX_SUCCESS;
    }
    dev_free(h, L->gb_mem);
    L->gb_mem = nullptr;
  }
  CGX_TRY(build_sellu(h, L->gptr, L->gcol, (size_t)L->nnzL, L->sg));
  CGX_TRY(build_sellu(h, L->tptr, L->tcol, (size_t)L->nnzL, L->st));
  if (!L->sg.ok || !L->st.ok) return CGX_SUCCESS;
  Carver c;
  size_t o_g = take_n<__nv_bfloat16>(c, L->sg.slots);
  size_t o_t = take_n<__nv_bfloat16>(c, L->st.slots);
  if (L->sell_val) dev_free(h, L->sell_val);
  L->sell_val = nullptr;
  CUDA_TRY(dev_alloc(h, (void **)&L->sell_val, c.off));
  CUDA_TRY(cudaMemsetAsync(L->sell_val, 0, c.off, h->stream));
  L->sg_val = (__nv_bfloat16 *)((char *)L->sell_val + o_g);
  L->st_val = (__nv_bfloat16 *)((char *)L->sell_val + o_t);
  L->sell_ok = true;
  return CGX_SUCCESS;
}

// Forward pass of the network on h's scaled graph; writes Ghat (and the
// scaled G, G^T for the apply when `scaled`).
cudaError_t gnn_forward(cgx_handle *h, const float *P, bool scaled) {
  Learned *L = h->L;
  const int N = h->N;
  cudaStream_t s = h->stream;
  // Inference (scaled) keeps no pre-activations or aggregates: only the
  // backward pass needs them.
  const bool keep = !scaled;
  k_embed<<<grid_for(h, (size_t)N), kThreads, 0, s>>>(
      N, L->feat, P, L->h[0], keep ? L->pre[0] : nullptr);
  const int groups = (N + 15) / 16;
  const int lgrid = std::max(
      1, std::min(h->num_sms * 8, (groups + kLayerWarps - 1) / kLayerWarps));
  for (int l = 0; l < 3; l++)
    k_layer<<<lgrid, 32 * kLayerWarps, 0, s>>>(N, h->ptr, h->index, L->ahat, P,
                                               l, L->h[l], L->h[l + 1],
                                               keep ? L->agg[l] : nullptr,
                                               keep ? L->pre[l + 1] : nullptr);
  k_head<<<grid_for(h, (size_t)N), kThreads, 0, s>>>(N, L->h[3], P, L->o);
  k_assemble<<<grid_for(h, L->nnzL), kThreads, 0, s>>>(
      L->nnzL, L->grow, L->gcol, L->g2a, L->ahat, L->o, L->ghat, L->dis,
      L->g2t, scaled ? L->gs : nullptr, scaled ? L->gts : nullptr,
      scaled && L->sell_ok ? L->sg_val : nullptr,
      scaled && L->sell_ok ? L->st_val : nullptr, L->sg.map, L->st.map,
      scaled && L->gb_ok ? L->gb_val : nullptr, L->g2b);
  return cudaGetLastError();
}

// Loss and gradient (into L->grad) for the probes in L->V.
cudaError_t gnn_backward(cgx_handle *h, const float *P) {
  Learned *L = h->L;
  const int N = h->N;
  cudaStream_t s = h->stream;
  const int g = grid_for(h, N);
  // T1 = Ghat V, T2 = Ahat T1, R = Ghat^T T2 - V.
  k_spmm8<<<g, kThreads, 0, s>>>(N, L->gptr, L->gcol, L->ghat, nullptr, L->V, L->T1);
  k_spmm8<<<g, kThreads, 0, s>>>(N, h->ptr, h->index, L->ahat, nullptr, L->T1, L->T2);
  k_loss_residual<<<g, kThreads, 0, s>>>(N, L->tptr, L->tcol, L->ghat, L->t2g,
                                         L->T2, L->V, L->rho, h->partials,
                                         ticket(h, kTicketDot), L->loss);
  // dT2 = Ghat rho, dT1 = Ahat dT2, dGhat.
  k_spmm8<<<g, kThreads, 0, s>>>(N, L->gptr, L->gcol, L->ghat, nullptr, L->rho, L->dT2);
  k_spmm8<<<g, kThreads, 0, s>>>(N, h->ptr, h->index, L->ahat, nullptr, L->dT2, L->dT1);
  k_grad_factor<<<g, kThreads, 0, s>>>(N, L->gptr, L->gcol, L->T2, L->dT1, L->rho,
                                       L->V, L->dg);
  k_grad_head_out<<<g, kThreads, 0, s>>>(N, L->gptr, L->gcol, L->g2a, L->tptr,
                                         L->tcol, L->t2g, L->ahat, L->o, L->dg,
                                         L->dO);
  const int pg = std::max(1, std::min(kMaxGrid, (N + 31) / 32));
  // Head weights: dW_h = sum dO h3^T, db_h = sum dO.
  k_outer_partials<NOUT, W, __nv_bfloat16><<<pg, kThreads, 0, s>>>(
      N, L->dO, L->h[3], L->partial);
  k_reduce_partials<<<grid_for(h, NOUT * W + NOUT), kThreads, 0, s>>>(
      pg, NOUT * W + NOUT, L->partial, L->grad + OFF_WH);
  k_grad_head_in<<<grid_for(h, (size_t)N * W), kThreads, 0, s>>>(N, P, L->dO, L->dh);
  // Layers 2..0.
  float *dcur = L->dh, *dnext = L->dh2;
  for (int l = 2; l >= 0; l--) {
    k_layer_back1<<<grid_for(h, (size_t)N * W), kThreads, 0, s>>>(
        N, P, l, dcur, L->pre[l + 1], L->dpre, L->dself, L->dagg);
    // dW_l[:, 0:W] = sum dpre h_l^T (+ bias), dW_l[:, W:2W] = sum dpre agg^T.
    k_outer_partials<W, W, __nv_bfloat16><<<pg, kThreads, 0, s>>>(
        N, L->dpre, L->h[l], L->partial);
    k_reduce_partials<<<grid_for(h, W * W + W), kThreads, 0, s>>>(
        pg, W * W + W, L->partial, L->gtmp);
    k_outer_partials<W, W, __nv_bfloat16><<<pg, kThreads, 0, s>>>(
        N, L->dpre, L->agg[l], L->partial);
    k_reduce_partials<<<grid_for(h, W * W + W), kThreads, 0, s>>>(
        pg, W * W + W, L->partial, L->gtmp + (W * W + W));
    k_pack_layer_grad<<<1, kThreads, 0, s>>>(L->gtmp, L->grad + OFF_L0 + l * L_STRIDE);
    k_layer_back2<<<grid_for(h, (size_t)N * 32), kThreads, 0, s>>>(
        N, h->ptr, h->index, L->ahat, L->dself, L->dagg, dnext);
    std::swap(dcur, dnext);
  }
  // Embedding.
  k_relu_back<<<grid_for(h, (size_t)N * W), kThreads, 0, s>>>(N * W, L->pre[0], dcur);
  k_outer_partials<W, NIN, float><<<pg, kThreads, 0, s>>>(N, dcur, L->feat,
                                                          L->partial);
  k_reduce_partials<<<grid_for(h, W * NIN + W), kThreads, 0, s>>>(
      pg, W * NIN + W, L->partial, L->grad + OFF_WIN);
  return cudaGetLastError();
}

}  // namespace

static cgx_status ensure_rows(cgx_handle *h) {
  if (h->format == CGX_FORMAT_CRS || h->format == CGX_FORMAT_COO) return CGX_SUCCESS;
  if (h->format != CGX_FORMAT_ELL)
    return fail(CGX_ERROR_INVALID_STATE, "no matrix has been uploaded");
  if (h->rows_mem) return CGX_SUCCESS;
  // Row i's slots j < length[i] in slot order (the reference's ELL keeps a
  // row's CRS order in its slots, Matrix.cpp:339-361). The row pointers come
  // first: the total sizes the index and value arrays.
  const int N = h->N;
  const int nb = (N + cgx::learned::kScanBlock - 1) / cgx::learned::kScanBlock;
  Carver c;
  const size_t o_ptr = c.take<int>((size_t)N + 1 + kPad), o_sums = c.take<int>((size_t)nb);
  void *pmem = nullptr;
  CUDA_TRY(dev_alloc(h, &pmem, c.off));
  int *ptr = (int *)((char *)pmem + o_ptr);
  std::vector<int> hptr((size_t)N + 1);
  cudaError_t e = scan(h, N, h->ell_length, ptr, (int *)((char *)pmem + o_sums));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hptr.data(), ptr, sizeof(int) * ((size_t)N + 1),
                        cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    dev_free(h, pmem);
    CUDA_TRY(e);
  }
  const size_t nz = (size_t)hptr[N];
  Carver d;
  const size_t q_ptr = d.take<int>((size_t)N + 1 + kPad), q_idx = d.take<int>(nz + kPad);
  const size_t q_val = d.take<double>(nz + kPad);
  e = dev_alloc(h, &h->rows_mem, d.off);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->rows_mem, 0, d.off, h->stream);
  char *base = (char *)h->rows_mem;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + q_ptr, ptr, sizeof(int) * ((size_t)N + 1),
                        cudaMemcpyDeviceToDevice, h->stream);
  if (e == cudaSuccess) {
    k_ell_to_rows<<<grid_stream(h, N), kThreads, 0, h->stream>>>(
        N, h->ell_width, h->ell_length, h->ell_index, h->ell_data,
        (const int *)(base + q_ptr), (int *)(base + q_idx), (double *)(base + q_val));
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  dev_free(h, pmem);
  CUDA_TRY(e);
  h->ptr = (int *)(base + q_ptr);
  h->index = (int *)(base + q_idx);
  h->value = (double *)(base + q_val);
  set_tile_caps(h, hptr.data(), N);
  return CGX_SUCCESS;
}

extern "C" {

int cgx_gnn_param_count(void) { return NPARAMS; }

cgx_status cgx_gnn_create(cgx_gnn **out, int device, const float *params) {
  if (!out) return fail(CGX_ERROR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  int n = 0;
  cgx_device_count(&n);
  if (device < 0 || device >= n)
    return fail(CGX_ERROR_INVALID_ARGUMENT, "no CUDA device " + std::to_string(device));
  DeviceGuard guard(device);
  cgx_gnn *g = new cgx_gnn();
  g->device = device;
  cudaError_t e = cudaMalloc(&g->params, sizeof(float) * 3 * NPARAMS);
  if (e != cudaSuccess) {
    delete g;
    return cuda_fail(e, "cudaMalloc (network parameters)");
  }
  g->m = g->params + NPARAMS;
  g->v = g->params + 2 * NPARAMS;
  e = cudaMemset(g->params, 0, sizeof(float) * 3 * NPARAMS);
  if (e == cudaSuccess && params)
    e = cudaMemcpy(g->params, params, sizeof(float) * NPARAMS,
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(g->params);
    delete g;
    return cuda_fail(e, "network parameter upload");
  }
  *out = g;
  return CGX_SUCCESS;
}

cgx_status cgx_gnn_destroy(cgx_gnn *g) {
  if (!g) return CGX_SUCCESS;
  DeviceGuard guard(g->device);
  cudaFree(g->params);
  delete g;
  return CGX_SUCCESS;
}

cgx_status cgx_gnn_set_params(cgx_gnn *g, const float *params) {
  if (!g || !params) return fail(CGX_ERROR_INVALID_ARGUMENT, "NULL argument");
  DeviceGuard guard(g->device);
  CUDA_TRY(cudaMemcpy(g->params, params, sizeof(float) * NPARAMS,
                      cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemset(g->m, 0, sizeof(float) * 2 * NPARAMS));
  g->step = 0;
  return CGX_SUCCESS;
}

cgx_status cgx_gnn_get_params(cgx_gnn *g, float *params) {
  if (!g || !params) return fail(CGX_ERROR_INVALID_ARGUMENT, "NULL argument");
  DeviceGuard guard(g->device);
  CUDA_TRY(cudaMemcpy(params, g->params, sizeof(float) * NPARAMS,
                      cudaMemcpyDeviceToHost));
  return CGX_SUCCESS;
}

cgx_status cgx_update_crs_values(cgx_handle *h, const double *value) {
  CGX_TRY(need_matrix(h));
  if (h->format != CGX_FORMAT_CRS)
    return fail(CGX_ERROR_INVALID_STATE, "the uploaded matrix is not CRS");
  if (!value && h->nz > 0) return fail(CGX_ERROR_INVALID_ARGUMENT, "value is NULL");
  DeviceGuard guard(h->device);
  if (h->nz > 0)
    CUDA_TRY(cudaMemcpyAsync(h->value, value, sizeof(double) * h->nz,
                             cudaMemcpyDefault, h->stream));
  h->f32_valid = false;
  h->c_valid = false;
  if (h->L) h->L->has_factor = false;
  return CGX_SUCCESS;
}

cgx_status cgx_learned_setup(cgx_handle *h) {
  CGX_TRY(need_matrix(h));
  DeviceGuard guard(h->device);
  CGX_TRY(ensure_rows(h));
  cudaStream_t s = h->stream;
  const int N = h->N;
  const bool fresh = !h->L;
  if (fresh) {
    h->L = new Learned();
    h->L->N = N;
    h->L->nnz = h->nz;
    h->L->nblocks = (N + kScanBlock - 1) / kScanBlock;
  }
  Learned *L = h->L;
  // Pass 1: scaling, features, counts (needs a temporary flag and counts;
  // on a fresh set-up the buffers are sized after the counts are known).
  int *flag = nullptr, *nlow = nullptr, *nup = nullptr;
  double *dis = nullptr;
  float *ahat = nullptr, *feat = nullptr;
  void *tmp = nullptr;
  if (fresh) {
    Carver c;
    size_t o_dis = c.take<double>(N + kPad), o_ahat = c.take<float>(h->nz + kPad);
    size_t o_feat = c.take<float>((size_t)N * NIN + kPad);
    size_t o_nl = c.take<int>(N + kPad), o_nu = c.take<int>(N + kPad);
    size_t o_f = c.take<int>(4);
    CUDA_TRY(dev_alloc(h, (void **)&tmp, c.off));
    char *b = (char *)tmp;
    dis = (double *)(b + o_dis);
    ahat = (float *)(b + o_ahat);
    feat = (float *)(b + o_feat);
    nlow = (int *)(b + o_nl);
    nup = (int *)(b + o_nu);
    flag = (int *)(b + o_f);
  } else {
    dis = L->dis; ahat = L->ahat; feat = L->feat;
    nlow = L->nlow; nup = L->nup; flag = L->flag;
  }
  CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), s));
  const int g = grid_stream(h, N);
  k_inv_sqrt_diag<<<g, kThreads, 0, s>>>(N, h->ptr, h->index, h->value, dis, flag);
  k_scaled_rows<<<g, kThreads, 0, s>>>(N, h->ptr, h->index, h->value, dis, ahat,
                                       feat, nlow, nup);
  CUDA_TRY(cudaGetLastError());
  if (!fresh) {
    CUDA_TRY(cudaMemcpyAsync(h->host_scalar, flag, sizeof(int),
                             cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (*(int *)h->host_scalar)
      return fail(CGX_ERROR_UNSUPPORTED,
                  "learned preconditioner: a diagonal entry is missing or not positive");
    L->has_factor = false;
    L->snap_valid = 0;  // snapshots belong to the previous values
    return CGX_SUCCESS;  // pattern unchanged (cgx_update_crs_values)
  }
  // Lower/upper totals.
  {
    // Scan lower counts into a temporary ptr to learn nnzL.
    int nb = L->nblocks;
    int *tptr_tmp = nullptr, *sums_tmp = nullptr;
    Carver c;
    size_t o_p = c.take<int>(N + 1 + kPad), o_s = c.take<int>(nb + kPad);
    void *t2 = nullptr;
    CUDA_TRY(dev_alloc(h, (void **)&t2, c.off));
    tptr_tmp = (int *)((char *)t2 + o_p);
    sums_tmp = (int *)((char *)t2 + o_s);
    CUDA_TRY(scan(h, N, nlow, tptr_tmp, sums_tmp));
    int totals[2] = {0, 0};
    CUDA_TRY(cudaMemcpyAsync(&totals[0], tptr_tmp + N, sizeof(int),
                             cudaMemcpyDeviceToHost, s));
    CUDA_TRY(scan(h, N, nup, tptr_tmp, sums_tmp));
    CUDA_TRY(cudaMemcpyAsync(&totals[1], tptr_tmp + N, sizeof(int),
                             cudaMemcpyDeviceToHost, s));
    int fl = 0;
    CUDA_TRY(cudaMemcpyAsync(&fl, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    dev_free(h, t2);
    if (fl) {
      dev_free(h, tmp);
      free_learned(h);
      return fail(CGX_ERROR_UNSUPPORTED,
                  "learned preconditioner: a diagonal entry is missing or not positive");
    }
    if (totals[0] != totals[1]) {
      dev_free(h, tmp);
      free_learned(h);
      return fail(CGX_ERROR_UNSUPPORTED,
                  "learned preconditioner: the matrix pattern is not symmetric");
    }
    L->nnzL = totals[0];
  }
  cgx_status st = learned_alloc(h, L->nnzL);
  if (st != CGX_SUCCESS) {
    dev_free(h, tmp);
    free_learned(h);
    return st;
  }
  // Move pass-1 results into place, build the patterns and maps.
  CUDA_TRY(cudaMemcpyAsync(L->dis, dis, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(L->ahat, ahat, sizeof(float) * h->nz, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(L->feat, feat, sizeof(float) * N * NIN, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(L->nlow, nlow, sizeof(int) * N, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(L->nup, nup, sizeof(int) * N, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  dev_free(h, tmp);
  CUDA_TRY(scan(h, N, L->nlow, L->gptr, L->sums));
  CUDA_TRY(scan(h, N, L->nup, L->tptr, L->sums));
  k_fill_patterns<<<g, kThreads, 0, s>>>(N, h->ptr, h->index, L->gptr, L->tptr,
                                         L->gcol, L->grow, L->tcol, L->g2a);
  CUDA_TRY(cudaMemsetAsync(L->flag, 0, sizeof(int), s));
  k_transpose_map<<<grid_stream(h, L->nnzL), kThreads, 0, s>>>(
      L->nnzL, L->grow, L->gcol, L->tptr, L->tcol, L->g2t, L->t2g, L->flag);
  CUDA_TRY(cudaGetLastError());
  CGX_TRY(build_sell(h));
  CUDA_TRY(cudaMemcpyAsync(h->host_scalar, L->flag, sizeof(int),
                           cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (*(int *)h->host_scalar) {
    free_learned(h);
    return fail(CGX_ERROR_UNSUPPORTED,
                "learned preconditioner: the matrix pattern is not symmetric");
  }
  drop_graphs(h);  // graphs that use the learned buffers are rebuilt
  return CGX_SUCCESS;
}

cgx_status cgx_learned_factor(cgx_handle *h, cgx_gnn *gn, double eps) {
  CGX_TRY(need_matrix(h));
  if (!gn) return fail(CGX_ERROR_INVALID_ARGUMENT, "network is NULL");
  if (!h->L) return fail(CGX_ERROR_INVALID_STATE, "call cgx_learned_setup first");
  if (gn->device != h->device)
    return fail(CGX_ERROR_INVALID_ARGUMENT, "network and handle on different devices");
  if (!(eps >= 0)) return fail(CGX_ERROR_INVALID_ARGUMENT, "eps must be >= 0");
  DeviceGuard guard(h->device);
  CUDA_TRY(gnn_forward(h, gn->params, true));
  // eps is a kernel argument of the captured inner-solve graphs: a new value
  // needs new graphs (the factor's values are in device memory and need none).
  if (h->L->eps != (float)eps) drop_graphs(h);
  h->L->eps = (float)eps;
  h->L->has_factor = true;
  return CGX_SUCCESS;
}

cgx_status cgx_learned_apply(cgx_handle *h, const float *r, float *z) {
  CGX_TRY(need_matrix(h));
  if (!r || !z) return fail(CGX_ERROR_INVALID_ARGUMENT, "r or z is NULL");
  if (!h->L || !h->L->has_factor)
    return fail(CGX_ERROR_INVALID_STATE, "call cgx_learned_factor first");
  if (!h->c_valid)
    return fail(CGX_ERROR_INVALID_STATE, "Jacobi preconditioner not set");
  DeviceGuard guard(h->device);
  CGX_TRY(ensure_f32(h));
  CGX_TRY(pull_state(h));
  h->host_st->in_stop = 0;
  h->host_st->in_finished = 0;
  h->host_st->use_cond = 0;
  CGX_TRY(push_state(h));
  const size_t bytes = sizeof(float) * (size_t)h->N;
  CUDA_TRY(cudaMemcpyAsync(h->r32, r, bytes, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(launch_learned_apply(h, true));
  CUDA_TRY(cudaMemcpyAsync(z, h->L->z32, bytes, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  CGX_TRY(device_errors(h));
  return CGX_SUCCESS;
}

cgx_status cgx_learned_get_factor(cgx_handle *h, int *nnzL, float *ghat,
                                  int *rows, int *cols) {
  CGX_TRY(need_matrix(h));
  if (!h->L) return fail(CGX_ERROR_INVALID_STATE, "call cgx_learned_setup first");
  DeviceGuard guard(h->device);
  Learned *L = h->L;
  if (nnzL) *nnzL = L->nnzL;
  if (ghat)
    CUDA_TRY(cudaMemcpyAsync(ghat, L->ghat, sizeof(float) * L->nnzL,
                             cudaMemcpyDeviceToHost, h->stream));
  if (rows)
    CUDA_TRY(cudaMemcpyAsync(rows, L->grow, sizeof(int) * L->nnzL,
                             cudaMemcpyDeviceToHost, h->stream));
  if (cols)
    CUDA_TRY(cudaMemcpyAsync(cols, L->gcol, sizeof(int) * L->nnzL,
                             cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CGX_SUCCESS;
}

// Rademacher probes from `seed` into L->V, then the network's smoothing of
// its last columns.
// Columns: [0, S - rc - sc) Rademacher, [S - rc - sc, S - rc) smoothed
// Rademacher, [S - rc, S) the handle's residual snapshots (rc =
// residual_cols, sc = smooth_cols).
static cgx_status make_probes(const cgx_gnn *gn, cgx_handle *h,
                              unsigned long long seed) {
  Learned *L = h->L;
  cudaStream_t s = h->stream;
  const int rc = gn->residual_cols, c1 = S - rc, c0 = c1 - gn->smooth_cols;
  const unsigned need = rc > 0 ? (((1u << rc) - 1u) << c1) : 0u;
  if ((L->snap_valid & need) != need)
    return fail(CGX_ERROR_INVALID_STATE,
                "the probe recipe needs residual snapshots of this matrix "
                "(cgx_learned_capture_residual)");
  const int gs = grid_stream(h, (size_t)h->N * S);
  k_rademacher<<<gs, kThreads, 0, s>>>(h->N, seed, L->V);
  for (int k = 0; k < gn->smooth_steps && c1 > c0; k++) {
    k_spmm8<<<grid_stream(h, h->N), kThreads, 0, s>>>(h->N, h->ptr, h->index,
                                                       L->ahat, nullptr, L->V, L->T1);
    k_smooth_probes<<<gs, kThreads, 0, s>>>(
        h->N, L->V, L->T1, 2.f / 3.f,
        k == gn->smooth_steps - 1 ? gn->smooth_scale : 1.f, c0, c1);
  }
  if (rc > 0) k_copy_probe_cols<<<gs, kThreads, 0, s>>>(h->N, L->snap, L->V, c1);
  CUDA_TRY(cudaGetLastError());
  return CGX_SUCCESS;
}

cgx_status cgx_gnn_set_probes(cgx_gnn *gn, int smooth_steps, int smooth_cols,
                              float smooth_scale, int residual_cols) {
  if (!gn) return fail(CGX_ERROR_INVALID_ARGUMENT, "network is NULL");
  if (smooth_steps < 0 || smooth_cols < 0 || residual_cols < 0 ||
      smooth_cols + residual_cols > S || !(smooth_scale > 0.f))
    return fail(CGX_ERROR_INVALID_ARGUMENT,
                "need smooth_steps >= 0, smooth_cols, residual_cols >= 0 with "
                "smooth_cols + residual_cols <= 8, smooth_scale > 0");
  gn->smooth_steps = smooth_steps;
  gn->smooth_cols = smooth_cols;
  gn->smooth_scale = smooth_scale;
  gn->residual_cols = residual_cols;
  return CGX_SUCCESS;
}

cgx_status cgx_learned_capture_residual(cgx_handle *h, int col) {
  CGX_TRY(need_matrix(h));
  if (!h->L) return fail(CGX_ERROR_INVALID_STATE, "call cgx_learned_setup first");
  if (col < 0 || col >= S) return fail(CGX_ERROR_INVALID_ARGUMENT, "col must be in [0, 8)");
  DeviceGuard guard(h->device);
  CGX_TRY(learned_train_alloc(h));
  Learned *L = h->L;
  cudaStream_t s = h->stream;
  CUDA_TRY(launch_spmv(h, h->vec[CGX_VECTOR_X],
                       OpTrueResidual{h->vec[CGX_VECTOR_K], h->tmp,
                                      ticket(h, kTicketTrue)}));
  const int g = grid_stream(h, h->N);
  k_snap_norm<<<g, kThreads, 0, s>>>(h->N, h->tmp, L->dis, h->partials,
                                     ticket(h, kTicketDot), L->snap_scale);
  k_snap_store<<<g, kThreads, 0, s>>>(h->N, h->tmp, L->dis, L->snap_scale, L->snap, col);
  CUDA_TRY(cudaGetLastError());
  L->snap_valid |= 1u << col;
  return CGX_SUCCESS;
}

cgx_status cgx_gnn_loss_grad(cgx_gnn *gn, cgx_handle *h, const float *probes,
                             unsigned long long seed, float *loss, float *grad) {
  CGX_TRY(need_matrix(h));
  if (!gn) return fail(CGX_ERROR_INVALID_ARGUMENT, "network is NULL");
  if (!h->L) return fail(CGX_ERROR_INVALID_STATE, "call cgx_learned_setup first");
  DeviceGuard guard(h->device);
  CGX_TRY(learned_train_alloc(h));
  Learned *L = h->L;
  cudaStream_t s = h->stream;
  if (probes)
    CUDA_TRY(cudaMemcpyAsync(L->V, probes, sizeof(float) * h->N * S,
                             cudaMemcpyHostToDevice, s));
  else
    CGX_TRY(make_probes(gn, h, seed));
  CUDA_TRY(gnn_forward(h, gn->params, false));
  CUDA_TRY(gnn_backward(h, gn->params));
  if (loss)
    CUDA_TRY(cudaMemcpyAsync(loss, L->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
  if (grad)
    CUDA_TRY(cudaMemcpyAsync(grad, L->grad, sizeof(float) * NPARAMS,
                             cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  L->has_factor = false;  // the factor buffers now hold unscaled values
  return CGX_SUCCESS;
}

cgx_status cgx_gnn_train_step(cgx_gnn *gn, cgx_handle *h, unsigned long long seed,
                              float lr, float *loss) {
  CGX_TRY(need_matrix(h));
  if (!gn) return fail(CGX_ERROR_INVALID_ARGUMENT, "network is NULL");
  if (!h->L) return fail(CGX_ERROR_INVALID_STATE, "call cgx_learned_setup first");
  if (!(lr > 0)) return fail(CGX_ERROR_INVALID_ARGUMENT, "lr must be > 0");
  DeviceGuard guard(h->device);
  CGX_TRY(learned_train_alloc(h));
  Learned *L = h->L;
  cudaStream_t s = h->stream;
  CGX_TRY(make_probes(gn, h, seed));
  CUDA_TRY(gnn_forward(h, gn->params, false));
  CUDA_TRY(gnn_backward(h, gn->params));
  gn->step++;
  k_adam<<<(NPARAMS + kThreads - 1) / kThreads, kThreads, 0, s>>>(
      NPARAMS, gn->params, gn->m, gn->v, L->grad, lr, 0.9f, 0.999f, 1e-8f, gn->step);
  CUDA_TRY(cudaGetLastError());
  if (loss) {
    CUDA_TRY(cudaMemcpyAsync(loss, L->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
  }
  L->has_factor = false;
  return CGX_SUCCESS;
}

}  // extern "C"


extern "C" {

cgx_status cgx_true_residual(cgx_handle *h, double *rel) {
  CGX_TRY(need_matrix(h));
  if (!rel) return fail(CGX_ERROR_INVALID_ARGUMENT, "rel is NULL");
  DeviceGuard guard(h->device);
  cudaStream_t s = h->stream;
  k_dot<<<grid_stream(h, h->N), kThreads, 0, s>>>(
      h->N, h->vec[CGX_VECTOR_K], h->vec[CGX_VECTOR_K], h->dot_out,
      h->partials, ticket(h, kTicketDot));
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(h->host_scalar + 1, h->dot_out, sizeof(double),
                           cudaMemcpyDeviceToHost, s));
  double r2;
  CGX_TRY(true_residual_r2(h, &r2));
  double b2 = h->host_scalar[1];
  *rel = b2 > 0 ? std::sqrt(r2 / b2) : std::sqrt(r2);
  return CGX_SUCCESS;
}

cgx_status cgx_solve(cgx_handle *h, const cgx_options *opts,
                     cgx_result *result) {
  CGX_TRY(need_matrix(h));
  cgx_options o;
  if (opts)
    o = *opts;
  else
    cgx_default_options(&o);
  if (o.max_iterations <= 0)
    return fail(CGX_ERROR_INVALID_ARGUMENT, "max_iterations must be > 0");
  if (!(o.tolerance > 0))
    return fail(CGX_ERROR_INVALID_ARGUMENT, "tolerance must be > 0");
  if (o.preconditioner < CGX_PRECONDITIONER_NONE ||
      o.preconditioner > CGX_PRECONDITIONER_LEARNED ||
      o.precision < CGX_PRECISION_FP64 || o.precision > CGX_PRECISION_MIXED ||
      o.loop < CGX_LOOP_GRAPH || o.loop > CGX_LOOP_PERSISTENT_SPLIT)
    return fail(CGX_ERROR_INVALID_ARGUMENT, "invalid option value");
  if (o.preconditioner == CGX_PRECONDITIONER_LEARNED &&
      o.precision != CGX_PRECISION_MIXED)
    return fail(CGX_ERROR_UNSUPPORTED,
                "the learned preconditioner runs in the mixed-precision solve");
  if (o.precision == CGX_PRECISION_MIXED && !(o.inner_tolerance > 0))
    return fail(CGX_ERROR_INVALID_ARGUMENT, "inner_tolerance must be > 0");
  DeviceGuard guard(h->device);
  cgx_result res;
  std::memset(&res, 0, sizeof(res));
  res.true_residual = -1;
  cgx_status st = o.precision == CGX_PRECISION_MIXED ? solve_mixed(h, o, res)
                                                     : solve_fp64(h, o, res);
  if (st != CGX_SUCCESS) return st;
  if (o.compute_true_residual && o.precision == CGX_PRECISION_FP64)
    CGX_TRY(cgx_true_residual(h, &res.true_residual));
  if (result) *result = res;
  return CGX_SUCCESS;
}

cgx_status cgx_inner_matvec(cgx_handle *h, const float *x, float *y) {
  CGX_TRY(need_matrix(h));
  if (!x || !y) return fail(CGX_ERROR_INVALID_ARGUMENT, "x or y is NULL");
  DeviceGuard guard(h->device);
  CGX_TRY(ensure_rows(h));
  CGX_TRY(ensure_f32(h));
  CGX_TRY(pull_state(h));
  h->host_st->in_stop = 0;
  h->host_st->in_finished = 0;
  h->host_st->use_cond = 0;
  CGX_TRY(push_state(h));
  const size_t bytes = sizeof(float) * (size_t)h->N;
  CUDA_TRY(cudaMemcpyAsync(h->p32, x, bytes, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(launch_inner_q(h));
  CUDA_TRY(cudaMemcpyAsync(y, h->q32, bytes, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  CGX_TRY(device_errors(h));
  return CGX_SUCCESS;
}

cgx_status cgx_check_wait_timeout(cgx_handle *h, int which, int *error_bits) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  if ((which != 0 && which != 1) || !error_bits)
    return fail(CGX_ERROR_INVALID_ARGUMENT, "which must be 0 or 1, error_bits not NULL");
  CGX_TRY(need_matrix(h));
  DeviceGuard guard(h->device);
  CGX_TRY(ensure_rows(h));
  CGX_TRY(ensure_f32(h));
  reset_host_state(h, 1, 0.0, false, 0);
  CGX_TRY(push_state(h));
  CUDA_TRY(cudaMemsetAsync(h->persist_sync, 0, sizeof(unsigned long long), h->stream));
  // Two CTAs, 4096 polls each: a few milliseconds before they give up.
  k_wait_timeout<<<2, 128, 0, h->stream>>>(h->persist_sync, which, 4096u, h->st);
  CUDA_TRY(cudaGetLastError());
  CGX_TRY(pull_state(h));
  *error_bits = h->host_st->error;
  const cgx_status s = device_errors(h);
  // The handle stays usable: the next solve starts from a clean state.
  reset_host_state(h, 1, 0.0, false, 0);
  CGX_TRY(push_state(h));
  return s;
}

cgx_status cgx_time_spmv(cgx_handle *h, cgx_precision precision, int reps,
                         double *us_per_launch) {
  CGX_TRY(need_matrix(h));
  if (reps < 1 || reps > 1000 || !us_per_launch)
    return fail(CGX_ERROR_INVALID_ARGUMENT, "need 1 <= reps <= 1000 and a result pointer");
  if (precision != CGX_PRECISION_FP64 && precision != CGX_PRECISION_MIXED)
    return fail(CGX_ERROR_INVALID_ARGUMENT, "unknown precision");
  DeviceGuard guard(h->device);
  if (precision == CGX_PRECISION_MIXED) {
    CGX_TRY(ensure_rows(h));
    CGX_TRY(ensure_f32(h));
  }
  // The products must not skip: clear the stop flags of the last solve.
  CGX_TRY(pull_state(h));
  h->host_st->stop = 0;
  h->host_st->finished = 0;
  h->host_st->in_stop = 0;
  h->host_st->in_finished = 0;
  h->host_st->use_cond = 0;
  CGX_TRY(push_state(h));
  cudaStream_t s = h->stream;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  for (int r = 0; r < reps && e == cudaSuccess; r++)
    e = precision == CGX_PRECISION_FP64
            ? launch_spmv(h, h->vec[CGX_VECTOR_P],
                          OpPcgQ{h->vec[CGX_VECTOR_P], h->vec[CGX_VECTOR_Q],
                                 ticket(h, kTicketQ)})
            : launch_inner_q(h);
  const cudaError_t ec = cudaStreamEndCapture(s, &graph);
  if (e == cudaSuccess) e = ec;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  float ms = 0;
  if (e == cudaSuccess) e = cudaGraphLaunch(exec, s);  // warm-up
  if (e == cudaSuccess) e = cudaEventRecord(h->ev[0], s);
  if (e == cudaSuccess) e = cudaGraphLaunch(exec, s);
  if (e == cudaSuccess) e = cudaEventRecord(h->ev[1], s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  CUDA_TRY(e);
  CGX_TRY(device_errors(h));
  *us_per_launch = 1000.0 * ms / reps;
  return CGX_SUCCESS;
}

}  // extern "C"
