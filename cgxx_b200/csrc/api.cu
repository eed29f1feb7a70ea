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
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cgx.h"
#include "kernels.cuh"

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

struct cgx_handle {
  int device = 0;
  int num_sms = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;

  // Matrix.
  int format = -1;
  int N = 0;
  int nz = 0;
  void *mat_mem = nullptr;
  int *ptr = nullptr, *index = nullptr;  // CRS
  double *value = nullptr;
  int tile_cap = 0;
  int *ell_length = nullptr, *ell_index = nullptr;  // ELL
  double *ell_data = nullptr;
  int ell_width = 0;
  int *coo_start = nullptr, *coo_perm = nullptr, *coo_J = nullptr;  // COO
  double *coo_V = nullptr;

  // Vectors K X P Q R Z and Jacobi C.
  void *vec_mem = nullptr;
  double *vec[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  double *C = nullptr;
  double *tmp = nullptr;  // FP64 scratch vector (true residual)
  bool c_valid = false;

  // FP32 mirror and inner vectors of the mixed path (allocated on demand).
  void *f32_mem = nullptr;
  float *value32 = nullptr, *C32 = nullptr;
  float *d32 = nullptr, *r32 = nullptr, *p32 = nullptr, *q32 = nullptr;
  double *r64 = nullptr;
  bool f32_valid = false;

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
};

static void drop_graphs(cgx_handle *h) {
  for (auto &g : h->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
  }
  h->graphs.clear();
}

static void free_matrix(cgx_handle *h) {
  drop_graphs(h);
  if (h->mat_mem) cudaFree(h->mat_mem);
  if (h->vec_mem) cudaFree(h->vec_mem);
  if (h->f32_mem) cudaFree(h->f32_mem);
  h->mat_mem = h->vec_mem = h->f32_mem = nullptr;
  h->format = -1;
  h->N = h->nz = 0;
  h->ptr = h->index = nullptr;
  h->value = nullptr;
  h->ell_length = h->ell_index = nullptr;
  h->ell_data = nullptr;
  h->coo_start = h->coo_perm = h->coo_J = nullptr;
  h->coo_V = nullptr;
  for (auto &v : h->vec) v = nullptr;
  h->C = nullptr;
  h->tmp = nullptr;
  h->c_valid = false;
  h->value32 = h->C32 = h->d32 = h->r32 = h->p32 = h->q32 = nullptr;
  h->r64 = nullptr;
  h->f32_valid = false;
}

// Grid of the streaming (vector) kernels: a few CTAs per SM, enough bytes in
// flight to saturate HBM, never more CTAs than there is work.
static int grid_stream(const cgx_handle *h, size_t work_items) {
  size_t need = (work_items + kThreads - 1) / kThreads;
  size_t g = std::min<size_t>((size_t)h->num_sms * 4, need);
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
      int c = index[(size_t)j * N + i];
      if (c < 0 || c >= N) atomicOr(flag, 2);
    }
  }
}

__global__ void k_validate_coo(int N, int nz, const int *J, int *flag) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nz;
       j += gridDim.x * blockDim.x) {
    int c = J[j];
    if (c < 0 || c >= N) atomicOr(flag, 2);
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

template <typename VT, typename Op>
static cudaError_t launch_crs(cgx_handle *h, const VT *value, int cap,
                              const VT *x, Op op) {
  CrsView<VT> A{h->ptr, h->index, value, h->N, cap};
  const size_t smem = crs_smem_bytes<VT>(cap);
  auto kern = k_crs<VT, Op>;
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

template <typename Op>
static cudaError_t launch_spmv(cgx_handle *h, const double *x, Op op) {
  switch (h->format) {
  case CGX_FORMAT_CRS:
    return launch_crs<double, Op>(h, h->value, h->tile_cap, x, op);
  case CGX_FORMAT_ELL: {
    EllView<double> A{h->ell_length, h->ell_index, h->ell_data, h->N,
                      h->ell_width};
    k_ell<double, Op><<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(
        A, x, op, h->st, h->partials);
    return cudaGetLastError();
  }
  case CGX_FORMAT_COO: {
    CooView A{h->coo_start, h->coo_perm, h->coo_J, h->coo_V, h->N};
    k_coo<Op><<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(
        A, x, op, h->st, h->partials);
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

// Inner FP32 PCG iteration of the mixed path.
static cudaError_t launch_inner_iteration(cgx_handle *h,
                                          cudaEvent_t *evs = nullptr) {
  cudaError_t e;
  if (evs) cudaEventRecord(evs[0], h->stream);
  e = launch_crs<float, OpInnerQ>(
      h, h->value32, h->tile_cap, h->p32,
      OpInnerQ{h->p32, h->q32, ticket(h, kTicketInnerQ)});
  if (e != cudaSuccess) return e;
  if (evs) cudaEventRecord(evs[1], h->stream);
  const int g = grid_stream(h, (size_t)(h->N + 3) / 4);
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
  o->inner_tolerance = 1e-5;
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
  for (auto &ev : h->ev)
    if (ev) cudaEventDestroy(ev);
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
  CUDA_TRY(cudaMalloc(&h->vec_mem, c.off));
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

cgx_status cgx_upload_crs(cgx_handle *h, int N, int nz, const int *ptr,
                          const int *index, const double *value) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  if (N <= 0 || nz < 0 || !ptr || (nz > 0 && (!index || !value)))
    return fail(CGX_ERROR_INVALID_ARGUMENT, "bad CRS sizes or pointers");
  if (ptr[0] != 0 || ptr[N] != nz)
    return fail(CGX_ERROR_INVALID_ARGUMENT,
                "CRS ptr must start at 0 and end at nz");
  DeviceGuard guard(h->device);
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  free_matrix(h);
  // Tile capacity of the staged SpMV: the largest nonzero count of a
  // 256-row tile, bounded so that two stages fit next to each other with
  // several CTAs per SM; larger tiles fall back to direct loads.
  int maxTile = 0;
  for (int r0 = 0; r0 < N; r0 += kThreads) {
    int r1 = std::min(N, r0 + kThreads);
    maxTile = std::max(maxTile, ptr[r1] - ptr[r0]);
  }
  h->tile_cap = std::min(maxTile, 4096);
  Carver c;
  size_t o_ptr = c.take<int>((size_t)N + 1 + kPad);
  size_t o_idx = c.take<int>((size_t)nz + kPad);
  size_t o_val = c.take<double>((size_t)nz + kPad);
  CUDA_TRY(cudaMalloc(&h->mat_mem, c.off));
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
  h->format = CGX_FORMAT_CRS;
  CGX_TRY(alloc_vectors(h, N));
  CUDA_TRY(cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream));
  k_validate_crs<<<grid_stream(h, std::max(N, nz)), kThreads, 0, h->stream>>>(
      N, nz, h->ptr, h->index, h->flag);
  CUDA_TRY(cudaGetLastError());
  return check_flag(h, "CRS");
}

cgx_status cgx_upload_ell(cgx_handle *h, int N, int nz, int maxNz,
                          const int *length, const int *index,
                          const double *data) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  if (N <= 0 || nz < 0 || maxNz < 0 || !length ||
      ((size_t)maxNz * N > 0 && (!index || !data)))
    return fail(CGX_ERROR_INVALID_ARGUMENT, "bad ELL sizes or pointers");
  DeviceGuard guard(h->device);
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  free_matrix(h);
  const size_t elems = (size_t)maxNz * (size_t)N;
  Carver c;
  size_t o_len = c.take<int>((size_t)N + kPad);
  size_t o_idx = c.take<int>(elems + kPad);
  size_t o_dat = c.take<double>(elems + kPad);
  CUDA_TRY(cudaMalloc(&h->mat_mem, c.off));
  char *base = (char *)h->mat_mem;
  h->ell_length = (int *)(base + o_len);
  h->ell_index = (int *)(base + o_idx);
  h->ell_data = (double *)(base + o_dat);
  h->ell_width = maxNz;
  CUDA_TRY(cudaMemsetAsync(h->mat_mem, 0, c.off, h->stream));
  CUDA_TRY(cudaMemcpyAsync(h->ell_length, length, sizeof(int) * (size_t)N,
                           cudaMemcpyHostToDevice, h->stream));
  if (elems > 0) {
    CUDA_TRY(cudaMemcpyAsync(h->ell_index, index, sizeof(int) * elems,
                             cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(h->ell_data, data, sizeof(double) * elems,
                             cudaMemcpyHostToDevice, h->stream));
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

cgx_status cgx_upload_coo(cgx_handle *h, int N, int nz, const int *I,
                          const int *J, const double *V) {
  if (!h) return fail(CGX_ERROR_INVALID_ARGUMENT, "handle is NULL");
  if (N <= 0 || nz < 0 || (nz > 0 && (!I || !J || !V)))
    return fail(CGX_ERROR_INVALID_ARGUMENT, "bad COO sizes or pointers");
  // Row-grouped permutation in entry order (stable counting sort on the
  // host): keeps serial/SerialCG.cpp:79-85's per-row summation order.
  std::vector<int> start((size_t)N + 1, 0), perm((size_t)(nz > 0 ? nz : 1));
  for (int e = 0; e < nz; e++) {
    if (I[e] < 0 || I[e] >= N)
      return fail(CGX_ERROR_INVALID_ARGUMENT,
                  "invalid COO matrix: row index outside [0, N)");
    start[(size_t)I[e] + 1]++;
  }
  for (int i = 0; i < N; i++) start[i + 1] += start[i];
  {
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int e = 0; e < nz; e++) perm[fill[I[e]]++] = e;
  }
  DeviceGuard guard(h->device);
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  free_matrix(h);
  Carver c;
  size_t o_st = c.take<int>((size_t)N + 1 + kPad);
  size_t o_pm = c.take<int>((size_t)nz + kPad);
  size_t o_j = c.take<int>((size_t)nz + kPad);
  size_t o_v = c.take<double>((size_t)nz + kPad);
  CUDA_TRY(cudaMalloc(&h->mat_mem, c.off));
  char *base = (char *)h->mat_mem;
  h->coo_start = (int *)(base + o_st);
  h->coo_perm = (int *)(base + o_pm);
  h->coo_J = (int *)(base + o_j);
  h->coo_V = (double *)(base + o_v);
  CUDA_TRY(cudaMemcpyAsync(h->coo_start, start.data(),
                           sizeof(int) * ((size_t)N + 1),
                           cudaMemcpyHostToDevice, h->stream));
  if (nz > 0) {
    CUDA_TRY(cudaMemcpyAsync(h->coo_perm, perm.data(), sizeof(int) * nz,
                             cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(h->coo_J, J, sizeof(int) * nz,
                             cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(h->coo_V, V, sizeof(double) * nz,
                             cudaMemcpyHostToDevice, h->stream));
  }
  h->N = N;
  h->nz = nz;
  h->format = CGX_FORMAT_COO;
  CGX_TRY(alloc_vectors(h, N));
  CUDA_TRY(cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream));
  k_validate_coo<<<grid_stream(h, nz), kThreads, 0, h->stream>>>(
      N, nz, h->coo_J, h->flag);
  CUDA_TRY(cudaGetLastError());
  // The host vectors above must outlive the asynchronous copies.
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return check_flag(h, "COO");
}

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
  if (h->format != CGX_FORMAT_CRS) {
    // ELL/COO: derive from the host-visible definition through a temporary
    // CRS view is not available; compute on the device per format.
    return fail(CGX_ERROR_UNSUPPORTED,
                "cgx_jacobi_from_matrix supports CRS; upload C for ELL/COO");
  }
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
  return CGX_SUCCESS;
}

static cgx_status solve_fp64(cgx_handle *h, const cgx_options &o,
                             cgx_result &res) {
  const bool jacobi = o.preconditioner == CGX_PRECONDITIONER_JACOBI;
  if (jacobi && !h->c_valid)
    return fail(CGX_ERROR_INVALID_STATE, "Jacobi preconditioner not set");
  cudaStream_t s = h->stream;

  if (o.loop == CGX_LOOP_GRAPH) {
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
  } else if (o.loop == CGX_LOOP_CHUNKED) {
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
    for (; it < o.max_iterations; it++) {
      CUDA_TRY(launch_pcg_iteration(h, jacobi, h->ev));
      CUDA_TRY(cudaMemcpyAsync(h->host_scalar, &h->st->stop, sizeof(int),
                               cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaStreamSynchronize(s));
      float a = 0, b = 0, c = 0;
      CUDA_TRY(cudaEventElapsedTime(&a, h->ev[0], h->ev[1]));
      CUDA_TRY(cudaEventElapsedTime(&b, h->ev[1], h->ev[2]));
      CUDA_TRY(cudaEventElapsedTime(&c, h->ev[2], h->ev[3]));
      t_spmv += a;
      t_upd += b;
      t_dir += c;
      if (*(int *)h->host_scalar) {
        it++;
        break;
      }
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
    size_t o_r64 = c.take<double>((size_t)N + kPad);
    CUDA_TRY(cudaMalloc(&h->f32_mem, c.off));
    CUDA_TRY(cudaMemsetAsync(h->f32_mem, 0, c.off, h->stream));
    char *base = (char *)h->f32_mem;
    h->value32 = (float *)(base + o_v);
    h->C32 = (float *)(base + o_c);
    h->d32 = (float *)(base + o_d);
    h->r32 = (float *)(base + o_r);
    h->p32 = (float *)(base + o_p);
    h->q32 = (float *)(base + o_q);
    h->r64 = (double *)(base + o_r64);
  }
  k_to_f32<<<grid_stream(h, h->nz), kThreads, 0, h->stream>>>(
      (size_t)h->nz, h->value, h->value32);
  CUDA_TRY(cudaGetLastError());
  k_to_f32<<<grid_stream(h, N), kThreads, 0, h->stream>>>((size_t)N, h->C,
                                                          h->C32);
  CUDA_TRY(cudaGetLastError());
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

static cgx_status solve_mixed(cgx_handle *h, const cgx_options &o,
                              cgx_result &res) {
  if (h->format != CGX_FORMAT_CRS)
    return fail(CGX_ERROR_UNSUPPORTED, "mixed precision needs CRS");
  if (o.preconditioner != CGX_PRECONDITIONER_JACOBI)
    return fail(CGX_ERROR_UNSUPPORTED,
                "mixed precision supports the Jacobi preconditioner");
  if (!h->c_valid)
    return fail(CGX_ERROR_INVALID_STATE, "Jacobi preconditioner not set");
  cudaStream_t s = h->stream;
  CUDA_TRY(cudaEventRecord(h->ev[6], s));
  CGX_TRY(ensure_f32(h));

  GraphEntry *ge = nullptr;
  if (o.loop == CGX_LOOP_GRAPH) {
    CGX_TRY(build_while_graph(
        h, 300,
        [&] {
          k_inner_start<<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(
              h->N, h->r64, h->r32, h->d32, h->p32, h->C32, h->st,
              h->partials, ticket(h, kTicketInnerStart));
          return cudaGetLastError();
        },
        [&] {
          cudaError_t e = launch_inner_iteration(h);
          if (e != cudaSuccess) return e;
          k_loop_guard<<<1, 1, 0, h->stream>>>(h->st);
          return cudaGetLastError();
        },
        [&] {
          k_outer_update<<<grid_stream(h, h->N), kThreads, 0, h->stream>>>(
              h->N, h->vec[CGX_VECTOR_X], h->d32, h->st);
          return cudaGetLastError();
        },
        &ge));
  } else if (o.loop == CGX_LOOP_CHUNKED) {
    CGX_TRY(build_chunk_graph(h, 400, [&] { return launch_inner_iteration(h); },
                              &ge));
  }

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
  reset_host_state(h, o.max_iterations, o.tolerance,
                   o.loop == CGX_LOOP_GRAPH, ge && o.loop == CGX_LOOP_GRAPH
                                                 ? ge->cond
                                                 : 0);
  h->host_st->bnorm = bnorm;
  h->host_st->inner_tol_min = o.inner_tolerance;
  CGX_TRY(push_state(h));

  double rel = 0;
  int outer = 0;
  double t_spmv = 0, t_upd = 0, t_dir = 0;
  int launches = 0;
  for (;;) {
    double r2;
    CGX_TRY(true_residual_r2(h, &r2));
    rel = bnorm > 0 ? std::sqrt(r2) / bnorm : std::sqrt(r2);
    if (!(rel > o.tolerance)) break;  // converged (or NaN: stop)
    if (outer >= o.max_outer) break;
    CGX_TRY(pull_state(h));
    if (h->host_st->total_inner >= o.max_iterations) break;
    outer++;
    double tin = std::max(o.inner_tolerance, 0.5 * o.tolerance / rel);
    // Inner tolerance and a fresh loop-guard count for this inner solve.
    h->host_st->in_tol = tin;
    h->host_st->body_count = 0;
    CUDA_TRY(cudaMemcpyAsync(&h->st->in_tol, &h->host_st->in_tol,
                             sizeof(double), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(&h->st->body_count, &h->host_st->body_count,
                             sizeof(int), cudaMemcpyHostToDevice, s));
    if (o.loop == CGX_LOOP_GRAPH) {
      CUDA_TRY(cudaGraphLaunch(ge->exec, s));
    } else {
      k_inner_start<<<grid_stream(h, h->N), kThreads, 0, s>>>(
          h->N, h->r64, h->r32, h->d32, h->p32, h->C32, h->st, h->partials,
          ticket(h, kTicketInnerStart));
      CUDA_TRY(cudaGetLastError());
      const int maxLaunches = o.max_iterations + 2;
      for (int l = 0; l < maxLaunches; l++) {
        if (o.loop == CGX_LOOP_CHUNKED) {
          CUDA_TRY(cudaGraphLaunch(ge->exec, s));
        } else {
          CUDA_TRY(launch_inner_iteration(h, h->ev));
        }
        CUDA_TRY(cudaMemcpyAsync(h->host_scalar, &h->st->in_stop, sizeof(int),
                                 cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        if (o.loop == CGX_LOOP_KERNELS) {
          float a = 0, b = 0, c = 0;
          CUDA_TRY(cudaEventElapsedTime(&a, h->ev[0], h->ev[1]));
          CUDA_TRY(cudaEventElapsedTime(&b, h->ev[1], h->ev[2]));
          CUDA_TRY(cudaEventElapsedTime(&c, h->ev[2], h->ev[3]));
          t_spmv += a;
          t_upd += b;
          t_dir += c;
          launches++;
        }
        if (*(int *)h->host_scalar) break;
      }
      k_outer_update<<<grid_stream(h, h->N), kThreads, 0, s>>>(
          h->N, h->vec[CGX_VECTOR_X], h->d32, h->st);
      CUDA_TRY(cudaGetLastError());
    }
  }
  CUDA_TRY(cudaEventRecord(h->ev[7], s));
  CGX_TRY(pull_state(h));
  CGX_TRY(device_errors(h));
  float ms = 0;
  CUDA_TRY(cudaEventElapsedTime(&ms, h->ev[6], h->ev[7]));
  res.solve_ms = ms;
  res.iterations = h->host_st->total_inner;
  res.outer_iterations = outer;
  res.residual = rel;
  res.true_residual = rel;
  res.converged = rel <= o.tolerance;
  res.spmv_ms = t_spmv;
  res.update_ms = t_upd;
  res.direction_ms = t_dir;
  res.spmv_launches = res.update_launches = res.direction_launches = launches;
  return CGX_SUCCESS;
}

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
      o.loop < CGX_LOOP_GRAPH || o.loop > CGX_LOOP_KERNELS)
    return fail(CGX_ERROR_INVALID_ARGUMENT, "invalid option value");
  if (o.preconditioner == CGX_PRECONDITIONER_LEARNED)
    return fail(CGX_ERROR_UNSUPPORTED,
                "learned preconditioner: use cgx_solve_learned");
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

}  // extern "C"
