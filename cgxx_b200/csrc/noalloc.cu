// cgx_dot_noalloc: the dot product <a, b> for callers that cannot allocate
// device memory.
//
// Who needs it: code that runs where cudaMalloc is not an option -- inside a
// host framework that owns all device memory through its own pool, in a
// real-time or safety-reviewed loop with a no-allocation rule after start-up,
// or in a process that must not grow its device footprint after
// initialisation. cgx_dot needs a handle, whose creation allocates its
// scratch with cudaMalloc; this entry point takes only the caller's input
// and output buffers and keeps its scratch in a fixed array in the library
// image instead.
//
// Scratch: one FP64 partial sum per 4096-element chunk of the input plus a
// completion counter, in a file-scope __device__ array of kSlots partials
// (512 KiB) that every GPU loading the library holds until the process exits.
// Hence n <= kSlots * kChunk = 268,435,456; larger n is rejected.
//
// The partial of each chunk is summed in a fixed order and the last CTA adds
// the partials in chunk order, so the result depends only on a, b and n (not
// on the GPU's SM count).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "cgx.h"
#include "device.cuh"

void cgx_internal_set_error(const std::string &msg);

namespace {

constexpr int kChunk = 4096;     // elements per CTA (16 per thread)
constexpr int kSlots = 65536;    // partial sums the scratch array holds
constexpr long long kMaxN = (long long)kSlots * kChunk;

// [0, kSlots) partial sums, then the completion counter.
struct NoAllocScratch {
  double partial[kSlots];
  unsigned ticket;
};

static __device__ __align__(256) NoAllocScratch g_scratch;

__global__ void __launch_bounds__(cgx::kThreads)
    k_dot_chunks(int n, const double *__restrict__ a,
                 const double *__restrict__ b, double *out,
                 NoAllocScratch *s) {
  __shared__ double sh[cgx::kWarps];
  __shared__ bool am_last;
  const int base = blockIdx.x * kChunk;
  const int end = min(n, base + kChunk);
  double acc = 0.0;
  for (int i = base + threadIdx.x; i < end; i += cgx::kThreads)
    acc = fma(a[i], b[i], acc);
  acc = cgx::block_sum(acc, sh);
  if (threadIdx.x == 0) {
    s->partial[blockIdx.x] = acc;
    __threadfence();
    am_last = atomicAdd(&s->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double t = 0.0;
  for (int c = threadIdx.x; c < (int)gridDim.x; c += cgx::kThreads)
    t += __ldcg(&s->partial[c]);
  t = cgx::block_sum(t, sh);
  if (threadIdx.x == 0) {
    *out = t;
    s->ticket = 0u;
  }
}

// Device address of g_scratch per device, looked up once per device with
// that device current. In host code the name g_scratch is only a host-side
// stand-in, never a device address. The address is kept until the process
// exits: a cudaDeviceReset may reload the library image elsewhere, and calls
// on that device after a reset are not supported.
std::mutex g_mutex;
constexpr int kMaxDevices = 64;
NoAllocScratch *g_addr[kMaxDevices] = {};

cgx_status scratch_for_current_device(NoAllocScratch **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cgx_internal_set_error("cgx_dot_noalloc: no usable current CUDA device");
    return CGX_ERROR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) {
      cgx_internal_set_error(std::string("CUDA error: ") +
                             cudaGetErrorString(e) +
                             " (cudaGetSymbolAddress of the scratch array)");
      return CGX_ERROR_CUDA;
    }
    g_addr[dev] = static_cast<NoAllocScratch *>(p);
  }
  *out = g_addr[dev];
  return CGX_SUCCESS;
}

}  // namespace

extern "C" cgx_status cgx_dot_noalloc(const double *a, const double *b, int n,
                                      double *result, void *stream) {
  if (n < 0 || (n > 0 && (!a || !b)) || !result) {
    cgx_internal_set_error(
        "cgx_dot_noalloc: need n >= 0, device vectors a and b, and result");
    return CGX_ERROR_INVALID_ARGUMENT;
  }
  if ((long long)n > kMaxN) {
    cgx_internal_set_error(
        "cgx_dot_noalloc: n = " + std::to_string(n) + " exceeds the maximum " +
        std::to_string(kMaxN) + " (65536 partial sums of 4096 elements in "
        "the library's fixed scratch array); use cgx_dot instead");
    return CGX_ERROR_INVALID_ARGUMENT;
  }
  NoAllocScratch *s = nullptr;
  cgx_status st = scratch_for_current_device(&s);
  if (st != CGX_SUCCESS) return st;
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  // The array keeps whatever the previous call left; the counter must start
  // at zero.
  cudaError_t e = cudaMemsetAsync(&s->ticket, 0, sizeof(unsigned), cs);
  if (e == cudaSuccess) {
    if (n == 0) {
      e = cudaMemsetAsync(result, 0, sizeof(double), cs);
    } else {
      const int grid = (n + kChunk - 1) / kChunk;
      k_dot_chunks<<<grid, cgx::kThreads, 0, cs>>>(n, a, b, result, s);
      e = cudaGetLastError();
    }
  }
  if (e != cudaSuccess) {
    cgx_internal_set_error(std::string("CUDA error: ") + cudaGetErrorString(e) +
                           " (cgx_dot_noalloc)");
    return CGX_ERROR_CUDA;
  }
  return CGX_SUCCESS;
}
