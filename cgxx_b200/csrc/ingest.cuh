// Device build of the row layout from COO entries.
//
// The reference converts its MatrixCOO on the host: DataMatrix<CRS>::convert
// (Matrix.cpp:203-228) and DataMatrix<ELL>::convert (Matrix.cpp:339-361)
// bucket the entries by row in entry (file) order, and its COO product
// (serial/SerialCG.cpp:79-85) adds a row's products in entry order. Every
// format therefore needs the same thing: the entries grouped by row, each
// row keeping its entries in file order -- a stable sort by row. Here it is
// a least-significant-digit radix sort of (row, entry) pairs on the device:
//
//   - 8 bits per pass, as many passes as N - 1 has significant bits;
//   - per 4096-entry tile, a histogram of the pass's digit (k_sort_hist);
//   - an exclusive scan over (digit, tile), digit-major, so that the tiles
//     of one digit follow each other in input order;
//   - a scatter (k_sort_scatter) in 16 rounds of 256 entries: within a warp,
//     the lanes with the same digit are ranked by __match_any_sync; the
//     warps' per-digit counts go through shared memory in warp order; a
//     running count per digit carries over the rounds. An entry therefore
//     lands after every earlier entry with the same digit: each pass is
//     stable, and so is the sort.
//
// The sorted rows give the row pointers (k_rows_ptr: row r starts at the
// first sorted entry whose row is >= r), and the entry numbers the column
// indices and values (k_rows_gather). The result is bit for bit the
// reference's CRS; the tile-major ELL of the SpMV is built from it
// (k_rows_to_ell).
#pragma once

#include "device.cuh"
#include "kernels.cuh"

namespace cgx {

constexpr int kSortTile = 4096;  // entries per tile: kThreads x 16 rounds
constexpr int kRadix = 256;      // 8-bit digits
static_assert(kThreads == kRadix, "one thread per digit in the scatter");

// *flag |= 1 for a row and |= 2 for a column index outside [0, N).
__global__ void __launch_bounds__(kThreads)
    k_coo_validate(int N, int nz, const int *__restrict__ I,
                   const int *__restrict__ J, int *flag) {
  for (int e = blockIdx.x * kThreads + threadIdx.x; e < nz; e += gridDim.x * kThreads) {
    if ((unsigned)I[e] >= (unsigned)N) atomicOr(flag, 1);
    if ((unsigned)J[e] >= (unsigned)N) atomicOr(flag, 2);
  }
}

// hist[d * ntiles + t] = entries of tile t whose digit (key >> shift) & 255
// is d. One CTA per tile.
__global__ void __launch_bounds__(kThreads)
    k_sort_hist(int n, const int *__restrict__ keys, int shift, int ntiles,
                int *__restrict__ hist) {
  __shared__ int sh[kRadix];
  sh[threadIdx.x] = 0;
  __syncthreads();
  const int start = blockIdx.x * kSortTile;
  const int end = min(n, start + kSortTile);
  for (int i = start + threadIdx.x; i < end; i += kThreads)
    atomicAdd(&sh[(keys[i] >> shift) & (kRadix - 1)], 1);
  __syncthreads();
  hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = sh[threadIdx.x];
}

// Stable scatter of one pass: offs is the exclusive scan of hist. vals_in
// NULL means the entry numbers themselves (the first pass).
__global__ void __launch_bounds__(kThreads)
    k_sort_scatter(int n, const int *__restrict__ keys_in,
                   const int *__restrict__ vals_in, int shift, int ntiles,
                   const int *__restrict__ offs, int *__restrict__ keys_out,
                   int *__restrict__ vals_out) {
  __shared__ int wcnt[kWarps][kRadix + 1];  // column kRadix: empty slots
  __shared__ int run[kRadix];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  run[threadIdx.x] = offs[(size_t)threadIdx.x * ntiles + blockIdx.x];
  const int start = blockIdx.x * kSortTile;
  for (int round = 0; round < kSortTile / kThreads; round++) {
    const int i = start + round * kThreads + threadIdx.x;
    const bool valid = i < n;
    const int key = valid ? keys_in[i] : 0;
    const int d = valid ? (key >> shift) & (kRadix - 1) : kRadix;
    for (int k = threadIdx.x; k < kWarps * (kRadix + 1); k += kThreads)
      (&wcnt[0][0])[k] = 0;
    __syncthreads();
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & below);
    if (rank == 0) wcnt[w][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      int pos = run[d] + rank;
      for (int v = 0; v < w; v++) pos += wcnt[v][d];
      keys_out[pos] = key;
      vals_out[pos] = vals_in ? vals_in[i] : i;
    }
    __syncthreads();
    int t = 0;
    for (int v = 0; v < kWarps; v++) t += wcnt[v][threadIdx.x];
    run[threadIdx.x] += t;
    __syncthreads();
  }
}

// ptr[r] = the first position k whose sorted row is >= r (ptr[N] = nz):
// position k writes the pointers of the rows between its predecessor's row
// and its own, so empty rows get the same pointer as the next non-empty one.
__global__ void __launch_bounds__(kThreads)
    k_rows_ptr(int N, int nz, const int *__restrict__ rows, int *__restrict__ ptr) {
  for (int k = blockIdx.x * kThreads + threadIdx.x; k <= nz; k += gridDim.x * kThreads) {
    const int prev = k > 0 ? rows[k - 1] : -1;
    const int cur = k < nz ? rows[k] : N;
    for (int r = prev + 1; r <= cur; r++) ptr[r] = k;
  }
}

// index[k] = J[e_k], value[k] = V[e_k] for the sorted entry numbers e_k.
__global__ void __launch_bounds__(kThreads)
    k_rows_gather(int nz, const int *__restrict__ order, const int *__restrict__ J,
                  const double *__restrict__ V, int *__restrict__ index,
                  double *__restrict__ value) {
  for (int k = blockIdx.x * kThreads + threadIdx.x; k < nz; k += gridDim.x * kThreads) {
    const int e = order[k];
    index[k] = J[e];
    value[k] = V[e];
  }
}

// *width = the longest row (atomicMax of the row lengths).
__global__ void __launch_bounds__(kThreads)
    k_row_len_max(int N, const int *__restrict__ ptr, int *width) {
  int m = 0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N; i += gridDim.x * kThreads)
    m = max(m, ptr[i + 1] - ptr[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(width, m);
}

// Row layout to the tile-major ELL of the SpMV: row i's entries in slots
// 0 .. len - 1 in storage order, length[i] = len. Padding slots keep the zero
// the caller filled them with.
__global__ void __launch_bounds__(kThreads)
    k_rows_to_ell(int N, int width, const int *__restrict__ ptr,
                  const int *__restrict__ index, const double *__restrict__ value,
                  int *__restrict__ length, int *__restrict__ eidx,
                  double *__restrict__ edat) {
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < N; i += gridDim.x * kThreads) {
    const int j0 = ptr[i], len = ptr[i + 1] - j0;
    length[i] = len;
    for (int j = 0; j < len; j++) {
      eidx[ell_at(i, j, width)] = index[j0 + j];
      edat[ell_at(i, j, width)] = value[j0 + j];
    }
  }
}

// Tile-major ELL back to the reference's column-major arrays (element (i, j)
// at j * N + i; padding slots 0), for the read-back of the layout.
__global__ void __launch_bounds__(kThreads)
    k_ell_columns(int N, int width, const int *__restrict__ length,
                  const int *__restrict__ eidx, const double *__restrict__ edat,
                  int *__restrict__ ci, double *__restrict__ cd) {
  const size_t total = (size_t)N * (size_t)width;
  for (size_t e = (size_t)blockIdx.x * kThreads + threadIdx.x; e < total;
       e += (size_t)gridDim.x * kThreads) {
    const int j = (int)(e / (size_t)N), i = (int)(e - (size_t)j * N);
    const bool used = j < length[i];
    ci[e] = used ? eidx[ell_at(i, j, width)] : 0;
    cd[e] = used ? edat[ell_at(i, j, width)] : 0.0;
  }
}

}  // namespace cgx
