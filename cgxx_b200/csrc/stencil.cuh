// Z-marching kernels for the band form of a 3-D 7-point stencil.
//
// When the band offsets of A are those of a grid numbered x fastest
// (d = 0, 1, nx, nx ny), row i is the cell (x, y, z) with
// i = (z ny + y) nx + x. A CTA owns a 32 x 8 tile of the x-y plane (one warp
// per grid line, one lane per cell) and marches through a chunk of planes.
// For each plane a thread loads its own cell's values once (one 16-byte load
// of U, or one 8-byte load of the factor's four values) and the vector
// entries it needs; the x and y neighbours come from shared memory (the
// tile's cells plus a one-cell halo that the edge lanes and warps load), the
// z neighbours from registers (the previous and the next plane of the same
// column). The generic band kernels issue 11 to 12 dependent loads per row;
// these issue 3 plus a few halo loads, so the products are bound by the
// streaming bytes, not by gather latency.
//
// The arithmetic is the generic band kernels' (band.cuh): the same products
// added in the same order, the same masks, so q, y and z are bit-identical
// to theirs for the same inputs. The fused kernels also form the vectors
// they read from the previous iteration's (p = z + b p_old, r = r_old - a q)
// for every cell and halo cell, with the single roundings of the unfused
// updates, and write the new vector to the other buffer of a ping-pong pair
// (the old one is still read by neighbouring tiles).
//
//   k_st_dir:  p = z + b p_old, d += a_old p_old, q = A p, <p,q> -> a
//   k_st_res:  r = r_old - a q, y = G^T r, <r,r> -> residual test (learned)
//   k_st_gz:   z = G y + eps C r, <r,z> -> b (learned; any row epilogue Op)
#pragma once

#include "band.cuh"
#include "kernels.cuh"

namespace cgx {

constexpr int kStX = 32;  // tile width: one lane per cell of a grid line
constexpr int kStY = 8;   // tile height: one warp per grid line

// Grid and work decomposition: tiles_x x tiles_y tiles of the x-y plane,
// each marching over chunks of lz planes; work item b = (chunk ty) tx. The
// per-phase kernels launch one CTA per item; a persistent kernel loops its
// CTAs over the items.
struct StencilGeom {
  int nx, ny, nz;
  int tiles_x, tiles_y, lz;
};

__host__ __device__ inline int st_items(const StencilGeom &g) {
  return g.tiles_x * g.tiles_y * ((g.nz + g.lz - 1) / g.lz);
}

// Loads of vectors: the read-only path in the per-phase kernels, the L2 path
// inside a persistent kernel, where another CTA wrote the value in an
// earlier phase of the same launch and a stale L1 line must not be read.
template <bool CG>
__device__ __forceinline__ float st_ld(const float *p) {
  return CG ? __ldcg(p) : __ldg(p);
}

struct StPos {
  int lane, w;   // cell (lane, w) of the tile
  int col;       // y nx + x of the (clamped) cell
  int z0, z1;    // planes of this CTA's chunk
  bool valid;    // the cell lies inside the grid
  bool xlast, ylast;  // x = nx - 1, y = ny - 1: no neighbour at x + 1, y + 1
};

__device__ __forceinline__ StPos st_pos(const StencilGeom &g, int item) {
  StPos s;
  int b = item;
  const int tx = b % g.tiles_x;
  b /= g.tiles_x;
  const int ty = b % g.tiles_y;
  b /= g.tiles_y;
  s.lane = threadIdx.x & 31;
  s.w = threadIdx.x >> 5;
  const int x = tx * kStX + s.lane, y = ty * kStY + s.w;
  s.valid = x < g.nx && y < g.ny;
  s.xlast = x == g.nx - 1;
  s.ylast = y == g.ny - 1;
  s.col = min(y, g.ny - 1) * g.nx + min(x, g.nx - 1);
  s.z0 = b * g.lz;
  s.z1 = min(g.nz, s.z0 + g.lz);
  return s;
}

// Fused step 1 of a band inner iteration (both mixed paths). See DirArgs
// (band.cuh side: z, pold, pnew, d, q, ticket, pnew_slot).
struct StDirArgs {
  const float *z;     // preconditioned residual
  const float *pold;  // search direction of the last iteration
  float *pnew;        // the new one (other buffer of the pair)
  float *d;           // inner solution: d += a_old p_old
  float *q;           // A p
  unsigned *ticket;
  int pnew_slot;      // which buffer of the pair pnew is (0 or 1)
};

// One work item of k_st_dir: this thread's partial sum of <p,q>.
template <bool CG>
__device__ __forceinline__ double st_dir_item(const StencilGeom &g, const BandView<4> &B,
                                              const StDirArgs &a, float al, float be,
                                              int item) {
  const StPos s = st_pos(g, item);
  const int nx = g.nx, N = B.N, plane = nx * g.ny;
  const float4 *__restrict__ U = reinterpret_cast<const float4 *>(B.U);
  const float *__restrict__ zv = a.z;
  const float *__restrict__ po = a.pold;
  __shared__ float sp[kStY + 2][kStX + 2];  // p of the plane, one-cell halo
  __shared__ float suy[kStY][kStX + 1];     // U.y = A(i, i + 1), left halo
  __shared__ float suz[kStY + 1][kStX];     // U.z = A(i, i + nx), bottom halo
  double acc = 0.0;
  if (s.z0 >= s.z1) return acc;
  int i = s.z0 * plane + s.col;
  // The column below the chunk (nothing below plane 0: masked).
  float p_m = 0.f, lw = 0.f;
  if (s.z0 > 0) {
    p_m = fmaf(be, st_ld<CG>(po + i - plane), st_ld<CG>(zv + i - plane));
    lw = __ldg(&U[i - plane]).w;
  }
  float po_c = st_ld<CG>(po + i);
  float p_c = fmaf(be, po_c, st_ld<CG>(zv + i));
  for (int zz = s.z0; zz < s.z1; zz++, i += plane) {
    const float4 u = __ldg(&U[i]);
    const int in = (int)min((long long)i + plane, (long long)N - 1);  // top plane: u.w = 0
    const float po_n = st_ld<CG>(po + in);
    const float p_n = fmaf(be, po_n, st_ld<CG>(zv + in));
    sp[s.w + 1][s.lane + 1] = p_c;
    suy[s.w][s.lane + 1] = u.y;
    suz[s.w + 1][s.lane] = u.z;
    if (s.lane == 0) {
      const int j = max(i - 1, 0);
      sp[s.w + 1][0] = fmaf(be, st_ld<CG>(po + j), st_ld<CG>(zv + j));
      suy[s.w][0] = __ldg(&U[j]).y;
    }
    if (s.lane == kStX - 1) {
      const int j = min(i + 1, N - 1);
      sp[s.w + 1][kStX + 1] = fmaf(be, st_ld<CG>(po + j), st_ld<CG>(zv + j));
    }
    if (s.w == 0) {
      const int j = max(i - nx, 0);
      sp[0][s.lane + 1] = fmaf(be, st_ld<CG>(po + j), st_ld<CG>(zv + j));
      suz[0][s.lane] = __ldg(&U[j]).z;
    }
    if (s.w == kStY - 1) {
      const int j = min(i + nx, N - 1);
      sp[kStY + 1][s.lane + 1] = fmaf(be, st_ld<CG>(po + j), st_ld<CG>(zv + j));
    }
    __syncthreads();
    const float lv1 = i < 1 ? 0.f : suy[s.w][s.lane];
    const float lv2 = i < nx ? 0.f : suz[s.w][s.lane];
    const float lv3 = i < plane ? 0.f : lw;
    float sum = fmaf(u.x, p_c, 0.f);
    sum = fmaf(u.y, sp[s.w + 1][s.lane + 2], sum);
    sum = fmaf(u.z, sp[s.w + 2][s.lane + 1], sum);
    sum = fmaf(u.w, p_n, sum);
    sum = fmaf(lv1, sp[s.w + 1][s.lane], sum);
    sum = fmaf(lv2, sp[s.w][s.lane + 1], sum);
    sum = fmaf(lv3, p_m, sum);
    if (s.valid) {
      a.d[i] = fmaf(al, po_c, a.d[i]);
      a.pnew[i] = p_c;
      a.q[i] = sum;
      acc = fma((double)p_c, (double)sum, acc);
    }
    __syncthreads();
    p_m = p_c;
    p_c = p_n;
    po_c = po_n;
    lw = u.w;
  }
  return acc;
}

__global__ void __launch_bounds__(kThreads)
    k_st_dir(StencilGeom g, BandView<4> B, StDirArgs a, CgState *st, double *partials) {
  if (st->in_stop) return;
  const float al = (float)st->in_alpha, be = (float)st->in_beta;
  double acc = 0.0;
  for (int item = blockIdx.x; item < st_items(g); item += gridDim.x)
    acc += st_dir_item<false>(g, B, a, al, be, item);
  double in[1] = {acc}, out[1];
  if (grid_reduce<1>(in, partials, a.ticket, out) && threadIdx.x == 0) {
    st->in_alpha = st->in_rho / out[0];
    st->in_pslot = a.pnew_slot;
  }
}

// The learned factor's values of row i (G(i, i), G(i, i-1), G(i, i-nx),
// G(i, i-nx ny)) from the row-major BF16 band copy (one 8-byte load).
__device__ __forceinline__ float4 st_gvals(const __nv_bfloat16 *val, int i) {
  const uint2 raw = __ldg(reinterpret_cast<const uint2 *>(val) + i);
  return make_float4(__uint_as_float(raw.x << 16), __uint_as_float(raw.x & 0xffff0000u),
                     __uint_as_float(raw.y << 16), __uint_as_float(raw.y & 0xffff0000u));
}

// Fused step 2 of a learned band inner iteration:
//   r = r_old - a q       for the cell, the next plane's cell and the halo;
//   y = G^T r:  y_i = G(i,i) r_i + G(i+1,i) r_{i+1} + G(i+nx,i) r_{i+nx}
//                     + G(i+nx ny,i) r_{i+nx ny}   (values of the rows below);
//   partials of <r,r>; last CTA: inner residual test, stop flag, condition.
struct StResArgs {
  const float *rold;  // residual of the last iteration
  const float *q;     // A p of this iteration
  float *rnew;        // the new residual (other buffer of the pair)
  float *y;           // G^T r
  unsigned *ticket;
};

// One work item of k_st_res: this thread's partial sum of <r,r>.
template <bool CG>
__device__ __forceinline__ double st_res_item(const StencilGeom &g, const GBandView &G,
                                              const StResArgs &a, float na, int item) {
  const StPos s = st_pos(g, item);
  const int nx = g.nx, N = G.N, plane = nx * g.ny;
  const float *__restrict__ ro = a.rold;
  const float *__restrict__ qv = a.q;
  __shared__ float sr[kStY + 1][kStX + 1];   // r of the plane, right and top halo
  __shared__ float sg1[kStY][kStX + 1];      // G(j, j-1) of the cells, right halo
  __shared__ float sg2[kStY + 1][kStX];      // G(j, j-nx) of the cells, top halo
  double rr = 0.0;
  if (s.z0 >= s.z1) return rr;
  int i = s.z0 * plane + s.col;
  float r_c = fmaf(na, st_ld<CG>(qv + i), st_ld<CG>(ro + i));
  float4 gc = st_gvals(G.val, i);
  for (int zz = s.z0; zz < s.z1; zz++, i += plane) {
    const int in = (int)min((long long)i + plane, (long long)N - 1);
    const float r_n = fmaf(na, st_ld<CG>(qv + in), st_ld<CG>(ro + in));
    const float4 gn = st_gvals(G.val, in);
    sr[s.w][s.lane] = r_c;
    sg1[s.w][s.lane] = gc.y;
    sg2[s.w][s.lane] = gc.z;
    if (s.lane == kStX - 1) {
      const int j = min(i + 1, N - 1);
      sr[s.w][kStX] = fmaf(na, st_ld<CG>(qv + j), st_ld<CG>(ro + j));
      sg1[s.w][kStX] = st_gvals(G.val, j).y;
    }
    if (s.w == kStY - 1) {
      const int j = min(i + nx, N - 1);
      sr[kStY][s.lane] = fmaf(na, st_ld<CG>(qv + j), st_ld<CG>(ro + j));
      sg2[kStY][s.lane] = st_gvals(G.val, j).z;
    }
    __syncthreads();
    // G(i+1, i) and G(i+nx, i) come from the neighbouring cells; past the
    // grid's edge (a tile wider than the grid holds clamped copies there)
    // the true value is 0.
    const float v1 = (i + 1 < N && !s.xlast) ? sg1[s.w][s.lane + 1] : 0.f;
    const float v2 = (i + nx < N && !s.ylast) ? sg2[s.w + 1][s.lane] : 0.f;
    const float v3 = (long long)i + plane < N ? gn.w : 0.f;
    float sum = fmaf(gc.x, r_c, 0.f);
    sum = fmaf(v1, sr[s.w][s.lane + 1], sum);
    sum = fmaf(v2, sr[s.w + 1][s.lane], sum);
    sum = fmaf(v3, r_n, sum);
    if (s.valid) {
      a.rnew[i] = r_c;
      a.y[i] = sum;
      rr = fma((double)r_c, (double)r_c, rr);
    }
    __syncthreads();
    r_c = r_n;
    gc = gn;
  }
  return rr;
}

// The inner residual test after <r,r> (the last CTA of k_st_res).
__device__ __forceinline__ void st_residual_test(CgState *st, double rr) {
  st->in_iter += 1;
  st->total_inner += 1;
  const double res = sqrt(rr) / st->in_nrm0;
  st->in_res = res;
  if (!(res > st->in_tol) || inner_broke_down(st) || st->total_inner >= st->max_iter)
    st->in_stop = 1;
  if (st->use_cond)
    cudaGraphSetConditional((cudaGraphConditionalHandle)st->cond, st->in_stop ? 0u : 1u);
}

__global__ void __launch_bounds__(kThreads)
    k_st_res(StencilGeom g, GBandView G, StResArgs a, CgState *st, double *partials) {
  if (st->in_stop) return;
  const float na = (float)(-st->in_alpha);
  double rr = 0.0;
  for (int item = blockIdx.x; item < st_items(g); item += gridDim.x)
    rr += st_res_item<false>(g, G, a, na, item);
  double in[1] = {rr}, out[1];
  if (grid_reduce<1>(in, partials, a.ticket, out) && threadIdx.x == 0)
    st_residual_test(st, out[0]);
}

// z = G y with the row epilogue of Op:
//   z_i = G(i,i) y_i + G(i,i-1) y_{i-1} + G(i,i-nx) y_{i-nx} + G(i,i-nx ny) y_{i-nx ny}.
// One work item, accumulating into acc.
template <typename Op, bool CG>
__device__ __forceinline__ void st_gz_item(const StencilGeom &g, const GBandView &G,
                                           const float *__restrict__ y, const Op &op,
                                           typename Op::Acc &acc, int item) {
  const StPos s = st_pos(g, item);
  const int nx = g.nx, plane = nx * g.ny;
  __shared__ float sy[kStY + 1][kStX + 1];  // y of the plane, left and bottom halo
  if (s.z0 >= s.z1) return;
  int i = s.z0 * plane + s.col;
  float y_m = s.z0 > 0 ? st_ld<CG>(y + i - plane) : st_ld<CG>(y);
  float y_c = st_ld<CG>(y + i);
  for (int zz = s.z0; zz < s.z1; zz++, i += plane) {
    const typename Op::Pre pre = op.prefetch(i);
    const float4 gv = st_gvals(G.val, i);
    sy[s.w + 1][s.lane + 1] = y_c;
    if (s.lane == 0) sy[s.w + 1][0] = st_ld<CG>(y + max(i - 1, 0));
    if (s.w == 0) sy[0][s.lane + 1] = st_ld<CG>(y + max(i - nx, 0));
    // The next plane's y of the same column (needed after this plane).
    const float y_n = st_ld<CG>(y + min(i + plane, G.N - 1));
    __syncthreads();
    float sum = fmaf(gv.x, y_c, 0.f);
    sum = fmaf(gv.y, sy[s.w + 1][s.lane], sum);
    sum = fmaf(gv.z, sy[s.w][s.lane + 1], sum);
    sum = fmaf(gv.w, y_m, sum);
    if (s.valid) op.row(i, sum, acc, pre);
    __syncthreads();
    y_m = y_c;
    y_c = y_n;
  }
}

template <typename Op>
__global__ void __launch_bounds__(kThreads)
    k_st_gz(StencilGeom g, GBandView G, const float *__restrict__ y, Op op,
            CgState *st, double *partials) {
  if (op.skip(st)) return;
  typename Op::Acc acc;
  for (int item = blockIdx.x; item < st_items(g); item += gridDim.x)
    st_gz_item<Op, false>(g, G, y, op, acc, item);
  op.finish(acc, st, partials);
}

}  // namespace cgx
