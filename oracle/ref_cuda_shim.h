/* Pre-included (nvcc --pre-include) when oracle/Makefile compiles the
 * reference's CUDA backend (cuda/CGCUDABase.cu, cuda/CGCUDA.cu,
 * cuda/kernel.cu) unmodified -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference's warp reduction (cuda/kernel.cu:80-86) calls the pre-CUDA-9
 * shuffle __shfl_down(v, o), which CUDA 12 no longer declares for sm_70 and
 * later. Every call reaches it with all 32 lanes of the warp (blockReduceSum,
 * kernel.cu:111-137: every thread, then all of warp 0; the blocks hold 128 or
 * 1024 threads), so __shfl_down_sync over the full warp computes the same sum.
 * The CUDA headers are read first so that the macro only touches the
 * reference's code. */
#pragma once
#if defined(__CUDACC__)
#include <cuda_runtime.h>
#define __shfl_down(v, o) __shfl_down_sync(0xffffffffu, (v), (o))
#endif
