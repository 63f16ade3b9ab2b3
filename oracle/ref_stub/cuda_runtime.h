/*
 * Host-emulation header for compiling the reference's CUDA kernel file
 * (multi_gpuRkdg/src/kernelfunctions.cu) as plain C++ on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY: this header lets oracle/ref_harness.cpp run the
 * reference's unmodified kernel bodies as ordinary functions, one emulated
 * thread at a time.  It is placed ahead of the CUDA include path so that the
 * reference's `#include "cuda_runtime.h"` resolves here.
 *
 * - `__global__`/`__device__`/`__host__` vanish, so kernels become functions.
 * - `__shared__` becomes `thread_local`: the reference's `extern __shared__`
 *   arrays are then thread-local globals defined by the harness, so several
 *   OS threads can emulate separate CUDA blocks at the same time.
 * - threadIdx/blockIdx/blockDim are thread-local structs set by the harness
 *   before each emulated thread runs.
 * - __syncthreads() is a no-op: every per-thread kernel only touches its own
 *   shared-memory slots; the two block reductions are run with one thread per
 *   block, which makes their tree phase read zero-initialised padding only.
 */
#pragma once

struct rkdg_emu_dim3 {
    unsigned int x, y, z;
};

extern thread_local rkdg_emu_dim3 threadIdx;
extern thread_local rkdg_emu_dim3 blockIdx;
extern thread_local rkdg_emu_dim3 blockDim;

#define __global__
#define __device__
#define __host__
#define __shared__ thread_local

inline void __syncthreads() {}

typedef int cudaError_t;
