// Bounded grid-wide barrier for cooperative launches.
//
// Generation-counting barrier: thread 0 of every CTA arrives on bar[0]; the
// last arrival resets it and bumps the generation bar[1].  The wait polls a
// bounded number of times; on a timeout (or when another CTA has already
// timed out) it sets *err and returns false, so every CTA can leave the
// kernel instead of hanging the GPU.  Launch with cudaLaunchCooperativeKernel
// so that all CTAs are co-resident.
#pragma once
#include <cuda_runtime.h>

namespace bbt {

constexpr long GRID_SPIN_LIMIT = 20000000;   // ~seconds of polling before giving up

__device__ __forceinline__ bool grid_sync(unsigned* bar, int* err) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = bar + 1;
    const unsigned g0 = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u) + 1u;
    if (arrived == gridDim.x) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long spins = 0;
      while (*gen == g0) {
        if (++spins > GRID_SPIN_LIMIT) { atomicExch(err, 1); break; }
        if (*(volatile int*)err) break;
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile int*)err == 0;
}

}  // namespace bbt
