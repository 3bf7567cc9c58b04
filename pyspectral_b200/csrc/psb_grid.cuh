// Grid-wide barrier with a bounded wait, for kernels launched cooperatively
// (every CTA co-resident, so a barrier completes once all CTAs reach it).
//
// Thread 0 of each CTA arrives on a counter; the last arrival resets it and
// advances the generation word, the others poll the generation.  A poll loop
// that exceeds `limit` polls (or sees another CTA's abort) gives up: it raises
// the abort word and the caller's status word and returns false, and the
// kernel then returns instead of waiting further.  Nothing waits without a
// limit, so a lost CTA cannot hang the GPU.
#pragma once
#include <cuda_runtime.h>

namespace psb {

struct GridBar {
  unsigned count;  // CTAs arrived in the current generation
  unsigned gen;    // generation, advanced by the last arrival
  int abort;       // raised by a CTA whose wait gave up
  int pad;
};

__device__ __forceinline__ bool grid_barrier(GridBar* gb, unsigned nblocks, unsigned limit, int* status) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned* vgen = &gb->gen;
    volatile int* vabort = &gb->abort;
    const unsigned g = *vgen;
    __threadfence();  // this CTA's writes before its arrival
    if (atomicAdd(&gb->count, 1u) == nblocks - 1) {
      atomicExch(&gb->count, 0u);
      __threadfence();
      atomicAdd(&gb->gen, 1u);
    } else {
      unsigned i = 0;
      while (*vgen == g) {
        if (++i > limit || *vabort) {
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    if (!ok) {
      atomicExch(&gb->abort, 1);
      atomicExch(status, 1);
    }
    __threadfence();  // the other CTAs' writes before this CTA reads them
  }
  __syncthreads();
  return ok != 0;
}

}  // namespace psb
