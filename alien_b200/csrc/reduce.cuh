// reduce.cuh -- deterministic single-pass grid reductions.
//
// Every block reduces its threads' running values with warp shuffles and one
// shared-memory step, writes NC partials, and bumps an arrival counter.  The
// last block to arrive sums the partials of all blocks in block order and
// writes the NC results.  The grid size is a function of the problem size
// only, so the summation tree -- and therefore the rounding -- is identical on
// every run.  The result stays on the device: no host round trip per dot.
#pragma once

#include <cuda_runtime.h>

namespace ab2 {

enum class Combine { Sum, Max };

template <Combine C>
__device__ __forceinline__ double combine(double a, double b) {
  if constexpr (C == Combine::Sum) return a + b;
  else return a > b ? a : b;
}

template <Combine C>
__device__ __forceinline__ double warp_reduce(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = combine<C>(v, __shfl_down_sync(0xffffffffu, v, off));
  return v;
}

// Reduces acc[0..NC) over the whole grid.  Must be called by every thread of
// every block (no early returns before it).  Returns true in the thread that
// wrote the final results (thread 0 of the last block), so callers can run
// scalar epilogues there; `out` then holds the NC results.
template <int NC, Combine C = Combine::Sum>
__device__ __forceinline__ bool grid_reduce(double (&acc)[NC], double* partials, unsigned int* counter, double* out) {
  __shared__ double s_warp[NC][32];
  __shared__ bool s_last;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    double v = warp_reduce<C>(acc[c]);
    if (lane == 0) s_warp[c][warp] = v;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      double v = lane < nwarps ? s_warp[c][lane] : (C == Combine::Sum ? 0.0 : -1.0 / 0.0);
      v = warp_reduce<C>(v);
      if (lane == 0) partials[(size_t)c * gridDim.x + blockIdx.x] = v;
    }
    if (lane == 0) {
      __threadfence();
      unsigned int ticket = atomicAdd(counter, 1u);
      s_last = (ticket == gridDim.x - 1);
    }
  }
  __syncthreads();
  bool writer = false;
  if (s_last && warp == 0) {
    __threadfence();
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      double v = (C == Combine::Sum ? 0.0 : -1.0 / 0.0);
      for (int b = lane; b < (int)gridDim.x; b += 32) v = combine<C>(v, __ldcg(partials + (size_t)c * gridDim.x + b));
      v = warp_reduce<C>(v);
      if (lane == 0) out[c] = v;
    }
    if (lane == 0) {
      *counter = 0u;  // ready for the next launch that uses this slot
      __threadfence();
      writer = true;
    }
  }
  return writer;
}

}  // namespace ab2
