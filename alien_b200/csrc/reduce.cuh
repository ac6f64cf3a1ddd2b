// reduce.cuh -- deterministic single-pass grid reductions.
//
// Every block reduces its threads' running values with warp shuffles and one
// shared-memory step, writes NC partials, and bumps an arrival counter.  The
// last block to arrive sums the partials of all blocks in block order and
// writes the NC results.  The grid size is a function of the problem size
// only, so the summation tree -- and therefore the rounding -- is identical on
// every run.  The result stays on the device: no host round trip per dot.
//
// T is the accumulation type: double for the FP64 path, float for the FP32
// inner solves of the mixed-precision solver (partials and results then live
// in the same slot buffers, reinterpreted).
#pragma once

#include <cuda_runtime.h>

namespace ab2 {

enum class Combine { Sum, Max };

template <Combine C, class T>
__device__ __forceinline__ T combine(T a, T b) {
  if constexpr (C == Combine::Sum) return a + b;
  else return a > b ? a : b;
}

template <Combine C, class T>
__device__ __forceinline__ T warp_reduce(T v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = combine<C, T>(v, __shfl_down_sync(0xffffffffu, v, off));
  return v;
}

template <Combine C, class T>
__device__ __forceinline__ T reduce_identity() {
  return C == Combine::Sum ? T(0) : -T(1) / T(0);
}

// Reduces acc[0..NC) over the whole grid.  Must be called by every thread of
// every block (no early returns before it).  Returns true in the thread that
// wrote the final results (thread 0 of the last block), so callers can run
// scalar epilogues there; `out` then holds the NC results.
template <int NC, Combine C = Combine::Sum, class T>
__device__ __forceinline__ bool grid_reduce(T (&acc)[NC], T* partials, unsigned int* counter, T* out) {
  __shared__ T s_warp[NC][32];
  __shared__ bool s_last;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    T v = warp_reduce<C, T>(acc[c]);
    if (lane == 0) s_warp[c][warp] = v;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      T v = lane < nwarps ? s_warp[c][lane] : reduce_identity<C, T>();
      v = warp_reduce<C, T>(v);
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
      T v = reduce_identity<C, T>();
      for (int b = lane; b < (int)gridDim.x; b += 32) v = combine<C, T>(v, __ldcg(partials + (size_t)c * gridDim.x + b));
      v = warp_reduce<C, T>(v);
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

// The same reduction for a kernel whose logical grid of V * gridDim.x blocks
// runs on gridDim.x blocks: block b stands for logical blocks
// v * gridDim.x + b (v < V), reduces acc[v] exactly as that logical block
// would (the same shuffle tree over its 256 threads) and writes its partial
// at that logical position; the last block to arrive sums all V * gridDim.x
// partials in logical order.  So the summation tree -- and the rounding --
// is grid_reduce's on the logical grid, while a logical grid that does not
// fit the GPU at once runs in one wave.
template <int NC, int V, Combine C = Combine::Sum, class T>
__device__ __forceinline__ bool grid_reduce_v(T (&acc)[V][NC], T* partials, unsigned int* counter, T* out) {
  if constexpr (V == 1) {
    return grid_reduce<NC, C, T>(acc[0], partials, counter, out);
  } else {
    __shared__ T s_warp[V][NC][32];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    const int G = (int)gridDim.x * V;
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        T x = warp_reduce<C, T>(acc[v][c]);
        if (lane == 0) s_warp[v][c][warp] = x;
      }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
      for (int v = 0; v < V; ++v)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          T x = lane < nwarps ? s_warp[v][c][lane] : reduce_identity<C, T>();
          x = warp_reduce<C, T>(x);
          if (lane == 0) partials[(size_t)c * G + v * gridDim.x + blockIdx.x] = x;
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
        T x = reduce_identity<C, T>();
        for (int b = lane; b < G; b += 32) x = combine<C, T>(x, __ldcg(partials + (size_t)c * G + b));
        x = warp_reduce<C, T>(x);
        if (lane == 0) out[c] = x;
      }
      if (lane == 0) {
        *counter = 0u;
        __threadfence();
        writer = true;
      }
    }
    return writer;
  }
}

// The same reduction for a kernel whose threads each carry R consecutive
// logical threads of a logical grid of G blocks of 256 threads: thread t of
// the launch (256-thread blocks) holds the NC running values of logical
// threads R t .. R t + R - 1 (acc[u][c]), so launched block b holds logical
// blocks R b .. R b + R - 1.  The values are staged in shared memory by
// logical thread; every logical warp is reduced by the same shuffle tree on
// the same values, every logical block's eight warp sums likewise, and the
// last launched block sums the G partials of each component in logical
// order: the rounding of grid_reduce on a G-block grid.
template <int NC, int R, class T>
__device__ __forceinline__ bool grid_reduce_r(const T (&acc)[R][NC], int G, T* partials, unsigned int* counter,
                                              T* out) {
  constexpr int kB = 256;  // blockDim.x of the launch and of the logical grid
  constexpr int kW = kB / 32;
  __shared__ T s_val[NC][R * kB];
  __shared__ T s_warp[NC][R][kW];
  __shared__ bool s_last;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int u = 0; u < R; ++u) s_val[c][R * threadIdx.x + u] = acc[u][c];
  __syncthreads();
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int m = 0; m < R; ++m) {  // logical block m of this block, its warp `warp`
      T x = warp_reduce<Combine::Sum, T>(s_val[c][(m * kW + warp) * 32 + lane]);
      if (lane == 0) s_warp[c][m][warp] = x;
    }
  __syncthreads();
  if (warp < R) {  // warp m finishes logical block m
    const int L = R * (int)blockIdx.x + warp;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      T x = lane < kW ? s_warp[c][warp][lane] : T(0);
      x = warp_reduce<Combine::Sum, T>(x);
      if (lane == 0 && L < G) partials[(size_t)c * G + L] = x;
    }
    if (lane == 0) __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned int ticket = atomicAdd(counter, 1u);
    s_last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  bool writer = false;
  if (s_last && warp == 0) {
    __threadfence();
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      T x = T(0);
      for (int b = lane; b < G; b += 32) x = x + __ldcg(partials + (size_t)c * G + b);
      x = warp_reduce<Combine::Sum, T>(x);
      if (lane == 0) out[c] = x;
    }
    if (lane == 0) {
      *counter = 0u;
      __threadfence();
      writer = true;
    }
  }
  return writer;
}

}  // namespace ab2
