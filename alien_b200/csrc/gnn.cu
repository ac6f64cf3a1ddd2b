// gnn.cu -- the learned preconditioner: a message-passing network on the
// matrix graph, its training kernels, and flexible CG with ILU(0) fallback.
// No counterpart in the reference; the network is defined (and checked) by
// oracle/gnn_oracle.py:
//   s = rms(r); x0_i = [r_i/s, log(a_ii)/10]; h1 = relu(W0 x0 + b0)            (2 -> 64)
//   4 x { g_ij = sigmoid(u e_ij + c), e_ij = log|a_ij| - log a_ii ;
//         m_i = sum_j g_ij h_j ; h <- relu(W [h; m] + b) }                       (128 -> 64)
//   z_i = s (wd . h_i + bd) / a_ii
// Activations are stored in BF16 ([n][64], 128 B per node); the dense layers
// are BF16 x BF16 -> FP32 tensor-core MMAs (mma.sync m16n8k16; a warp computes
// 16 nodes x 64 outputs over K = 128); aggregation is a warp per node with two
// features per lane.  Training: hand-written backward kernels (loss
// (z-e)^T A (z-e) / e^T A e on (residual, error) pairs), per-block partial
// sums reduced in a fixed order (deterministic), Adam on FP32 master weights
// with BF16 copies for the forward.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "ab2_internal.cuh"
#include "precond.cuh"
#include "reduce.cuh"
#include "spmv_view.cuh"

namespace ab2 {
namespace {

constexpr int kH = 64;          // hidden width
constexpr int kLayers = 4;
constexpr int kIn = 2 * kH;     // dense layer input [h ; m]
constexpr int kWStride = kIn + 8;  // padded smem row (bf16): conflict-free fragment loads
// flat parameter layout (oracle/gnn_oracle.py Params.flat)
constexpr int kOffW0 = 0;
constexpr int kOffB0 = kOffW0 + kH * 2;
constexpr int kOffW = kOffB0 + kH;
constexpr int kOffB = kOffW + kLayers * kH * kIn;
constexpr int kOffU = kOffB + kLayers * kH;
constexpr int kOffC = kOffU + kLayers;
constexpr int kOffWd = kOffC + kLayers;
constexpr int kOffBd = kOffWd + kH;
constexpr int kParams = kOffBd + 1;

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned*>(&v);
}
__device__ __forceinline__ float2 unpack_bf16(unsigned u) {
  __nv_bfloat162 v = *reinterpret_cast<__nv_bfloat162*>(&u);
  return __bfloat1622float2(v);
}
__device__ __forceinline__ float sigmoidf(float t) { return 1.f / (1.f + expf(-t)); }

// D = A B + D, m16n8k16, A row-major BF16 (4 regs), B col-major BF16 (2 regs), FP32 accumulators.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ------------------------------------------------------------------ graph features
// diag, 1/diag, log(diag)/10 per row; per CSR entry the edge feature
// log|a_ij| - log a_ii (0 and flagged on the diagonal) and the position of the
// transposed entry (the pattern must be structurally symmetric).
__global__ void k_gnn_prep(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                           const int* __restrict__ dcol, float* __restrict__ invd, float* __restrict__ logd10,
                           float* __restrict__ efeat, int* __restrict__ tidx, int* bad) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int dk = dcol[i];
    const bool has_d = dk < rp[i + 1] && ci[dk] == i && v[dk] > 0;
    if (!has_d) {
      atomicOr(bad, 1);
      continue;
    }
    const double d = v[dk];
    invd[i] = (float)(1.0 / d);
    logd10[i] = (float)(log(d) / 10.0);
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = ci[k];
      if (j == i) {
        efeat[k] = 0.f;
        tidx[k] = -1;
        continue;
      }
      efeat[k] = (float)(log(fabs(v[k])) - log(d));
      int t = -1;  // (j, i) in row j (columns sorted: binary search)
      int lo = rp[j], hi = rp[j + 1] - 1;
      while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        if (ci[mid] == i) {
          t = mid;
          break;
        }
        if (ci[mid] < i) lo = mid + 1;
        else hi = mid - 1;
      }
      tidx[k] = t;
      if (t < 0) atomicOr(bad, 2);
    }
  }
}

// ------------------------------------------------------------------ forward
// h1 = relu(W0 [r_i/s, logd10_i] + b0), one thread per node.
__global__ void k_gnn_encode(int n, const double* __restrict__ r, const double* __restrict__ rr,
                             const float* __restrict__ logd10, const float* __restrict__ P, bf16* __restrict__ h1) {
  const double rms = sqrt(*rr / (double)max(n, 1));
  const float inv_s = rms > 0 ? (float)(1.0 / rms) : 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float x0 = (float)r[i] * inv_s, x1 = logd10[i];
    unsigned* out = reinterpret_cast<unsigned*>(h1 + (size_t)i * kH);
#pragma unroll 8
    for (int j = 0; j < kH; j += 2) {
      const float p0 = fmaf(P[kOffW0 + 2 * j], x0, fmaf(P[kOffW0 + 2 * j + 1], x1, P[kOffB0 + j]));
      const float p1 = fmaf(P[kOffW0 + 2 * j + 2], x0, fmaf(P[kOffW0 + 2 * j + 3], x1, P[kOffB0 + j + 1]));
      out[j / 2] = pack_bf16(fmaxf(p0, 0.f), fmaxf(p1, 0.f));
    }
  }
}

// m_i = sum_{j != i} sigmoid(u e_ij + c) h_j: a warp per node, lane = features 2l, 2l+1.
__global__ void k_gnn_aggregate(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                const float* __restrict__ efeat, const float* __restrict__ P, int layer,
                                const bf16* __restrict__ h, bf16* __restrict__ m) {
  const int lane = threadIdx.x & 31;
  const float u = P[kOffU + layer], c = P[kOffC + layer];
  const unsigned* hv = reinterpret_cast<const unsigned*>(h);
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
    float a0 = 0.f, a1 = 0.f;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = ci[k];
      if (j == i) continue;
      const float g = sigmoidf(fmaf(u, efeat[k], c));
      const float2 x = unpack_bf16(hv[(size_t)j * (kH / 2) + lane]);
      a0 = fmaf(g, x.x, a0);
      a1 = fmaf(g, x.y, a1);
    }
    reinterpret_cast<unsigned*>(m)[(size_t)i * (kH / 2) + lane] = pack_bf16(a0, a1);
  }
}

// h_out = relu(W [h ; m] + b) on tensor cores.  W (64 x 128, BF16) is staged
// in shared memory with padded rows; a warp takes 16 nodes at a time.
__global__ void __launch_bounds__(256) k_gnn_dense(int n, const bf16* __restrict__ h, const bf16* __restrict__ m,
                                                   const bf16* __restrict__ W, const float* __restrict__ bias,
                                                   bf16* __restrict__ hout) {
  __shared__ __align__(16) bf16 Ws[kH * kWStride];
  __shared__ float bs[kH];
  for (int t = threadIdx.x; t < kH * kIn; t += blockDim.x) Ws[(t / kIn) * kWStride + t % kIn] = W[t];
  if (threadIdx.x < kH) bs[threadIdx.x] = bias[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const unsigned* hv = reinterpret_cast<const unsigned*>(h);
  const unsigned* mv = reinterpret_cast<const unsigned*>(m);
  for (int tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile * 16 < n; tile += warps) {
    const int r0 = tile * 16 + g, r1 = r0 + 8;
    const bool ok0 = r0 < n, ok1 = r1 < n;
    float acc[8][4];
#pragma unroll
    for (int nb = 0; nb < 8; ++nb) acc[nb][0] = acc[nb][1] = acc[nb][2] = acc[nb][3] = 0.f;
#pragma unroll
    for (int ks = 0; ks < 8; ++ks) {
      const unsigned* src = ks < 4 ? hv : mv;
      const int col = (ks & 3) * 16 + 2 * t;  // feature of a0 (bf16 index within the 64)
      unsigned a[4];
      a[0] = ok0 ? src[((size_t)r0 * kH + col) >> 1] : 0u;
      a[1] = ok1 ? src[((size_t)r1 * kH + col) >> 1] : 0u;
      a[2] = ok0 ? src[((size_t)r0 * kH + col + 8) >> 1] : 0u;
      a[3] = ok1 ? src[((size_t)r1 * kH + col + 8) >> 1] : 0u;
      const int k0 = ks * 16 + 2 * t;
#pragma unroll
      for (int nb = 0; nb < 8; ++nb) {
        const bf16* wrow = Ws + (nb * 8 + g) * kWStride;
        const unsigned b0 = *reinterpret_cast<const unsigned*>(wrow + k0);
        const unsigned b1 = *reinterpret_cast<const unsigned*>(wrow + k0 + 8);
        mma_bf16(acc[nb], a, b0, b1);
      }
    }
    unsigned* out = reinterpret_cast<unsigned*>(hout);
#pragma unroll
    for (int nb = 0; nb < 8; ++nb) {
      const int c = nb * 8 + 2 * t;
      if (ok0) out[((size_t)r0 * kH + c) >> 1] = pack_bf16(fmaxf(acc[nb][0] + bs[c], 0.f), fmaxf(acc[nb][1] + bs[c + 1], 0.f));
      if (ok1) out[((size_t)r1 * kH + c) >> 1] = pack_bf16(fmaxf(acc[nb][2] + bs[c], 0.f), fmaxf(acc[nb][3] + bs[c + 1], 0.f));
    }
  }
}

// z_i = s (wd . h5_i + bd) / a_ii (FP64 out, for the solver).
__global__ void k_gnn_decode(int n, const bf16* __restrict__ h5, const float* __restrict__ P,
                             const float* __restrict__ invd, const double* __restrict__ rr, double* __restrict__ z) {
  const double rms = sqrt(*rr / (double)max(n, 1));
  const unsigned* hv = reinterpret_cast<const unsigned*>(h5);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float y = P[kOffBd];
#pragma unroll 8
    for (int j = 0; j < kH / 2; ++j) {
      const float2 x = unpack_bf16(hv[(size_t)i * (kH / 2) + j]);
      y = fmaf(P[kOffWd + 2 * j], x.x, y);
      y = fmaf(P[kOffWd + 2 * j + 1], x.y, y);
    }
    z[i] = rms * (double)y * (double)invd[i];
  }
}

// FP32 master weights -> BF16 copies of the dense layers' W.
__global__ void k_gnn_wcopy(const float* __restrict__ P, bf16* __restrict__ Wb) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < kLayers * kH * kIn; t += gridDim.x * blockDim.x)
    Wb[t] = __float2bfloat16_rn(P[kOffW + t]);
}

// ------------------------------------------------------------------ backward
// Warp-per-node kernels leave per-block partial sums in part[block][width];
// k_gnn_reduce_partials adds them in block order (deterministic).
constexpr int kWarpsPerBlock = 8;

// dy_i = dz_i s / a_ii ; dh5_i = dy_i wd ; partials of grad wd (64) and bd (1).
__global__ void __launch_bounds__(256) k_gnn_decode_bwd(int n, const double* __restrict__ dz, const double* __restrict__ rr,
                                                        const float* __restrict__ invd, const bf16* __restrict__ h5,
                                                        const float* __restrict__ P, float* __restrict__ dh,
                                                        float* __restrict__ part) {
  __shared__ float s_acc[kWarpsPerBlock][kH + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double rms = sqrt(*rr / (double)max(n, 1));
  const unsigned* hv = reinterpret_cast<const unsigned*>(h5);
  const float w0 = P[kOffWd + 2 * lane], w1 = P[kOffWd + 2 * lane + 1];
  float g0 = 0.f, g1 = 0.f, gb = 0.f;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
    const float dy = (float)(dz[i] * rms * (double)invd[i]);
    const float2 x = unpack_bf16(hv[(size_t)i * (kH / 2) + lane]);
    g0 = fmaf(dy, x.x, g0);
    g1 = fmaf(dy, x.y, g1);
    gb += dy;
    reinterpret_cast<float2*>(dh)[(size_t)i * (kH / 2) + lane] = make_float2(dy * w0, dy * w1);
  }
  s_acc[warp][2 * lane] = g0;
  s_acc[warp][2 * lane + 1] = g1;
  if (lane == 0) s_acc[warp][kH] = gb;
  __syncthreads();
  for (int k = threadIdx.x; k <= kH; k += blockDim.x) {
    float s = 0.f;
    for (int w = 0; w < kWarpsPerBlock; ++w) s += s_acc[w][k];
    part[(size_t)blockIdx.x * (kH + 1) + k] = s;
  }
}

// [dh_in ; dm] = dpre W on tensor cores, dpre = dh (.) (h_out > 0) rounded to
// BF16; W^T (128 x 64) staged in shared memory with padded rows.
constexpr int kWTStride = kH + 8;
__global__ void __launch_bounds__(256) k_gnn_dense_bwd(int n, const float* __restrict__ dh, const bf16* __restrict__ hout,
                                                       const bf16* __restrict__ W, float* __restrict__ dh_in,
                                                       float* __restrict__ dm) {
  __shared__ __align__(16) bf16 WT[kIn * kWTStride];
  for (int t = threadIdx.x; t < kH * kIn; t += blockDim.x) {
    const int o = t / kIn, k = t % kIn;
    WT[k * kWTStride + o] = W[t];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const unsigned* hv = reinterpret_cast<const unsigned*>(hout);
  auto dpre2 = [&](int row, int col) -> unsigned {  // BF16 pair of dpre[row][col], [col+1]
    const float2 d = reinterpret_cast<const float2*>(dh)[((size_t)row * kH + col) >> 1];
    const float2 hv2 = unpack_bf16(hv[((size_t)row * kH + col) >> 1]);
    return pack_bf16(hv2.x > 0.f ? d.x : 0.f, hv2.y > 0.f ? d.y : 0.f);
  };
  for (int tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile * 16 < n; tile += warps) {
    const int r0 = tile * 16 + g, r1 = r0 + 8;
    const bool ok0 = r0 < n, ok1 = r1 < n;
    float acc[16][4];
#pragma unroll
    for (int nb = 0; nb < 16; ++nb) acc[nb][0] = acc[nb][1] = acc[nb][2] = acc[nb][3] = 0.f;
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const int col = ks * 16 + 2 * t;
      unsigned a[4];
      a[0] = ok0 ? dpre2(r0, col) : 0u;
      a[1] = ok1 ? dpre2(r1, col) : 0u;
      a[2] = ok0 ? dpre2(r0, col + 8) : 0u;
      a[3] = ok1 ? dpre2(r1, col + 8) : 0u;
#pragma unroll
      for (int nb = 0; nb < 16; ++nb) {
        const bf16* wrow = WT + (nb * 8 + g) * kWTStride;
        const unsigned b0 = *reinterpret_cast<const unsigned*>(wrow + col);
        const unsigned b1 = *reinterpret_cast<const unsigned*>(wrow + col + 8);
        mma_bf16(acc[nb], a, b0, b1);
      }
    }
#pragma unroll
    for (int nb = 0; nb < 16; ++nb) {
      const int c = nb * 8 + 2 * t;
      float* dst = c < kH ? dh_in : dm;
      const int cc = c & (kH - 1);
      if (ok0) reinterpret_cast<float2*>(dst)[((size_t)r0 * kH + cc) >> 1] = make_float2(acc[nb][0], acc[nb][1]);
      if (ok1) reinterpret_cast<float2*>(dst)[((size_t)r1 * kH + cc) >> 1] = make_float2(acc[nb][2], acc[nb][3]);
    }
  }
}

// dh_j += sum_{i neighbour of j} g_ij dm_i (in place on dh_in) and the gate
// gradients of row j's edges: dg = dm_j . h_i, ds = dg g (1-g), du += ds e, dc += ds.
__global__ void __launch_bounds__(256) k_gnn_agg_bwd(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                                     const float* __restrict__ efeat, const int* __restrict__ tidx,
                                                     const float* __restrict__ P, int layer, const bf16* __restrict__ h,
                                                     const float* __restrict__ dm, float* dh, float* __restrict__ part) {
  __shared__ float s_acc[kWarpsPerBlock][2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float u = P[kOffU + layer], c = P[kOffC + layer];
  const unsigned* hv = reinterpret_cast<const unsigned*>(h);
  const float2* dm2 = reinterpret_cast<const float2*>(dm);
  float du = 0.f, dc = 0.f;
  for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < n; j += (gridDim.x * blockDim.x) >> 5) {
    float2 acc = reinterpret_cast<float2*>(dh)[(size_t)j * (kH / 2) + lane];
    const float2 dmj = dm2[(size_t)j * (kH / 2) + lane];
    for (int k = rp[j]; k < rp[j + 1]; ++k) {
      const int i = ci[k];
      if (i == j) continue;
      const float gt = sigmoidf(fmaf(u, efeat[tidx[k]], c));  // g of entry (i, j)
      const float2 dmi = dm2[(size_t)i * (kH / 2) + lane];
      acc.x = fmaf(gt, dmi.x, acc.x);
      acc.y = fmaf(gt, dmi.y, acc.y);
      const float2 hi = unpack_bf16(hv[(size_t)i * (kH / 2) + lane]);
      float dg = fmaf(dmj.x, hi.x, dmj.y * hi.y);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) dg += __shfl_xor_sync(0xffffffffu, dg, off);
      const float e = efeat[k];
      const float gk = sigmoidf(fmaf(u, e, c));
      const float ds = dg * gk * (1.f - gk);
      du = fmaf(ds, e, du);
      dc += ds;
    }
    reinterpret_cast<float2*>(dh)[(size_t)j * (kH / 2) + lane] = acc;
  }
  if (lane == 0) {
    s_acc[warp][0] = du;
    s_acc[warp][1] = dc;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    float s = 0.f;
    for (int w = 0; w < kWarpsPerBlock; ++w) s += s_acc[w][threadIdx.x];
    part[(size_t)blockIdx.x * 2 + threadIdx.x] = s;
  }
}

// Partials of grad W (64 x 128) and grad b (64): sum_i dpre_i [h_i ; m_i]^T,
// staged 32 nodes at a time; thread t owns output o = t/4, inputs (t%4)*32 ..+32.
__global__ void __launch_bounds__(256) k_gnn_wgrad(int n, const float* __restrict__ dh, const bf16* __restrict__ hout,
                                                   const bf16* __restrict__ h, const bf16* __restrict__ m,
                                                   float* __restrict__ part) {
  __shared__ float s_dp[32][kH + 1];
  __shared__ float s_in[32][kIn + 1];
  const int o = threadIdx.x >> 2, k0 = (threadIdx.x & 3) * 32;
  float acc[32];
#pragma unroll
  for (int q = 0; q < 32; ++q) acc[q] = 0.f;
  float accb = 0.f;
  const int per = (n + gridDim.x - 1) / gridDim.x;
  const int lo = blockIdx.x * per, hi = min(n, lo + per);
  for (int base = lo; base < hi; base += 32) {
    __syncthreads();
    for (int t = threadIdx.x; t < 32 * kH; t += blockDim.x) {
      const int r = t / kH, c = t % kH, i = base + r;
      float dp = 0.f, hh = 0.f, mm = 0.f;
      if (i < hi) {
        const float hv = __bfloat162float(hout[(size_t)i * kH + c]);
        dp = hv > 0.f ? dh[(size_t)i * kH + c] : 0.f;
        hh = __bfloat162float(h[(size_t)i * kH + c]);
        mm = __bfloat162float(m[(size_t)i * kH + c]);
      }
      s_dp[r][c] = dp;
      s_in[r][c] = hh;
      s_in[r][kH + c] = mm;
    }
    __syncthreads();
    const int rows = min(32, hi - base);
    for (int r = 0; r < rows; ++r) {
      const float d = s_dp[r][o];
#pragma unroll
      for (int q = 0; q < 32; ++q) acc[q] = fmaf(d, s_in[r][k0 + q], acc[q]);
      if (k0 == 0) accb += d;
    }
  }
  float* out = part + (size_t)blockIdx.x * (kH * kIn + kH);
#pragma unroll
  for (int q = 0; q < 32; ++q) out[o * kIn + k0 + q] = acc[q];
  if (k0 == 0) out[kH * kIn + o] = accb;
}

// Partials of grad W0 (64 x 2) and b0: dpre0 = dh1 (.) (h1 > 0), x0 recomputed.
__global__ void __launch_bounds__(256) k_gnn_encode_bwd(int n, const double* __restrict__ r, const double* __restrict__ rr,
                                                        const float* __restrict__ logd10, const bf16* __restrict__ h1,
                                                        const float* __restrict__ dh, float* __restrict__ part) {
  __shared__ float s_acc[kWarpsPerBlock][3 * kH];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double rms = sqrt(*rr / (double)max(n, 1));
  const float inv_s = rms > 0 ? (float)(1.0 / rms) : 0.f;
  const unsigned* hv = reinterpret_cast<const unsigned*>(h1);
  float a[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // (W0[o][0], W0[o][1], b0[o]) for o = 2 lane, 2 lane + 1
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
    const float x0 = (float)r[i] * inv_s, x1 = logd10[i];
    const float2 hh = unpack_bf16(hv[(size_t)i * (kH / 2) + lane]);
    const float2 d = reinterpret_cast<const float2*>(dh)[(size_t)i * (kH / 2) + lane];
    const float d0 = hh.x > 0.f ? d.x : 0.f, d1 = hh.y > 0.f ? d.y : 0.f;
    a[0] = fmaf(d0, x0, a[0]);
    a[1] = fmaf(d0, x1, a[1]);
    a[2] += d0;
    a[3] = fmaf(d1, x0, a[3]);
    a[4] = fmaf(d1, x1, a[4]);
    a[5] += d1;
  }
  // layout: W0 (o, 0..1) at 2o, 2o+1 ; b0 at 128 + o
  s_acc[warp][4 * lane + 0] = a[0];
  s_acc[warp][4 * lane + 1] = a[1];
  s_acc[warp][4 * lane + 2] = a[3];
  s_acc[warp][4 * lane + 3] = a[4];
  s_acc[warp][2 * kH + 2 * lane] = a[2];
  s_acc[warp][2 * kH + 2 * lane + 1] = a[5];
  __syncthreads();
  for (int k = threadIdx.x; k < 3 * kH; k += blockDim.x) {
    float s = 0.f;
    for (int w = 0; w < kWarpsPerBlock; ++w) s += s_acc[w][k];
    part[(size_t)blockIdx.x * (3 * kH) + k] = s;
  }
}

// out[k] = sum_b part[b][k], block order.
__global__ void k_gnn_reduce_partials(int nb, int width, const float* __restrict__ part, float* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < width; k += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nb; ++b) s += part[(size_t)b * width + k];
    out[k] = s;
  }
}

// Adam on the FP32 master weights.
__global__ void k_gnn_adam(int np, float* __restrict__ P, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
    const float gk = g[k];
    const float mk = fmaf(b1, m[k], (1.f - b1) * gk);
    const float vk = fmaf(b2, v[k], (1.f - b2) * gk * gk);
    m[k] = mk;
    v[k] = vk;
    P[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
  }
}

}  // namespace
}  // namespace ab2

using namespace ab2;

struct ab2_gnn {
  ab2_context* ctx = nullptr;
  float* d_P = nullptr;      // FP32 master parameters (flat)
  float* d_grad = nullptr;
  float* d_am = nullptr;     // Adam moments
  float* d_av = nullptr;
  bf16* d_Wb = nullptr;      // BF16 copies of the dense layers' W
  int step = 0;
  // binding to a matrix
  const ab2_matrix* A = nullptr;
  int n = 0;
  float *d_invd = nullptr, *d_logd10 = nullptr, *d_efeat = nullptr;
  int* d_tidx = nullptr;
  bf16* d_h = nullptr;       // h1..h5, n x 64 each
  bf16* d_m = nullptr;       // m1..m4
  double* d_rr = nullptr;
  float *d_dh = nullptr, *d_dh2 = nullptr, *d_dm = nullptr;
  double *d_z = nullptr, *d_d = nullptr, *d_Ad = nullptr, *d_Ae = nullptr;
  float* d_part = nullptr;
  float* d_red = nullptr;    // reduced partials scratch (64 x 128 + 64)
  long long part_cap = 0;
};

namespace ab2 {
namespace {

int warp_grid(ab2_context* ctx, int n) {
  return std::max(1, std::min((n + kWarpsPerBlock - 1) / kWarpsPerBlock, ctx->num_sms * 8));
}
int tile_grid(ab2_context* ctx, int n) { return std::max(1, std::min((n + 127) / 128, ctx->num_sms * 4)); }
int wgrad_grid(ab2_context* ctx, int n) { return std::max(1, std::min((n + 2047) / 2048, ctx->num_sms * 2)); }

bf16* hbuf(ab2_gnn* G, int l) { return G->d_h + (size_t)l * G->n * kH; }
bf16* mbuf(ab2_gnn* G, int l) { return G->d_m + (size_t)l * G->n * kH; }

void release_binding(ab2_gnn* G) {
  ab2_context* ctx = G->ctx;
  for (void* p : {(void*)G->d_invd, (void*)G->d_logd10, (void*)G->d_efeat, (void*)G->d_tidx, (void*)G->d_h,
                  (void*)G->d_m, (void*)G->d_rr, (void*)G->d_dh, (void*)G->d_dh2, (void*)G->d_dm, (void*)G->d_z,
                  (void*)G->d_d, (void*)G->d_Ad, (void*)G->d_Ae, (void*)G->d_part, (void*)G->d_red})
    dev_free(ctx, p);
  G->d_invd = G->d_logd10 = G->d_efeat = nullptr;
  G->d_tidx = nullptr;
  G->d_h = G->d_m = nullptr;
  G->d_rr = nullptr;
  G->d_dh = G->d_dh2 = G->d_dm = nullptr;
  G->d_z = G->d_d = G->d_Ad = G->d_Ae = nullptr;
  G->d_part = G->d_red = nullptr;
  G->A = nullptr;
  G->n = 0;
}

// z = network(r) (FP64 in and out).
void gnn_forward(ab2_gnn* G, const double* r, double* z) {
  ab2_context* ctx = G->ctx;
  const int n = G->n;
  const ab2_matrix* A = G->A;
  op_dot(ctx, n, r, r, G->d_rr, 0);
  k_gnn_encode<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, r, G->d_rr, G->d_logd10, G->d_P, hbuf(G, 0));
  check_launch(ctx, "gnn_encode");
  for (int l = 0; l < kLayers; ++l) {
    k_gnn_aggregate<<<warp_grid(ctx, n), 256, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, G->d_efeat, G->d_P, l,
                                                                hbuf(G, l), mbuf(G, l));
    check_launch(ctx, "gnn_aggregate");
    k_gnn_dense<<<tile_grid(ctx, n), 256, 0, ctx->stream>>>(n, hbuf(G, l), mbuf(G, l), G->d_Wb + (size_t)l * kH * kIn,
                                                            G->d_P + kOffB + l * kH, hbuf(G, l + 1));
    check_launch(ctx, "gnn_dense");
  }
  k_gnn_decode<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, hbuf(G, kLayers), G->d_P, G->d_invd, G->d_rr, z);
  check_launch(ctx, "gnn_decode");
}

void reduce_into(ab2_gnn* G, int nb, int width, float* out) {
  k_gnn_reduce_partials<<<(width + 255) / 256, 256, 0, G->ctx->stream>>>(nb, width, G->d_part, out);
  check_launch(G->ctx, "gnn_reduce");
}

// Loss (z-e)^T A (z-e) / e^T A e and its gradient into d_grad.
double gnn_loss_grad(ab2_gnn* G, const double* r, const double* e) {
  ab2_context* ctx = G->ctx;
  const ab2_matrix* A = G->A;
  const int n = G->n;
  gnn_forward(G, r, G->d_z);
  op_copy(ctx, n, G->d_z, G->d_d);
  op_axpy(ctx, n, -1.0, e, G->d_d);
  op_spmv(ctx, A, G->d_d, G->d_Ad, AB2_SPMV_AUTO);
  op_spmv(ctx, A, e, G->d_Ae, AB2_SPMV_AUTO);
  double* s = red_slot(ctx, 6).result;
  op_dot(ctx, n, e, G->d_Ae, s, 6);
  const double eAe = read_scalar(ctx, s);
  op_dot(ctx, n, G->d_d, G->d_Ad, s, 6);
  const double dAd = read_scalar(ctx, s);
  require(eAe > 0, "gnn training pair: e^T A e must be positive");
  op_scal(ctx, n, 2.0 / eAe, G->d_Ad);  // dz
  const int wg = warp_grid(ctx, n);
  k_gnn_decode_bwd<<<wg, 256, 0, ctx->stream>>>(n, G->d_Ad, G->d_rr, G->d_invd, hbuf(G, kLayers), G->d_P, G->d_dh,
                                                G->d_part);
  check_launch(ctx, "gnn_decode_bwd");
  reduce_into(G, wg, kH + 1, G->d_grad + kOffWd);
  float* dh = G->d_dh;
  float* dh2 = G->d_dh2;
  for (int l = kLayers - 1; l >= 0; --l) {
    const int gg = wgrad_grid(ctx, n);
    k_gnn_wgrad<<<gg, 256, 0, ctx->stream>>>(n, dh, hbuf(G, l + 1), hbuf(G, l), mbuf(G, l), G->d_part);
    check_launch(ctx, "gnn_wgrad");
    reduce_into(G, gg, kH * kIn + kH, G->d_red);
    AB2_CUDA(cudaMemcpyAsync(G->d_grad + kOffW + (size_t)l * kH * kIn, G->d_red, sizeof(float) * kH * kIn,
                             cudaMemcpyDeviceToDevice, ctx->stream));
    AB2_CUDA(cudaMemcpyAsync(G->d_grad + kOffB + l * kH, G->d_red + kH * kIn, sizeof(float) * kH,
                             cudaMemcpyDeviceToDevice, ctx->stream));
    k_gnn_dense_bwd<<<tile_grid(ctx, n), 256, 0, ctx->stream>>>(n, dh, hbuf(G, l + 1), G->d_Wb + (size_t)l * kH * kIn,
                                                                dh2, G->d_dm);
    check_launch(ctx, "gnn_dense_bwd");
    k_gnn_agg_bwd<<<wg, 256, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, G->d_efeat, G->d_tidx, G->d_P, l, hbuf(G, l),
                                               G->d_dm, dh2, G->d_part);
    check_launch(ctx, "gnn_agg_bwd");
    reduce_into(G, wg, 2, G->d_red);
    AB2_CUDA(cudaMemcpyAsync(G->d_grad + kOffU + l, G->d_red, sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
    AB2_CUDA(cudaMemcpyAsync(G->d_grad + kOffC + l, G->d_red + 1, sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
    std::swap(dh, dh2);
  }
  k_gnn_encode_bwd<<<wg, 256, 0, ctx->stream>>>(n, r, G->d_rr, G->d_logd10, hbuf(G, 0), dh, G->d_part);
  check_launch(ctx, "gnn_encode_bwd");
  reduce_into(G, wg, 3 * kH, G->d_grad + kOffW0);
  return dAd / eAe;
}

}  // namespace
}  // namespace ab2

extern "C" {

int ab2_gnn_param_count(void) { return kParams; }

int ab2_gnn_create(ab2_context* ctx, const float* params, unsigned long long seed, ab2_gnn** out) {
  if (!ctx || !out) return AB2_ERR_BAD_ARG;
  *out = nullptr;
  ab2_gnn* G = new (std::nothrow) ab2_gnn();
  if (!G) return AB2_ERR_OOM;
  G->ctx = ctx_retain(ctx);
  int rc = guard(ctx, [&] {
    std::vector<float> h(kParams, 0.f);
    if (params) {
      std::copy(params, params + kParams, h.begin());
    } else {  // He-style normal initialisation
      std::mt19937_64 gen(seed);
      std::normal_distribution<float> w0(0.f, 1.f), wl(0.f, std::sqrt(2.f / kIn)), wd(0.f, std::sqrt(1.f / kH));
      for (int k = 0; k < 2 * kH; ++k) h[kOffW0 + k] = w0(gen);
      for (int k = 0; k < kLayers * kH * kIn; ++k) h[kOffW + k] = wl(gen);
      for (int k = 0; k < kLayers * kH; ++k) h[kOffB + k] = 0.01f;
      for (int l = 0; l < kLayers; ++l) h[kOffU + l] = 0.5f;
      for (int k = 0; k < kH; ++k) h[kOffWd + k] = wd(gen);
    }
    G->d_P = dev_alloc<float>(ctx, kParams);
    G->d_grad = dev_alloc<float>(ctx, kParams);
    G->d_am = dev_alloc<float>(ctx, kParams);
    G->d_av = dev_alloc<float>(ctx, kParams);
    G->d_Wb = dev_alloc<bf16>(ctx, (size_t)kLayers * kH * kIn);
    AB2_CUDA(cudaMemcpyAsync(G->d_P, h.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice, ctx->stream));
    AB2_CUDA(cudaMemsetAsync(G->d_grad, 0, sizeof(float) * kParams, ctx->stream));
    AB2_CUDA(cudaMemsetAsync(G->d_am, 0, sizeof(float) * kParams, ctx->stream));
    AB2_CUDA(cudaMemsetAsync(G->d_av, 0, sizeof(float) * kParams, ctx->stream));
    k_gnn_wcopy<<<64, 256, 0, ctx->stream>>>(G->d_P, G->d_Wb);
    check_launch(ctx, "gnn_wcopy");
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  });
  if (rc != AB2_OK) {
    ab2_gnn_destroy(G);
    return rc;
  }
  *out = G;
  return AB2_OK;
}

int ab2_gnn_get_params(const ab2_gnn* G, float* params) {
  if (!G || !params) return AB2_ERR_BAD_ARG;
  return guard(G->ctx, [&] {
    AB2_CUDA(cudaMemcpyAsync(params, G->d_P, sizeof(float) * kParams, cudaMemcpyDeviceToHost, G->ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(G->ctx->stream));
  });
}

int ab2_gnn_set_params(ab2_gnn* G, const float* params) {
  if (!G || !params) return AB2_ERR_BAD_ARG;
  return guard(G->ctx, [&] {
    AB2_CUDA(cudaMemcpyAsync(G->d_P, params, sizeof(float) * kParams, cudaMemcpyHostToDevice, G->ctx->stream));
    k_gnn_wcopy<<<64, 256, 0, G->ctx->stream>>>(G->d_P, G->d_Wb);
    check_launch(G->ctx, "gnn_wcopy");
    AB2_CUDA(cudaStreamSynchronize(G->ctx->stream));
  });
}

int ab2_gnn_bind(ab2_gnn* G, const ab2_matrix* A) {
  if (!G || !A || A->n <= 0) return AB2_ERR_BAD_ARG;
  ab2_context* ctx = G->ctx;
  return guard(ctx, [&] {
    ctx_quiesce(ctx);
    release_binding(G);
    const int n = A->n;
    G->A = A;
    G->n = n;
    G->d_invd = dev_alloc<float>(ctx, (size_t)n);
    G->d_logd10 = dev_alloc<float>(ctx, (size_t)n);
    G->d_efeat = dev_alloc<float>(ctx, (size_t)A->nnz);
    G->d_tidx = dev_alloc<int>(ctx, (size_t)A->nnz);
    G->d_h = dev_alloc<bf16>(ctx, (size_t)(kLayers + 1) * n * kH);
    G->d_m = dev_alloc<bf16>(ctx, (size_t)kLayers * n * kH);
    G->d_rr = dev_alloc<double>(ctx, 1);
    G->d_dh = dev_alloc<float>(ctx, (size_t)n * kH);
    G->d_dh2 = dev_alloc<float>(ctx, (size_t)n * kH);
    G->d_dm = dev_alloc<float>(ctx, (size_t)n * kH);
    G->d_z = dev_alloc<double>(ctx, (size_t)n);
    G->d_d = dev_alloc<double>(ctx, (size_t)n);
    G->d_Ad = dev_alloc<double>(ctx, (size_t)n);
    G->d_Ae = dev_alloc<double>(ctx, (size_t)n);
    G->part_cap = std::max((long long)wgrad_grid(ctx, n) * (kH * kIn + kH), (long long)warp_grid(ctx, n) * 3 * kH);
    G->d_part = dev_alloc<float>(ctx, (size_t)G->part_cap);
    G->d_red = dev_alloc<float>(ctx, (size_t)(kH * kIn + kH));
    int* d_bad = dev_alloc<int>(ctx, 1);
    AB2_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), ctx->stream));
    k_gnn_prep<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, A->d_v, A->d_dcol, G->d_invd,
                                                          G->d_logd10, G->d_efeat, G->d_tidx, d_bad);
    check_launch(ctx, "gnn_prep");
    int bad = 0;
    AB2_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    dev_free(ctx, d_bad);
    if (bad) {
      release_binding(G);
      throw Error{AB2_ERR_BAD_ARG, bad & 1 ? "learned preconditioner needs a positive diagonal in every row"
                                           : "learned preconditioner needs a structurally symmetric matrix"};
    }
  });
}

int ab2_gnn_apply(ab2_gnn* G, const ab2_vector* r, ab2_vector* z) {
  if (!G || !r || !z || !G->A || r->n != G->n || z->n != G->n || r->d == z->d) return AB2_ERR_BAD_ARG;
  return guard(G->ctx, [&] { gnn_forward(G, r->d, z->d); });
}

int ab2_gnn_loss_grad(ab2_gnn* G, const ab2_vector* r, const ab2_vector* e, double* loss, float* grad) {
  if (!G || !r || !e || !G->A || r->n != G->n || e->n != G->n) return AB2_ERR_BAD_ARG;
  return guard(G->ctx, [&] {
    const double L = gnn_loss_grad(G, r->d, e->d);
    if (loss) *loss = L;
    if (grad) {
      AB2_CUDA(cudaMemcpyAsync(grad, G->d_grad, sizeof(float) * kParams, cudaMemcpyDeviceToHost, G->ctx->stream));
      AB2_CUDA(cudaStreamSynchronize(G->ctx->stream));
    }
  });
}

int ab2_gnn_train_step(ab2_gnn* G, const ab2_vector* r, const ab2_vector* e, double lr, double* loss) {
  if (!G || !r || !e || !G->A || r->n != G->n || e->n != G->n || !(lr >= 0)) return AB2_ERR_BAD_ARG;
  ab2_context* ctx = G->ctx;
  return guard(ctx, [&] {
    const double L = gnn_loss_grad(G, r->d, e->d);
    if (loss) *loss = L;
    G->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)G->step), c2 = 1.f - std::pow(b2, (float)G->step);
    k_gnn_adam<<<(kParams + 255) / 256, 256, 0, ctx->stream>>>(kParams, G->d_P, G->d_grad, G->d_am, G->d_av, (float)lr,
                                                               b1, b2, 1e-8f, c1, c2);
    check_launch(ctx, "gnn_adam");
    k_gnn_wcopy<<<64, 256, 0, ctx->stream>>>(G->d_P, G->d_Wb);
    check_launch(ctx, "gnn_wcopy");
  });
}

int ab2_gnn_destroy(ab2_gnn* G) {
  if (!G) return AB2_ERR_BAD_ARG;
  if (G->ctx) {
    ctx_quiesce(G->ctx);
    release_binding(G);
    for (void* p : {(void*)G->d_P, (void*)G->d_grad, (void*)G->d_am, (void*)G->d_av, (void*)G->d_Wb})
      dev_free(G->ctx, p);
    ctx_release(G->ctx);
  }
  delete G;
  return AB2_OK;
}

void ab2_fcg_options_default(ab2_fcg_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->tol = 1e-8;
  o->max_iter = 5000;
  o->fallback_ratio = 1.0;
}

// Flexible CG (Polak-Ribiere beta, as the preconditioner changes between
// steps): z = network(r) while the network's steps reduce ||r|| by at least
// the factor fallback_ratio, the fallback preconditioner from the first step
// that does not (for the rest of the solve).  No network: the fallback only.
int ab2_fcg_solve(ab2_context* ctx, const ab2_matrix* A, ab2_gnn* G, const ab2_precond* fallback,
                  const ab2_vector* b, ab2_vector* x, const ab2_fcg_options* o, ab2_fcg_status* st) {
  if (!ctx || !A || !b || !x || !o || !st || b->n != A->n || x->n != A->n) return AB2_ERR_BAD_ARG;
  if (!G && !fallback) return AB2_ERR_BAD_ARG;
  if (G && (G->A != A)) return AB2_ERR_BAD_ARG;
  if (fallback && fallback->A != A) return AB2_ERR_BAD_ARG;
  std::memset(st, 0, sizeof(*st));
  st->switched_at = -1;
  return guard(ctx, [&] {
    const int n = A->n;
    cudaEvent_t e0, e1;
    AB2_CUDA(cudaEventCreate(&e0));
    AB2_CUDA(cudaEventCreate(&e1));
    AB2_CUDA(cudaEventRecord(e0, ctx->stream));
    double* r = dev_alloc<double>(ctx, (size_t)n);
    double* rp = dev_alloc<double>(ctx, (size_t)n);
    double* z = dev_alloc<double>(ctx, (size_t)n);
    double* p = dev_alloc<double>(ctx, (size_t)n);
    double* q = dev_alloc<double>(ctx, (size_t)n);
    double* s = red_slot(ctx, 7).result;
    auto dot = [&](const double* u, const double* v) {
      op_dot(ctx, n, u, v, s, 7);
      return read_scalar(ctx, s);
    };
    bool use_gnn = G != nullptr;
    auto precond = [&](const double* in, double* out) {
      if (use_gnn) {
        gnn_forward(G, in, out);
        st->gnn_steps += 1;
      } else {
        pc_apply(ctx, fallback, in, out);
        if (pc_error(ctx, fallback)) {
          pc_reset(ctx, fallback);
          throw Error{AB2_ERR_TIMEOUT, "fallback preconditioner: a bounded wait gave up"};
        }
        st->fallback_steps += 1;
      }
    };
    const double nb = std::sqrt(dot(b->d, b->d));
    op_spmv(ctx, A, x->d, q, AB2_SPMV_AUTO);
    op_copy(ctx, n, b->d, r);
    op_axpy(ctx, n, -1.0, q, r);
    double rn = std::sqrt(dot(r, r));
    int it = 0;
    bool ok = nb == 0.0 || rn / nb < o->tol;
    if (!ok) {
      precond(r, z);
      op_copy(ctx, n, z, p);
      double rz = dot(r, z);
      while (it < o->max_iter) {
        op_spmv(ctx, A, p, q, AB2_SPMV_AUTO);
        const double pq = dot(p, q);
        if (pq == 0.0) {
          st->error = AB2_ERR_BREAKDOWN;
          break;
        }
        const double alpha = rz / pq;
        op_axpy(ctx, n, alpha, p, x->d);
        op_copy(ctx, n, r, rp);
        op_axpy(ctx, n, -alpha, q, r);
        ++it;
        const double rn_new = std::sqrt(dot(r, r));
        if (rn_new / nb < o->tol) {
          ok = true;
          rn = rn_new;
          break;
        }
        if (use_gnn && fallback && rn_new > o->fallback_ratio * rn) {
          use_gnn = false;  // ILU(0) takes over from here
          st->switched_at = it;
        }
        rn = rn_new;
        precond(r, z);
        op_axpy(ctx, n, -1.0, r, rp);  // rp = r_old - r_new
        const double beta = -dot(z, rp) / rz;
        rz = dot(r, z);
        op_aypx(ctx, n, beta, p, z);   // p = beta p + z
      }
    }
    AB2_CUDA(cudaEventRecord(e1, ctx->stream));
    AB2_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    AB2_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    op_spmv(ctx, A, x->d, q, AB2_SPMV_AUTO);
    op_copy(ctx, n, b->d, r);
    op_axpy(ctx, n, -1.0, q, r);
    st->true_residual = nb > 0 ? std::sqrt(dot(r, r)) / nb : 0.0;
    st->succeeded = ok ? 1 : 0;
    st->iterations = it;
    st->solve_ms = ms;
    if (!ok && st->error == AB2_OK) st->error = AB2_ERR_NOT_CONVERGED;
    for (double* v : {r, rp, z, p, q}) dev_free(ctx, v);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  });
}

}  // extern "C"
