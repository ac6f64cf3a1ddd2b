// gnn.cu -- the learned preconditioner: a message-passing network on the
// matrix graph, its training kernels, and flexible CG with ILU(0) fallback.
// No counterpart in the reference; the network is defined (and checked) by
// oracle/gnn_oracle.py.  It works on the diagonal-scaled system
// D^-1/2 A D^-1/2, so neither inputs nor outputs carry the coefficients'
// orders of magnitude:
//   xr_i = r_i / sqrt(a_ii), s = rms(xr); x0_i = [xr_i/s, log(a_ii)/10]
//   h1 = relu(W0 x0 + b0)                                                      (2 -> 64)
//   4 x { g_ij = sigmoid(u e_ij + c), e_ij = log|a_ij| - (log a_ii + log a_jj)/2 ;
//         m_i = sum_j g_ij h_j ; h <- relu(W [h; m] + b) }                       (128 -> 64)
//   z_i = s (wd . h5_i + bd + ws x0_i) / sqrt(a_ii)       (ws: the Jacobi skip)
// Activations are stored in BF16 ([n][64], 128 B per node).  Each layer is
// one fused kernel: neighbour gather, BF16 x BF16 -> FP32 tensor-core MMAs
// (mma.sync m16n8k16; a warp computes 16 nodes x 64 outputs over K = 128) and
// the bias/relu epilogue; the first layer recomputes h1 from x0 instead of
// reading it, the last one applies the decoder in its epilogue, so inference
// moves about 2 x 128 B per node and layer.  Training: hand-written backward kernels (loss
// (z-e)^T A (z-e) / e^T A e on (residual, error) pairs), per-block partial
// sums reduced in a fixed order (deterministic), Adam on FP32 master weights
// with BF16 copies for the forward.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include "ab2_internal.cuh"
#include "precond.cuh"
#include "reduce.cuh"
#include "sentinel.cuh"
#include "spmv_view.cuh"
#include "tcgen05.cuh"

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
constexpr int kOffWs = kOffBd + 1;
constexpr int kParams = kOffWs + 1;

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
// Per row: 1/sqrt(a_ii) and log(a_ii)/10; per CSR entry the edge feature
// log|a_ij| - (log a_ii + log a_jj)/2 (the entry of D^-1/2 A D^-1/2) and the
// position of the transposed entry (the pattern must be structurally
// symmetric).  bad |= 1: a row without a positive diagonal; |= 2: no (j, i).
__device__ __forceinline__ bool diag_of(int r, const int* __restrict__ rp, const int* __restrict__ ci,
                                        const double* __restrict__ v, const int* __restrict__ dcol, double* d) {
  const int dk = dcol[r];
  if (dk < rp[r + 1] && ci[dk] == r && v[dk] > 0) {
    *d = v[dk];
    return true;
  }
  return false;
}

__global__ void k_gnn_prep(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                           const int* __restrict__ dcol, float* __restrict__ isd, float* __restrict__ logd10,
                           float* __restrict__ efeat, int* __restrict__ tidx, int* bad) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 1.0;
    if (!diag_of(i, rp, ci, v, dcol, &d)) {
      atomicOr(bad, 1);
      continue;
    }
    isd[i] = (float)(1.0 / sqrt(d));
    logd10[i] = (float)(log(d) / 10.0);
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = ci[k];
      if (j == i) {
        efeat[k] = 0.f;
        tidx[k] = -1;
        continue;
      }
      double dj = 1.0;
      if (!diag_of(j, rp, ci, v, dcol, &dj)) atomicOr(bad, 1);
      efeat[k] = (float)(log(fabs(v[k])) - 0.5 * (log(d) + log(dj)));
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

// The forward pass reads the graph as a padded neighbour table: per node nbw
// (a multiple of 8) slots of (column, edge feature) in CSR order, -1 marking
// padding -- one 32-byte load per 8 neighbours instead of a row-pointer load
// followed by dependent column loads.
__global__ void k_gnn_nbr(int n, const int* __restrict__ rp, const int* __restrict__ ci, const float* __restrict__ efeat,
                          int nbw, int* __restrict__ nb_idx, float* __restrict__ nb_ef) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int w = 0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      if (ci[k] == i) continue;
      nb_idx[(size_t)i * nbw + w] = ci[k];
      nb_ef[(size_t)i * nbw + w] = efeat[k];
      ++w;
    }
    for (; w < nbw; ++w) {
      nb_idx[(size_t)i * nbw + w] = -1;
      nb_ef[(size_t)i * nbw + w] = 0.f;
    }
  }
}

// The grid layer's edge features: per node (rows padded to whole 128-node
// tiles) the feature of each direction -nx ny, -nx, -1, +1, +nx, +nx ny (the
// CSR column order), NaN where the row has no entry there.
__global__ void k_gnn_dir_table(int n, long long rows, int nx, int sxy, const int* __restrict__ rp,
                                const int* __restrict__ ci, const float* __restrict__ efeat, float* __restrict__ tab) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < rows; i += (long long)gridDim.x * blockDim.x) {
    float e[6];
#pragma unroll
    for (int d = 0; d < 6; ++d) e[d] = __int_as_float(0x7fc00000);
    if (i < n) {
      for (int k = rp[i]; k < rp[i + 1]; ++k) {
        const long long off = (long long)ci[k] - i;
        const int d = off == -sxy ? 0 : off == -nx ? 1 : off == -1 ? 2 : off == 1 ? 3 : off == nx ? 4 : off == sxy ? 5 : -1;
        if (d >= 0) e[d] = efeat[k];
      }
    }
#pragma unroll
    for (int d = 0; d < 6; ++d) tab[i * 6 + d] = e[d];
  }
}

// ------------------------------------------------------------------ forward
// xr_i = r_i / sqrt(a_ii) (FP32) and s = rms(xr): s2[0] = s, s2[1] = 1/s (0 if s = 0).
__global__ void __launch_bounds__(kThreads) k_gnn_scale(int n, const double* __restrict__ r, const float* __restrict__ isd,
                                                        float* __restrict__ xr, double* partials, unsigned* counter,
                                                        double* red_out, double* s2) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float t = (float)(r[i] * (double)isd[i]);
    xr[i] = t;
    acc[0] = fma((double)t, (double)t, acc[0]);
  }
  if (grid_reduce<1>(acc, partials, counter, red_out)) {
    const double s = sqrt(red_out[0] / (double)max(n, 1));
    s2[0] = s;
    s2[1] = s > 0 ? 1.0 / s : 0.0;
  }
}

// One message-passing layer, fused, on tensor cores for both of its products:
//   m = G H_nb       (G: the 16 nodes' gates as a 16 x K BF16 matrix, one
//                     nonzero run per row; H_nb: the K = 16 nbw neighbour rows)
//   h_out = relu(W [h ; m] + b)
// A warp takes 16 nodes at a time (persistent: it walks the tiles with a
// stride).  The neighbour rows (padding slots zero-filled) are copied into the
// warp's shared memory with cp.async, 8 lanes per 128-byte row so that every
// copy instruction moves 4 whole rows.  The neighbour-table entries of the
// warp's next tile are loaded while the current one computes, so a tile waits
// on one memory latency.  Gates are computed one (node, slot) pair per lane
// and shuffled straight into A fragments (G is block diagonal: row g of a
// 16-column chunk is nonzero only where the chunk's pairs belong to node g).
// The aggregation is K/16 mma.sync m16n8k16 steps (B from the neighbour rows
// via ldmatrix.trans); its FP32 accumulators, rounded to BF16, are already in
// the A-fragment layout of the dense layer's last four k-steps; the own rows'
// fragments are read from global memory.  W (64 x 128, BF16) is staged once
// per CTA and read with ldmatrix.  Epilogue: bias, relu, BF16, 128-byte row
// stores through shared memory; LAST fuses the decoder
// z_i = s (wd . h5_i + bd + ws x0_i) / sqrt(a_ii).
// Optional stores (training): m_out, h_out (LAST).
struct LayerArgs {
  int n;
  int nbw;              // neighbour slots per node (even, <= kMaxNbw)
  const int* nb_idx;    // [n][nbw], -1 = padding
  const float* nb_ef;   // [n][nbw] edge features
  const float* P;       // FP32 parameters
  const bf16* W;        // this layer's W in BF16 (64 x 128, row = output)
  int layer;
  const bf16* h_in;     // h_l
  const float* xr;      // r_i / sqrt(a_ii)
  const float* isd;
  const double* s2;     // s, 1/s
  bf16* m_out;          // m_l (or null)
  bf16* h_out;          // h_{l+1} (or null when LAST)
  double* z;            // LAST: the network's output
};

constexpr int kMaxNbw = 16;
constexpr int kMaxRounds = kMaxNbw / 2;  // 32 (node, slot) pairs a round
constexpr int kLayerWarps = 4;
constexpr int kRowStride = kH + 8;       // bf16: 144-byte rows, conflict-free ldmatrix
__host__ __device__ constexpr int agg_k(int nbw) { return 16 * nbw; }  // nbw even: a multiple of 32
size_t layer_smem_bytes(int nbw) {
  return sizeof(bf16) * ((size_t)kH * kWStride + (size_t)kLayerWarps * agg_k(nbw) * kRowStride) +
         sizeof(float) * 2 * kH;
}

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool fill) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(fill ? 16 : 0));
}
__device__ __forceinline__ void ldsm_x4(unsigned (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(unsigned (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(smem_u32(p)));
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
// (acc0, acc1) += g * (lo(w), hi(w)) as one packed FP32 FMA (fma.rn.f32x2):
// a BF16 value is the high half of its FP32 value, so the halves of w unpack
// with a shift and a mask; each product is exact and each sum rounds once.
__device__ __forceinline__ void fma2_bf16_pair(float& acc0, float& acc1, float g, unsigned w) {
  const float lo = __uint_as_float(w << 16), hi = __uint_as_float(w & 0xffff0000u);
  asm("{\n\t.reg .b64 a, x, y;\n\t"
      "mov.b64 a, {%0, %1};\n\t"
      "mov.b64 x, {%2, %3};\n\t"
      "mov.b64 y, {%4, %4};\n\t"
      "fma.rn.f32x2 a, y, x, a;\n\t"
      "mov.b64 {%0, %1}, a;\n\t}"
      : "+f"(acc0), "+f"(acc1)
      : "f"(lo), "f"(hi), "f"(g));
}
// Shared-memory words at 32-bit shared addresses.
__device__ __forceinline__ float lds_f32(unsigned a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ void lds_f32x2(unsigned a, float& x, float& y) {
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(x), "=f"(y) : "r"(a));
}
__device__ __forceinline__ void sts_f32(unsigned a, float v) {
  asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
// 16 bytes of shared memory at a 32-bit shared address.
__device__ __forceinline__ uint4 lds128(unsigned a) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
  return v;
}
__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
  return make_uint4(pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]), pack_bf16(f[6], f[7]));
}

template <bool LAST>
__global__ void __launch_bounds__(kLayerWarps * 32) k_gnn_layer(const LayerArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  bf16* Ws = reinterpret_cast<bf16*>(smem);
  float* bs = reinterpret_cast<float*>(Ws + kH * kWStride);
  float* wds = bs + kH;
  for (int t = threadIdx.x; t < kH * kIn / 8; t += blockDim.x)
    *reinterpret_cast<uint4*>(Ws + (t >> 4) * kWStride + (t & 15) * 8) = reinterpret_cast<const uint4*>(a.W)[t];
  for (int t = threadIdx.x; t < kH; t += blockDim.x) {
    bs[t] = a.P[kOffB + a.layer * kH + t];
    wds[t] = a.P[kOffWd + t];
  }
  __syncthreads();
  const unsigned kFull = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nbw = a.nbw, K = agg_k(nbw), rounds = K / 32;
  bf16* Nb = reinterpret_cast<bf16*>(wds + kH) + warp * K * kRowStride;  // neighbour rows [K][kRowStride]
  const float u = a.P[kOffU + a.layer], c = a.P[kOffC + a.layer];
  const int g = lane >> 2, t = lane & 3;
  const int lrow = (lane & 7) + ((lane >> 3) & 1) * 8, lcol = (lane >> 4) * 8;  // ldmatrix x4 lane address
  const int wrow = (lane & 7) + (lane >> 4) * 8, wcol = ((lane >> 3) & 1) * 8;  // W fragments
  const int ntiles = (a.n + 15) / 16;
  const int stride = gridDim.x * kLayerWarps;
  // neighbour-table entries of pair 32 r + lane of a tile
  int pidx[kMaxRounds];
  float pef[kMaxRounds];
  auto fetch = [&](int tile) {
#pragma unroll
    for (int r = 0; r < kMaxRounds; ++r) {
      pidx[r] = -1;
      pef[r] = 0.f;
      const long long e = (long long)tile * 16 * nbw + 32 * r + lane;
      if (r < rounds && tile < ntiles && e < (long long)a.n * nbw) {
        pidx[r] = a.nb_idx[e];
        pef[r] = a.nb_ef[e];
      }
    }
  };
  fetch(blockIdx.x * kLayerWarps + warp);
  for (int tile = blockIdx.x * kLayerWarps + warp; tile < ntiles; tile += stride) {
    const int base = tile * 16;
    // ---- neighbour rows into shared memory; gates of this lane's pairs
    float gr[kMaxRounds];
#pragma unroll
    for (int r = 0; r < kMaxRounds; ++r) {
      gr[r] = 0.f;
      if (r < rounds) {
        const int j = pidx[r];
        if (j >= 0) gr[r] = bf16r(sigmoidf(fmaf(u, pef[r], c)));
#pragma unroll
        for (int q = 0; q < 8; ++q) {  // rows 32 r + 4 q .. + 3, 8 lanes each
          const int src = q * 4 + (lane >> 3);
          const int jj = __shfl_sync(kFull, j, src);
          cp_async16(Nb + (32 * r + src) * kRowStride + (lane & 7) * 8,
                     a.h_in + (size_t)max(jj, 0) * kH + (lane & 7) * 8, jj >= 0);
        }
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    fetch(tile + stride);  // the next tile's table entries, in flight during this tile
    // own rows' A fragments (k-steps 0..3) straight from global memory
    unsigned hA[4][4];
    {
      const unsigned* hv = reinterpret_cast<const unsigned*>(a.h_in);
      const int r0 = base + g, r1 = r0 + 8;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        const int col = ks * 16 + 2 * t;
        hA[ks][0] = r0 < a.n ? __ldg(hv + (((size_t)r0 * kH + col) >> 1)) : 0u;
        hA[ks][1] = r1 < a.n ? __ldg(hv + (((size_t)r1 * kH + col) >> 1)) : 0u;
        hA[ks][2] = r0 < a.n ? __ldg(hv + (((size_t)r0 * kH + col + 8) >> 1)) : 0u;
        hA[ks][3] = r1 < a.n ? __ldg(hv + (((size_t)r1 * kH + col + 8) >> 1)) : 0u;
      }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncwarp();
    // ---- aggregation m = G H_nb on tensor cores
    float accm[8][4];
#pragma unroll
    for (int nb = 0; nb < 8; ++nb) accm[nb][0] = accm[nb][1] = accm[nb][2] = accm[nb][3] = 0.f;
#pragma unroll
    for (int r = 0; r < kMaxRounds; ++r) {
      if (r < rounds) {
#pragma unroll
        for (int hlf = 0; hlf < 2; ++hlf) {
          const int k0 = 32 * r + 16 * hlf;
          // pairs k0 + 2t (+1) and k0 + 2t + 8 (+1): gates from lanes 16 hlf + 2t + {0, 1, 8, 9}
          const float g0 = __shfl_sync(kFull, gr[r], 16 * hlf + 2 * t);
          const float g1 = __shfl_sync(kFull, gr[r], 16 * hlf + 2 * t + 1);
          const float g8 = __shfl_sync(kFull, gr[r], 16 * hlf + 2 * t + 8);
          const float g9 = __shfl_sync(kFull, gr[r], 16 * hlf + 2 * t + 9);
          const int na = (k0 + 2 * t) / nbw, nc = (k0 + 2 * t + 8) / nbw;  // their nodes
          const unsigned pa = pack_bf16(g0, g1), pc = pack_bf16(g8, g9);
          const unsigned af[4] = {na == g ? pa : 0u, na == g + 8 ? pa : 0u, nc == g ? pc : 0u, nc == g + 8 ? pc : 0u};
#pragma unroll
          for (int n0 = 0; n0 < kH; n0 += 16) {
            unsigned bf[4];
            ldsm_x4_t(bf, Nb + (k0 + lrow) * kRowStride + n0 + lcol);
            mma_bf16(accm[n0 / 8], af, bf[0], bf[1]);
            mma_bf16(accm[n0 / 8 + 1], af, bf[2], bf[3]);
          }
        }
      }
    }
    // m in BF16, already laid out as the A fragments of k-steps 4..7
    unsigned mA[4][4];
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      mA[ks][0] = pack_bf16(accm[2 * ks][0], accm[2 * ks][1]);
      mA[ks][1] = pack_bf16(accm[2 * ks][2], accm[2 * ks][3]);
      mA[ks][2] = pack_bf16(accm[2 * ks + 1][0], accm[2 * ks + 1][1]);
      mA[ks][3] = pack_bf16(accm[2 * ks + 1][2], accm[2 * ks + 1][3]);
    }
    // ---- dense layer [h ; m] W^T on tensor cores
    float acc[8][4];
#pragma unroll
    for (int nb = 0; nb < 8; ++nb) acc[nb][0] = acc[nb][1] = acc[nb][2] = acc[nb][3] = 0.f;
#pragma unroll
    for (int ks = 0; ks < 8; ++ks) {
#pragma unroll
      for (int n0 = 0; n0 < kH; n0 += 16) {
        unsigned bf[4];
        ldsm_x4(bf, Ws + (n0 + wrow) * kWStride + ks * 16 + wcol);
        const unsigned(&af)[4] = ks < 4 ? hA[ks] : mA[ks - 4];
        mma_bf16(acc[n0 / 8], af, bf[0], bf[1]);
        mma_bf16(acc[n0 / 8 + 1], af, bf[2], bf[3]);
      }
    }
    __syncwarp();  // every lane is done with the neighbour rows: rows 0..31 stage the outputs
    bf16* Ms = Nb;
    bf16* Hs = Nb + 16 * kRowStride;
    if (a.m_out) {
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        *reinterpret_cast<unsigned*>(Ms + g * kRowStride + ks * 16 + 2 * t) = mA[ks][0];
        *reinterpret_cast<unsigned*>(Ms + (g + 8) * kRowStride + ks * 16 + 2 * t) = mA[ks][1];
        *reinterpret_cast<unsigned*>(Ms + g * kRowStride + ks * 16 + 8 + 2 * t) = mA[ks][2];
        *reinterpret_cast<unsigned*>(Ms + (g + 8) * kRowStride + ks * 16 + 8 + 2 * t) = mA[ks][3];
      }
      __syncwarp();
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int idx = q * 32 + lane, row = idx >> 3, c8 = idx & 7;
        if (base + row < a.n)
          reinterpret_cast<uint4*>(a.m_out + (size_t)(base + row) * kH)[c8] =
              *reinterpret_cast<const uint4*>(Ms + row * kRowStride + c8 * 8);
      }
    }
    // ---- epilogue: bias, relu, BF16
    float y0 = 0.f, y1 = 0.f;
    unsigned o0[8], o1[8];
#pragma unroll
    for (int nb = 0; nb < 8; ++nb) {
      const int cc = nb * 8 + 2 * t;
      const float h00 = bf16r(fmaxf(acc[nb][0] + bs[cc], 0.f)), h01 = bf16r(fmaxf(acc[nb][1] + bs[cc + 1], 0.f));
      const float h10 = bf16r(fmaxf(acc[nb][2] + bs[cc], 0.f)), h11 = bf16r(fmaxf(acc[nb][3] + bs[cc + 1], 0.f));
      o0[nb] = pack_bf16(h00, h01);
      o1[nb] = pack_bf16(h10, h11);
      if constexpr (LAST) {
        y0 = fmaf(wds[cc], h00, fmaf(wds[cc + 1], h01, y0));
        y1 = fmaf(wds[cc], h10, fmaf(wds[cc + 1], h11, y1));
      }
    }
    if (a.h_out) {
#pragma unroll
      for (int nb = 0; nb < 8; ++nb) {
        *reinterpret_cast<unsigned*>(Hs + g * kRowStride + nb * 8 + 2 * t) = o0[nb];
        *reinterpret_cast<unsigned*>(Hs + (g + 8) * kRowStride + nb * 8 + 2 * t) = o1[nb];
      }
      __syncwarp();
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int idx = q * 32 + lane, row = idx >> 3, c8 = idx & 7;
        if (base + row < a.n)
          reinterpret_cast<uint4*>(a.h_out + (size_t)(base + row) * kH)[c8] =
              *reinterpret_cast<const uint4*>(Hs + row * kRowStride + c8 * 8);
      }
    }
    if constexpr (LAST) {
      y0 += __shfl_xor_sync(kFull, y0, 1);
      y0 += __shfl_xor_sync(kFull, y0, 2);
      y1 += __shfl_xor_sync(kFull, y1, 1);
      y1 += __shfl_xor_sync(kFull, y1, 2);
      if (t == 0) {
        const double s = a.s2[0], is = a.s2[1];
        const float bd = a.P[kOffBd], ws = a.P[kOffWs];
        const int r0 = base + g, r1 = r0 + 8;
        if (r0 < a.n) a.z[r0] = s * (double)(y0 + bd + ws * (float)(a.xr[r0] * is)) * (double)a.isd[r0];
        if (r1 < a.n) a.z[r1] = s * (double)(y1 + bd + ws * (float)(a.xr[r1] * is)) * (double)a.isd[r1];
      }
    }
    __syncwarp();  // the staging rows are refilled by the next tile's copies
  }
}

// ------------------------------------------------------------------ layer on a 3-D grid (tcgen05)
// The same layer for a matrix whose graph is a 3-D 7-point grid in
// lexicographic order (row i + nx (j + ny k), off-diagonal columns at -nx ny,
// -nx, -1, +1, +nx, +nx ny where inside the grid): 128 consecutive nodes a
// tile, so each direction's neighbour rows form one contiguous block of h and
// nothing is gathered by index.  A persistent CTA (one an SM) walks tiles with
// its warps in three roles that hand tiles on through mbarriers, so one
// tile's MMA and epilogue overlap the next tile's aggregation:
//   - control (one thread): issues each tile's inputs by bulk copy
//     (cp.async.bulk, no multicast) two tiles ahead into a two-stage ring --
//     the tile's own rows with one row either side (the +-1 neighbours), the
//     four +-nx / +-nx ny blocks, and the edge features in direction order
//     (NaN where no neighbour) -- and, once a tile's A operand is complete and
//     an accumulator buffer is free, eight tcgen05.mma (M = 128, N = 64,
//     K = 16) into that buffer (two 128 x 64 FP32 accumulators in tensor
//     memory); B is W (64 x 128 BF16), staged once per CTA;
//   - aggregation (16 warps): the gates sigmoid(u e + c) once per (node,
//     direction), then m = sum_d g_d h_nbr(d), four threads a node and two
//     8-feature chunks a thread
//     (BF16 x BF16 products, FP32 sums in the CSR column order, rounded to
//     BF16 as the tensor-core aggregation of k_gnn_layer is; absent neighbours
//     read a row of zeros), held in registers until the tensor core has
//     released A, then [h ; m] written as A (128 x 128 BF16, 128-byte swizzle);
//   - epilogue (4 warps, one a tensor-memory lane quarter): a row a thread,
//     bias, relu, BF16, stored to h (LAST: the decoder's z instead).
// Every wait is bounded: on expiry the kernel sets *err, every role stops at
// its next tile, and the CTA waits (bounded) for the copies and the MMA it
// issued and frees its tensor memory before it returns.
constexpr int kTcAggWarps = 16;
constexpr int kTcEpiWarps = 4;
constexpr int kTcAggThreads = kTcAggWarps * 32;
constexpr int kTcEpiThreads = kTcEpiWarps * 32;
constexpr int kTcThreads = kTcAggThreads + kTcEpiThreads + 32;  // + the control warp
constexpr int kTcTile = 128;
constexpr unsigned kTcRowB = kH * 2;                         // bytes of one h row
constexpr unsigned kTcW = 0;                                 // B: 2 regions x 64 rows x 128 B
constexpr unsigned kTcA = kTcW + 2 * kH * kTcRowB;           // A: 2 regions x 128 rows x 128 B
constexpr unsigned kTcARegion = kTcTile * kTcRowB;
constexpr unsigned kTcStage0 = kTcA + 2 * kTcARegion;
constexpr unsigned kTcXOff = 0;                              // rows b-1 .. b+128
constexpr unsigned kTcYmOff = kTcXOff + (kTcTile + 2) * kTcRowB;
constexpr unsigned kTcYpOff = kTcYmOff + kTcARegion;
constexpr unsigned kTcZmOff = kTcYpOff + kTcARegion;
constexpr unsigned kTcZpOff = kTcZmOff + kTcARegion;
constexpr unsigned kTcEfOff = kTcZpOff + kTcARegion;         // 128 x 6 floats
constexpr unsigned kTcEfBytes = kTcTile * 6 * 4;
constexpr unsigned kTcStageB = kTcEfOff + kTcEfBytes;
constexpr unsigned kTcStage1 = kTcStage0 + kTcStageB;
constexpr unsigned kTcBias = kTcStage1 + kTcStageB;          // bias, wd: 2 x 64 floats
constexpr unsigned kTcGate = kTcBias + 2 * kH * 4;           // gates (BF16 values as FP32): 2 tiles x 128 x 6
constexpr unsigned kTcGateB = kTcTile * 6 * 4;
constexpr unsigned kTcZero = kTcGate + 2 * kTcGateB;         // one row of zeros (absent neighbours)
constexpr unsigned kTcBar = kTcZero + kTcRowB;               // 8 mbarriers, tensor-memory address, abort flag
constexpr unsigned kTcSmem = kTcBar + 80 + 1024;             // + slack to align the base to 1024 bytes
constexpr unsigned kTcCols = 2 * kH;                         // tensor-memory columns: two accumulators
static_assert(kTcSmem <= 227 * 1024, "grid layer: shared memory");
static_assert(kTcStage0 % 1024 == 0 && kTcA % 1024 == 0 && kTcStageB % 16 == 0, "grid layer: alignment");
static_assert(kTcAggThreads == kTcTile * 4, "grid layer: four aggregation threads a node");

struct GridLayerArgs {
  LayerArgs a;
  int nx, sxy;           // grid strides along j and k
  const float* dir_ef;   // [ceil(n/128) * 128][6] edge features by direction, NaN = none
  int* err;              // set when a bounded wait gives up
};

// Named barrier `id` over `count` threads that ORs a flag across them.
__device__ __forceinline__ int bar_or(int id, int count, int v) {
  int r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.s32 p, %1, 0;\n\t"
      "barrier.cta.red.or.pred q, %2, %3, p;\n\t"
      "selp.s32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"(v), "r"(id), "r"(count)
      : "memory");
  return r;
}

template <bool LAST>
__global__ void __launch_bounds__(kTcThreads, 1) k_gnn_layer_grid(const GridLayerArgs ga) {
  const LayerArgs& a = ga.a;
  extern __shared__ unsigned char tc_smem_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) &
                                                       ~static_cast<uintptr_t>(1023));
  const unsigned sb = tc::smem_u32(sm);
  float* s_bias = reinterpret_cast<float*>(sm + kTcBias);
  float* s_wd = s_bias + kH;
  // mbarriers: inputs of stage 0/1 landed; A written; A released by the
  // tensor core; accumulator 0/1 complete; accumulator 0/1 read
  const unsigned bar_full = sb + kTcBar, bar_afull = bar_full + 16, bar_aempty = bar_full + 24;
  const unsigned bar_accf = bar_full + 32, bar_acce = bar_full + 48;
  volatile unsigned* s_tmem = reinterpret_cast<volatile unsigned*>(sm + kTcBar + 64);
  volatile int* s_abort = reinterpret_cast<volatile int*>(sm + kTcBar + 68);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n = a.n;
  const int ntiles = (n + kTcTile - 1) / kTcTile;
  const int count = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto tile_base = [&](int c) { return (long long)((int)blockIdx.x + c * (int)gridDim.x) * kTcTile; };
  auto give_up = [&]() {
    *s_abort = 1;
    atomicOr(ga.err, 1);
  };

  // W as the B operand (row o = output feature, K-major, 128-byte swizzle)
  for (int t = tid; t < kH * kIn / 8; t += kTcThreads) {
    const int o = t >> 4, reg = (t >> 3) & 1, c = t & 7;
    *reinterpret_cast<uint4*>(sm + kTcW + reg * (kH * kTcRowB) + o * kTcRowB + ((c ^ (o & 7)) << 4)) =
        reinterpret_cast<const uint4*>(a.W)[t];
  }
  for (int t = tid; t < kH; t += kTcThreads) {
    s_bias[t] = a.P[kOffB + a.layer * kH + t];
    s_wd[t] = a.P[kOffWd + t];
  }
  if (tid < (int)kTcRowB / 16) reinterpret_cast<uint4*>(sm + kTcZero)[tid] = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) {
    tc::mbar_init(bar_full, 1);
    tc::mbar_init(bar_full + 8, 1);
    tc::mbar_init(bar_afull, kTcAggThreads);
    tc::mbar_init(bar_aempty, 1);
    tc::mbar_init(bar_accf, 1);
    tc::mbar_init(bar_accf + 8, 1);
    tc::mbar_init(bar_acce, kTcEpiThreads);
    tc::mbar_init(bar_acce + 8, kTcEpiThreads);
    *s_abort = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(sb + kTcBar + 64, kTcCols);
    tc::tmem_relinquish();
  }
  tc::fence_proxy_async_smem();  // W (generic stores) is read by the tensor core
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const unsigned tmem = *s_tmem;

  if (warp < kTcAggWarps) {
    // ================================================================ aggregation
    const float u = a.P[kOffU + a.layer], cg = a.P[kOffC + a.layer];
    int failed = 0;
    for (int c = 0; c < count; ++c) {
      const int s = c & 1;
      const long long b = tile_base(c);
      if (!tc::mbar_wait(bar_full + 8 * s, (unsigned)(c >> 1) & 1u, kWaitCycles, s_abort)) {
        failed = 1;
        give_up();
      }
      // gates, once per (node, direction), rounded to BF16 (0 where no neighbour)
      {
        const unsigned ef = sb + (s ? kTcStage1 : kTcStage0) + kTcEfOff, gt = sb + kTcGate + s * kTcGateB;
        for (int q = tid; q < kTcTile * 6; q += kTcAggThreads) {
          const float e = lds_f32(ef + 4 * q);
          sts_f32(gt + 4 * q, e == e ? bf16r(sigmoidf(fmaf(u, e, cg))) : 0.f);
        }
      }
      if (bar_or(1, kTcAggThreads, failed)) break;
      const int ln = tid >> 2, qq = tid & 3;  // node, and its chunks qq and qq + 4
      const unsigned sst = sb + (s ? kTcStage1 : kTcStage0) + ln * kTcRowB;  // this node's row of each block
      unsigned src[6] = {sst + kTcZmOff, sst + kTcYmOff, sst + kTcXOff, sst + kTcXOff + 2 * kTcRowB, sst + kTcYpOff,
                         sst + kTcZpOff};
      float g[6], e[6];
      {
        const unsigned efa = sb + (s ? kTcStage1 : kTcStage0) + kTcEfOff + ln * 24;
        const unsigned gta = sb + kTcGate + s * kTcGateB + ln * 24;
#pragma unroll
        for (int d = 0; d < 6; d += 2) {
          lds_f32x2(efa + 4 * d, e[d], e[d + 1]);
          lds_f32x2(gta + 4 * d, g[d], g[d + 1]);
        }
      }
#pragma unroll
      for (int d = 0; d < 6; ++d) src[d] = e[d] == e[d] ? src[d] : sb + kTcZero;
      uint4 hv[2], mv[2];
#pragma unroll
      for (int jj = 0; jj < 2; ++jj) {
        const int ch = 4 * ((ln & 1) ^ jj) + qq;  // the 8 threads of a quarter-warp touch 8 distinct banks
        float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int d = 0; d < 6; ++d) {
          const uint4 w = lds128(src[d] + ch * 16);
          fma2_bf16_pair(acc[0], acc[1], g[d], w.x);
          fma2_bf16_pair(acc[2], acc[3], g[d], w.y);
          fma2_bf16_pair(acc[4], acc[5], g[d], w.z);
          fma2_bf16_pair(acc[6], acc[7], g[d], w.w);
        }
        mv[jj] = pack8(acc);
        hv[jj] = b + ln < n ? lds128(sst + kTcXOff + kTcRowB + ch * 16) : make_uint4(0u, 0u, 0u, 0u);
      }
      // A is free once the tensor core has read the previous tile's
      if (c > 0 && !tc::mbar_wait(bar_aempty, (unsigned)(c - 1) & 1u, kWaitCycles, s_abort)) {
        failed = 1;
        give_up();
      }
#pragma unroll
      for (int jj = 0; jj < 2; ++jj) {
        const int ch = 4 * ((ln & 1) ^ jj) + qq;
        const unsigned pos = ln * kTcRowB + ((ch ^ (ln & 7)) << 4);
        *reinterpret_cast<uint4*>(sm + kTcA + pos) = hv[jj];
        *reinterpret_cast<uint4*>(sm + kTcA + kTcARegion + pos) = mv[jj];
        if (a.m_out && b + ln < n) reinterpret_cast<uint4*>(a.m_out + (b + ln) * kH)[ch] = mv[jj];
      }
      tc::fence_proxy_async_smem();
      tc::mbar_arrive(bar_afull);
    }
  } else if (warp < kTcAggWarps + kTcEpiWarps) {
    // ================================================================ epilogue
    const int q = warp & 3;  // the tensor-memory lane quarter this warp may read
    const int row = 32 * q + lane;
    for (int c = 0; c < count; ++c) {
      const int bsel = c & 1;
      const long long gi = tile_base(c) + row;
      int failed = !tc::mbar_wait(bar_accf + 8 * bsel, (unsigned)(c >> 1) & 1u, kWaitCycles, s_abort);
      if (__any_sync(0xffffffffu, failed)) {
        give_up();
        break;
      }
      tc::fence_after_sync();
      const unsigned ta = tmem + ((unsigned)(32 * q) << 16) + bsel * kH;
      float y = 0.f;
#pragma unroll
      for (int h = 0; h < 2; ++h) {  // 32 columns at a time
        float v[32];
        tc::tmem_ld32(ta + 32 * h, v);
        if (h == 1) {
          tc::fence_before_sync();
          tc::mbar_arrive(bar_acce + 8 * bsel);  // the accumulator is read
        }
        if (gi < n) {
#pragma unroll
          for (int j4 = 0; j4 < 8; ++j4) {
            const float4 bb = reinterpret_cast<const float4*>(s_bias)[8 * h + j4];
            const float bv[4] = {bb.x, bb.y, bb.z, bb.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) v[4 * j4 + e] = fmaxf(v[4 * j4 + e] + bv[e], 0.f);
            if constexpr (LAST) {
              const float4 ww = reinterpret_cast<const float4*>(s_wd)[8 * h + j4];
              const float wv[4] = {ww.x, ww.y, ww.z, ww.w};
#pragma unroll
              for (int e = 0; e < 4; ++e) y = fmaf(wv[e], bf16r(v[4 * j4 + e]), y);
            }
          }
          if (a.h_out) {
#pragma unroll
            for (int c8 = 0; c8 < 4; ++c8) {
              float f8[8];
#pragma unroll
              for (int e = 0; e < 8; ++e) f8[e] = v[8 * c8 + e];
              reinterpret_cast<uint4*>(a.h_out + gi * kH)[4 * h + c8] = pack8(f8);
            }
          }
        }
      }
      if constexpr (LAST) {
        if (gi < n) {
          const double s2 = a.s2[0], is = a.s2[1];
          const float bd = a.P[kOffBd], ws = a.P[kOffWs];
          a.z[gi] = s2 * (double)(y + bd + ws * (float)(a.xr[gi] * is)) * (double)a.isd[gi];
        }
      }
    }
  } else if (lane == 0) {
    // ================================================================ control
    // in flight, for the drain after a failure: the parity of each stage's
    // last issued phase and of the last MMA commit (-1: none)
    int last_in[2] = {-1, -1}, last_mma = -1;
    auto issue = [&](int c) {
      const int s = c & 1;
      const long long b = tile_base(c);
      const unsigned st = sb + (s ? kTcStage1 : kTcStage0);
      const long long first[5] = {b - 1, b - ga.nx, b + ga.nx, b - ga.sxy, b + ga.sxy};
      const int rows[5] = {kTcTile + 2, kTcTile, kTcTile, kTcTile, kTcTile};
      const unsigned dst[5] = {kTcXOff, kTcYmOff, kTcYpOff, kTcZmOff, kTcZpOff};
      long long lo[5], hi[5];
      unsigned bytes = kTcEfBytes;
      for (int k = 0; k < 5; ++k) {
        lo[k] = first[k] < 0 ? 0 : first[k];
        hi[k] = first[k] + rows[k] > n ? n : first[k] + rows[k];
        if (hi[k] > lo[k]) bytes += (unsigned)(hi[k] - lo[k]) * kTcRowB;
      }
      tc::mbar_expect_tx(bar_full + 8 * s, bytes);
      for (int k = 0; k < 5; ++k)
        if (hi[k] > lo[k])
          tc::bulk_g2s(st + dst[k] + (unsigned)(lo[k] - first[k]) * kTcRowB, a.h_in + lo[k] * kH,
                       (unsigned)(hi[k] - lo[k]) * kTcRowB, bar_full + 8 * s);
      tc::bulk_g2s(st + kTcEfOff, ga.dir_ef + b * 6, kTcEfBytes, bar_full + 8 * s);
      last_in[s] = (c >> 1) & 1;
    };
    for (int c = 0; c < 2 && c < count; ++c) issue(c);
    bool ok = true;
    for (int c = 0; c < count && ok; ++c) {
      const int bsel = c & 1;
      ok = tc::mbar_wait(bar_afull, (unsigned)c & 1u, kWaitCycles, s_abort);  // A of tile c written
      if (ok && c + 2 < count) issue(c + 2);  // stage c & 1 read by every aggregation thread
      if (ok && c >= 2)  // the epilogue has read this accumulator's previous tile
        ok = tc::mbar_wait(bar_acce + 8 * bsel, (unsigned)((c >> 1) - 1) & 1u, kWaitCycles, s_abort);
      if (!ok) {
        give_up();
        break;
      }
      tc::fence_after_sync();
      constexpr uint32_t idesc = tc::idesc_bf16_f32(kTcTile, kH);
#pragma unroll
      for (int k = 0; k < kIn / 16; ++k) {
        const unsigned aoff = (k >> 2) * kTcARegion + (k & 3) * 32, boff = (k >> 2) * (kH * kTcRowB) + (k & 3) * 32;
        tc::mma_bf16_ss(tmem + bsel * kH, tc::sdesc_sw128(sb + kTcA + aoff), tc::sdesc_sw128(sb + kTcW + boff), idesc,
                        k > 0);
      }
      tc::mma_commit(bar_aempty);
      tc::mma_commit(bar_accf + 8 * bsel);
      last_mma = c & 1;
    }
    if (!ok) {  // drain: nothing of this CTA's may still write its shared or tensor memory at exit
      for (int s = 0; s < 2; ++s)
        if (last_in[s] >= 0) tc::mbar_wait(bar_full + 8 * s, (unsigned)last_in[s], kWaitCycles, nullptr);
      if (last_mma >= 0) tc::mbar_wait(bar_aempty, (unsigned)last_mma, kWaitCycles, nullptr);
    }
  }
  __syncwarp();  // the control warp reconverges before the CTA barrier
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, kTcCols);
  }
}

// h1 = relu(W0 x0 + b0), x0 = [xr / s, log(a_ii)/10]: 8 lanes per node, 8 features a lane.
__global__ void __launch_bounds__(kThreads) k_gnn_encode(int n, const float* __restrict__ xr,
                                                         const float* __restrict__ logd10, const double* __restrict__ s2,
                                                         const float* __restrict__ P, bf16* __restrict__ h1) {
  const int sub = threadIdx.x & 7;
  const float inv_s = (float)s2[1];
  float w0a[8], w0b[8], b0v[8];
#pragma unroll
  for (int f = 0; f < 8; ++f) {
    w0a[f] = P[kOffW0 + 2 * (8 * sub + f)];
    w0b[f] = P[kOffW0 + 2 * (8 * sub + f) + 1];
    b0v[f] = P[kOffB0 + 8 * sub + f];
  }
  for (long long v = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 3; v < n;
       v += ((long long)gridDim.x * blockDim.x) >> 3) {
    const float x = xr[v] * inv_s, l = logd10[v];
    float f8[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) f8[q] = fmaxf(fmaf(w0a[q], x, fmaf(w0b[q], l, b0v[q])), 0.f);
    reinterpret_cast<uint4*>(h1 + (size_t)v * kH)[sub] = pack8(f8);
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

// dy_i = dz_i s / sqrt(a_ii) ; dh5_i = dy_i wd ; partials of grad wd (64), bd and ws.
__global__ void __launch_bounds__(256) k_gnn_decode_bwd(int n, const double* __restrict__ dz, const double* __restrict__ s2,
                                                        const float* __restrict__ isd, const float* __restrict__ xr,
                                                        const bf16* __restrict__ h5, const float* __restrict__ P,
                                                        float* __restrict__ dh, float* __restrict__ part) {
  __shared__ float s_acc[kWarpsPerBlock][kH + 2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double s = s2[0];
  const float is = (float)s2[1];
  const unsigned* hv = reinterpret_cast<const unsigned*>(h5);
  const float w0 = P[kOffWd + 2 * lane], w1 = P[kOffWd + 2 * lane + 1];
  float g0 = 0.f, g1 = 0.f, gb = 0.f, gs = 0.f;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
    const float dy = (float)(dz[i] * s * (double)isd[i]);
    const float2 x = unpack_bf16(hv[(size_t)i * (kH / 2) + lane]);
    g0 = fmaf(dy, x.x, g0);
    g1 = fmaf(dy, x.y, g1);
    gb += dy;
    gs = fmaf(dy, xr[i] * is, gs);
    reinterpret_cast<float2*>(dh)[(size_t)i * (kH / 2) + lane] = make_float2(dy * w0, dy * w1);
  }
  s_acc[warp][2 * lane] = g0;
  s_acc[warp][2 * lane + 1] = g1;
  if (lane == 0) {
    s_acc[warp][kH] = gb;
    s_acc[warp][kH + 1] = gs;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < kH + 2; k += blockDim.x) {
    float v = 0.f;
    for (int w = 0; w < kWarpsPerBlock; ++w) v += s_acc[w][k];
    part[(size_t)blockIdx.x * (kH + 2) + k] = v;
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
__global__ void __launch_bounds__(256) k_gnn_encode_bwd(int n, const float* __restrict__ xr, const double* __restrict__ s2,
                                                        const float* __restrict__ logd10, const bf16* __restrict__ h1,
                                                        const float* __restrict__ dh, float* __restrict__ part) {
  __shared__ float s_acc[kWarpsPerBlock][3 * kH];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float inv_s = (float)s2[1];
  const unsigned* hv = reinterpret_cast<const unsigned*>(h1);
  float a[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // (W0[o][0], W0[o][1], b0[o]) for o = 2 lane, 2 lane + 1
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
    const float x0 = xr[i] * inv_s, x1 = logd10[i];
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

// ------------------------------------------------------------------ flexible CG
// Notay's FCG(m): p_k = z_k - sum_i (z_k . q_i / d_i) p_i over the last m
// directions (q_i = A p_i, d_i = p_i . q_i), alpha_k = p_k . r_k / d_k.  The
// scalars stay on the device; one iteration needs a single host read (of rr,
// for the stop and fallback decisions).
constexpr int kMaxTrunc = 16;
struct FcgScalars {
  double rr;                // r . r after the update
  double alpha;
  double d[kMaxTrunc];      // p_i . A p_i, by window slot
  double coef[kMaxTrunc];   // z . A p_i / d_i of the current step
  int breakdown;            // p . A p == 0
};
struct Window {
  const double* v[kMaxTrunc];
};

// coef_k = z . q_k / d_k for the window's slots 0..count-1
__global__ void __launch_bounds__(kThreads) k_fcg_zq(int n, const double* __restrict__ z, const Window q, int count,
                                                     FcgScalars* sc, double* partials, unsigned* counter,
                                                     double* red_out) {
  double acc[kMaxTrunc];
#pragma unroll
  for (int k = 0; k < kMaxTrunc; ++k) acc[k] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double zi = z[i];
#pragma unroll
    for (int k = 0; k < kMaxTrunc; ++k)
      if (k < count) acc[k] = fma(zi, q.v[k][i], acc[k]);
  }
  if (grid_reduce<kMaxTrunc>(acc, partials, counter, red_out)) {
    for (int k = 0; k < count; ++k) sc->coef[k] = sc->d[k] != 0.0 ? red_out[k] / sc->d[k] : 0.0;
  }
}

// p = z - sum_k coef_k p_k (p may be one of the window's vectors: element-wise in place)
__global__ void k_fcg_dir(int n, const double* __restrict__ z, const Window pw, int count, const FcgScalars* sc,
                          double* p) {
  double coef[kMaxTrunc];
#pragma unroll
  for (int k = 0; k < kMaxTrunc; ++k) coef[k] = k < count ? sc->coef[k] : 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = z[i];
#pragma unroll
    for (int k = 0; k < kMaxTrunc; ++k)
      if (k < count) v = fma(-coef[k], pw.v[k][i], v);
    p[i] = v;
  }
}

// d_slot = p . q, alpha = p . r / d_slot (breakdown if d_slot == 0)
__global__ void __launch_bounds__(kThreads) k_fcg_pq(int n, const double* __restrict__ p, const double* __restrict__ q,
                                                     const double* __restrict__ r, int slot, FcgScalars* sc,
                                                     double* partials, unsigned* counter, double* red_out) {
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double pi = p[i];
    acc[0] = fma(pi, q[i], acc[0]);
    acc[1] = fma(pi, r[i], acc[1]);
  }
  if (grid_reduce<2>(acc, partials, counter, red_out)) {
    const double d = red_out[0];
    sc->d[slot] = d;
    sc->alpha = d != 0.0 ? red_out[1] / d : 0.0;
    if (d == 0.0) sc->breakdown = 1;
  }
}

// x += alpha p; r -= alpha q; rr = r . r
__global__ void __launch_bounds__(kThreads) k_fcg_update(int n, const double* __restrict__ p, const double* __restrict__ q,
                                                         double* __restrict__ x, double* __restrict__ r, FcgScalars* sc,
                                                         double* partials, unsigned* counter, double* red_out) {
  const double alpha = sc->alpha;
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = fma(alpha, p[i], x[i]);
    const double rv = fma(-alpha, q[i], r[i]);
    r[i] = rv;
    acc[0] = fma(rv, rv, acc[0]);
  }
  if (grid_reduce<1>(acc, partials, counter, red_out)) sc->rr = red_out[0];
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
  float *d_isd = nullptr, *d_logd10 = nullptr, *d_efeat = nullptr;
  int* d_tidx = nullptr;
  int nbw = 0;               // neighbour table: slots per node
  int* d_nb_idx = nullptr;
  float* d_nb_ef = nullptr;
  bf16* d_h = nullptr;       // h1..h5, n x 64 each
  bf16* d_m = nullptr;       // m1..m4
  float* d_xr = nullptr;     // r_i / sqrt(a_ii) of the last forward
  double* d_s2 = nullptr;    // its scale s and 1/s
  float *d_dh = nullptr, *d_dh2 = nullptr, *d_dm = nullptr;
  double *d_z = nullptr, *d_d = nullptr, *d_Ad = nullptr, *d_Ae = nullptr;
  float* d_part = nullptr;
  float* d_red = nullptr;    // reduced partials scratch (64 x 128 + 64)
  long long part_cap = 0;
  // the layer kernel: AB2_GNN_LAYER_* requested, and whether the bound
  // matrix's graph is a 3-D 7-point grid (then the grid layer's inputs)
  int layout = AB2_GNN_LAYER_AUTO;
  bool grid = false;
  int gnx = 0, gny = 0, gnz = 0;
  float* d_dir_ef = nullptr;  // [ceil(n/128) 128][6] edge features by direction
  int* d_err = nullptr;       // set by the grid layer when a bounded wait gives up
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
  for (void* p : {(void*)G->d_isd, (void*)G->d_logd10, (void*)G->d_efeat, (void*)G->d_tidx, (void*)G->d_h,
                  (void*)G->d_m, (void*)G->d_xr, (void*)G->d_s2, (void*)G->d_dh, (void*)G->d_dh2, (void*)G->d_dm,
                  (void*)G->d_z, (void*)G->d_d, (void*)G->d_Ad, (void*)G->d_Ae, (void*)G->d_part, (void*)G->d_red,
                  (void*)G->d_nb_idx, (void*)G->d_nb_ef, (void*)G->d_dir_ef, (void*)G->d_err})
    dev_free(ctx, p);
  G->d_dir_ef = nullptr;
  G->d_err = nullptr;
  G->grid = false;
  G->gnx = G->gny = G->gnz = 0;
  G->d_nb_idx = nullptr;
  G->d_nb_ef = nullptr;
  G->nbw = 0;
  G->d_isd = G->d_logd10 = G->d_efeat = G->d_xr = nullptr;
  G->d_tidx = nullptr;
  G->d_h = G->d_m = nullptr;
  G->d_s2 = nullptr;
  G->d_dh = G->d_dh2 = G->d_dm = nullptr;
  G->d_z = G->d_d = G->d_Ad = G->d_Ae = nullptr;
  G->d_part = G->d_red = nullptr;
  G->A = nullptr;
  G->n = 0;
}

template <bool LAST>
void launch_layer(ab2_context* ctx, const LayerArgs& la) {
  static thread_local int configured_device = -1, per_sm = 0, per_sm_nbw = -1;  // per device and table width
  if (configured_device != ctx->device) {
    AB2_CUDA(cudaFuncSetAttribute(k_gnn_layer<LAST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)layer_smem_bytes(kMaxNbw)));
    configured_device = ctx->device;
    per_sm_nbw = -1;
  }
  if (per_sm_nbw != la.nbw) {
    AB2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gnn_layer<LAST>, kLayerWarps * 32,
                                                           layer_smem_bytes(la.nbw)));
    per_sm = std::max(per_sm, 1);
    per_sm_nbw = la.nbw;
  }
  const int ntiles = (la.n + 15) / 16;
  const int grid = std::max(1, std::min((ntiles + kLayerWarps - 1) / kLayerWarps, per_sm * ctx->num_sms));
  k_gnn_layer<LAST><<<grid, kLayerWarps * 32, layer_smem_bytes(la.nbw), ctx->stream>>>(la);
  check_launch(ctx, "gnn_layer");
}

template <bool LAST>
void launch_layer_grid(ab2_context* ctx, const GridLayerArgs& ga) {
  static thread_local int configured_device = -1;
  if (configured_device != ctx->device) {
    AB2_CUDA(cudaFuncSetAttribute(k_gnn_layer_grid<LAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    configured_device = ctx->device;
  }
  const int ntiles = (ga.a.n + kTcTile - 1) / kTcTile;
  const int grid = std::max(1, std::min(ntiles, ctx->num_sms));
  k_gnn_layer_grid<LAST><<<grid, kTcThreads, kTcSmem, ctx->stream>>>(ga);
  check_launch(ctx, "gnn_layer_grid");
}

bool use_grid_layer(const ab2_gnn* G) { return G->grid && G->layout != AB2_GNN_LAYER_GATHER; }

// A bounded wait of the grid layer gave up (its outputs are then garbage):
// AB2_ERR_TIMEOUT, the flag cleared for the next call.  Synchronises.
void check_grid_wait(ab2_gnn* G) {
  if (!G->d_err) return;
  ab2_context* ctx = G->ctx;
  int e = 0;
  AB2_CUDA(cudaMemcpyAsync(&e, G->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  if (e) {
    AB2_CUDA(cudaMemsetAsync(G->d_err, 0, sizeof(int), ctx->stream));
    throw Error{AB2_ERR_TIMEOUT, "learned preconditioner: a bounded wait of the grid layer gave up"};
  }
}

// z = network(r) (FP64 in and out).  training: keep m1..m4 and h5 for the
// backward pass (h1..h4 are always written).
void gnn_forward(ab2_gnn* G, const double* r, double* z, bool training = false) {
  ab2_context* ctx = G->ctx;
  const int n = G->n;
  RedSlot red = red_slot(ctx, 5);
  k_gnn_scale<<<red_grid(ctx, n), kThreads, 0, ctx->stream>>>(n, r, G->d_isd, G->d_xr, red.partials, red.counter,
                                                             red.result, G->d_s2);
  check_launch(ctx, "gnn_scale");
  k_gnn_encode<<<grid_for((long long)n * 8), kThreads, 0, ctx->stream>>>(n, G->d_xr, G->d_logd10, G->d_s2, G->d_P,
                                                                         hbuf(G, 0));
  check_launch(ctx, "gnn_encode");
  for (int l = 0; l < kLayers; ++l) {
    LayerArgs la{};
    la.n = n;
    la.nbw = G->nbw;
    la.nb_idx = G->d_nb_idx;
    la.nb_ef = G->d_nb_ef;
    la.P = G->d_P;
    la.W = G->d_Wb + (size_t)l * kH * kIn;
    la.layer = l;
    la.h_in = hbuf(G, l);
    la.xr = G->d_xr;
    la.isd = G->d_isd;
    la.s2 = G->d_s2;
    la.m_out = training ? mbuf(G, l) : nullptr;
    la.h_out = (training || l + 1 < kLayers) ? hbuf(G, l + 1) : nullptr;
    la.z = l + 1 == kLayers ? z : nullptr;
    if (use_grid_layer(G)) {
      const GridLayerArgs ga{la, G->gnx, G->gnx * G->gny, G->d_dir_ef, G->d_err};
      if (l + 1 < kLayers) launch_layer_grid<false>(ctx, ga);
      else launch_layer_grid<true>(ctx, ga);
    } else if (l + 1 < kLayers) {
      launch_layer<false>(ctx, la);
    } else {
      launch_layer<true>(ctx, la);
    }
  }
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
  gnn_forward(G, r, G->d_z, true);
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
  k_gnn_decode_bwd<<<wg, 256, 0, ctx->stream>>>(n, G->d_Ad, G->d_s2, G->d_isd, G->d_xr, hbuf(G, kLayers), G->d_P,
                                                G->d_dh, G->d_part);
  check_launch(ctx, "gnn_decode_bwd");
  reduce_into(G, wg, kH + 2, G->d_grad + kOffWd);
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
  k_gnn_encode_bwd<<<wg, 256, 0, ctx->stream>>>(n, G->d_xr, G->d_s2, G->d_logd10, hbuf(G, 0), dh, G->d_part);
  check_launch(ctx, "gnn_encode_bwd");
  reduce_into(G, wg, 3 * kH, G->d_grad + kOffW0);
  check_grid_wait(G);
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
      std::normal_distribution<float> w0(0.f, 1.f), wl(0.f, std::sqrt(2.f / kIn)),
          wd(0.f, 0.1f * std::sqrt(1.f / kH));  // small: the network starts close to its Jacobi skip
      for (int k = 0; k < 2 * kH; ++k) h[kOffW0 + k] = w0(gen);
      for (int k = 0; k < kLayers * kH * kIn; ++k) h[kOffW + k] = wl(gen);
      for (int k = 0; k < kLayers * kH; ++k) h[kOffB + k] = 0.01f;
      for (int l = 0; l < kLayers; ++l) h[kOffU + l] = 0.5f;
      for (int k = 0; k < kH; ++k) h[kOffWd + k] = wd(gen);
      h[kOffWs] = 1.f;
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
    G->d_isd = dev_alloc<float>(ctx, (size_t)n);
    G->d_logd10 = dev_alloc<float>(ctx, (size_t)n);
    G->d_efeat = dev_alloc<float>(ctx, (size_t)A->nnz);
    G->d_tidx = dev_alloc<int>(ctx, (size_t)A->nnz);
    G->d_h = dev_alloc<bf16>(ctx, (size_t)(kLayers + 1) * n * kH);
    G->d_m = dev_alloc<bf16>(ctx, (size_t)kLayers * n * kH);
    G->d_xr = dev_alloc<float>(ctx, (size_t)n);
    G->d_s2 = dev_alloc<double>(ctx, 2);
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
    k_gnn_prep<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, A->d_v, A->d_dcol, G->d_isd,
                                                          G->d_logd10, G->d_efeat, G->d_tidx, d_bad);
    check_launch(ctx, "gnn_prep");
    int bad = 0;
    AB2_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    dev_free(ctx, d_bad);
    if (!bad) {
      int maxlen = 0;  // off-diagonal entries of the longest row (every row has its diagonal)
      host_profile(A);
      for (int i = 0; i < n; ++i) maxlen = std::max(maxlen, A->h_rp[i + 1] - A->h_rp[i] - 1);
      G->nbw = std::max(2, (maxlen + 1) / 2 * 2);
      if (G->nbw > kMaxNbw) {
        release_binding(G);
        throw Error{AB2_ERR_UNSUPPORTED, "learned preconditioner: at most 16 off-diagonal entries a row"};
      }
      G->d_nb_idx = dev_alloc<int>(ctx, (size_t)n * G->nbw);
      G->d_nb_ef = dev_alloc<float>(ctx, (size_t)n * G->nbw);
      k_gnn_nbr<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, G->d_efeat, G->nbw, G->d_nb_idx,
                                                           G->d_nb_ef);
      check_launch(ctx, "gnn_nbr");
      int nx = 0, ny = 0, nz = 0;
      G->grid = stencil_geometry(ctx, A, &nx, &ny, &nz);
      if (G->grid) {
        G->gnx = nx;
        G->gny = ny;
        G->gnz = nz;
        const long long rows = ((long long)n + kTcTile - 1) / kTcTile * kTcTile;
        G->d_dir_ef = dev_alloc<float>(ctx, (size_t)rows * 6);
        G->d_err = dev_alloc<int>(ctx, 1);
        AB2_CUDA(cudaMemsetAsync(G->d_err, 0, sizeof(int), ctx->stream));
        k_gnn_dir_table<<<grid_for(rows), kThreads, 0, ctx->stream>>>(n, rows, nx, nx * ny, A->d_rp, A->d_ci,
                                                                      G->d_efeat, G->d_dir_ef);
        check_launch(ctx, "gnn_dir_table");
      } else if (G->layout == AB2_GNN_LAYER_GRID) {
        release_binding(G);
        throw Error{AB2_ERR_UNSUPPORTED, "learned preconditioner: the grid layer needs a 3-D 7-point matrix"};
      }
    }
    if (bad) {
      release_binding(G);
      throw Error{AB2_ERR_BAD_ARG, bad & 1 ? "learned preconditioner needs a positive diagonal in every row"
                                           : "learned preconditioner needs a structurally symmetric matrix"};
    }
  });
}

int ab2_gnn_set_layer(ab2_gnn* G, int layer) {
  if (!G || layer < AB2_GNN_LAYER_AUTO || layer > AB2_GNN_LAYER_GRID) return AB2_ERR_BAD_ARG;
  G->layout = layer;
  return AB2_OK;
}

int ab2_gnn_get_layer(const ab2_gnn* G, int* layer) {
  if (!G || !layer) return AB2_ERR_BAD_ARG;
  *layer = !G->A ? AB2_GNN_LAYER_AUTO : use_grid_layer(G) ? AB2_GNN_LAYER_GRID : AB2_GNN_LAYER_GATHER;
  return AB2_OK;
}

int ab2_gnn_apply(ab2_gnn* G, const ab2_vector* r, ab2_vector* z) {
  if (!G || !r || !z || !G->A || r->n != G->n || z->n != G->n || r->d == z->d) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(G->ctx, "GNN-APPLY");
  return guard(G->ctx, [&] {
    gnn_forward(G, r->d, z->d);
    check_grid_wait(G);
  });
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
  o->truncation = 8;
  o->fallback_mode = AB2_FCG_FALLBACK_STEP;
}

// Flexible CG, FCG(m) (truncated A-orthogonalisation of the directions, so
// that a preconditioner which is not a fixed linear operator keeps them
// conjugate): z = network(r) while the network's steps reduce ||r|| by at
// least the factor fallback_ratio, the fallback preconditioner from the first
// step that does not (for the rest of the solve, the direction window
// cleared).  No network: the fallback only.
int ab2_fcg_solve(ab2_context* ctx, const ab2_matrix* A, ab2_gnn* G, const ab2_precond* fallback,
                  const ab2_vector* b, ab2_vector* x, const ab2_fcg_options* o, ab2_fcg_status* st) {
  if (!ctx || !A || !b || !x || !o || !st || b->n != A->n || x->n != A->n) return AB2_ERR_BAD_ARG;
  if (!G && !fallback) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "FCG-SOLVE");
  if (G && (G->A != A)) return AB2_ERR_BAD_ARG;
  if (fallback && fallback->A != A) return AB2_ERR_BAD_ARG;
  std::memset(st, 0, sizeof(*st));
  st->switched_at = -1;
  if (!(o->truncation >= 1 && o->truncation <= kMaxTrunc)) return AB2_ERR_BAD_ARG;
  if (o->fallback_mode != AB2_FCG_FALLBACK_STICKY && o->fallback_mode != AB2_FCG_FALLBACK_STEP) return AB2_ERR_BAD_ARG;
  return guard(ctx, [&] {
    const int n = A->n;
    const int m = o->truncation;
    cudaEvent_t e0, e1;
    AB2_CUDA(cudaEventCreate(&e0));
    AB2_CUDA(cudaEventCreate(&e1));
    double* r = dev_alloc<double>(ctx, (size_t)n);
    double* z = dev_alloc<double>(ctx, (size_t)n);
    double* pv = dev_alloc<double>(ctx, (size_t)m * n);  // window of directions
    double* qv = dev_alloc<double>(ctx, (size_t)m * n);  // and their products with A
    FcgScalars* sc = dev_alloc<FcgScalars>(ctx, 1);
    double* zq_part = dev_alloc<double>(ctx, (size_t)kMaxTrunc * kMaxRedBlocks);
    double* zq_out = dev_alloc<double>(ctx, kMaxTrunc);
    unsigned* zq_counter = dev_alloc<unsigned>(ctx, 1);
    AB2_CUDA(cudaMemsetAsync(sc, 0, sizeof(FcgScalars), ctx->stream));
    AB2_CUDA(cudaMemsetAsync(zq_counter, 0, sizeof(unsigned), ctx->stream));
    AB2_CUDA(cudaEventRecord(e0, ctx->stream));
    RedSlot red = red_slot(ctx, 7);
    const int rg = red_grid(ctx, n);
    auto dot = [&](const double* u, const double* v) {
      op_dot(ctx, n, u, v, red.result, 7);
      return read_scalar(ctx, red.result);
    };
    bool use_gnn = G != nullptr;      // the network preconditions the next step
    bool gnn_retired = G == nullptr;  // STICKY fallback has taken over
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
    op_spmv(ctx, A, x->d, z, AB2_SPMV_AUTO);
    op_copy(ctx, n, b->d, r);
    op_axpy(ctx, n, -1.0, z, r);
    double rn = std::sqrt(dot(r, r));
    int it = 0, count = 0, next = 0;
    bool ok = nb == 0.0 || rn / nb < o->tol;
    while (!ok && it < o->max_iter) {
      precond(r, z);
      double* p = pv + (size_t)next * n;
      double* q = qv + (size_t)next * n;
      if (count > 0) {
        Window wq{}, wp{};
        for (int k = 0; k < count; ++k) {
          wq.v[k] = qv + (size_t)k * n;
          wp.v[k] = pv + (size_t)k * n;
        }
        k_fcg_zq<<<rg, kThreads, 0, ctx->stream>>>(n, z, wq, count, sc, zq_part, zq_counter, zq_out);
        check_launch(ctx, "fcg_zq");
        k_fcg_dir<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, z, wp, count, sc, p);
        check_launch(ctx, "fcg_dir");
      } else {
        op_copy(ctx, n, z, p);
      }
      op_spmv(ctx, A, p, q, AB2_SPMV_AUTO);
      k_fcg_pq<<<rg, kThreads, 0, ctx->stream>>>(n, p, q, r, next, sc, red.partials, red.counter, red.result);
      check_launch(ctx, "fcg_pq");
      k_fcg_update<<<rg, kThreads, 0, ctx->stream>>>(n, p, q, x->d, r, sc, red.partials, red.counter, red.result);
      check_launch(ctx, "fcg_update");
      FcgScalars h;
      AB2_CUDA(cudaMemcpyAsync(ctx->h_pinned, sc, sizeof(FcgScalars), cudaMemcpyDeviceToHost, ctx->stream));
      AB2_CUDA(cudaStreamSynchronize(ctx->stream));
      std::memcpy(&h, ctx->h_pinned, sizeof(FcgScalars));
      if (h.breakdown) {
        st->error = AB2_ERR_BREAKDOWN;
        break;
      }
      ++it;
      const double rn_new = std::sqrt(h.rr);
      if (rn_new / nb < o->tol) {
        ok = true;
        rn = rn_new;
        break;
      }
      const bool failed = use_gnn && fallback && rn_new > o->fallback_ratio * rn;
      if (failed && st->switched_at < 0) st->switched_at = it;
      if (failed && o->fallback_mode == AB2_FCG_FALLBACK_STICKY) {
        use_gnn = false;  // ILU(0) takes over from here, with the window cleared
        gnn_retired = true;
        count = 0;
        next = 0;
      } else {
        count = std::min(count + 1, m);
        next = (next + 1) % m;
        use_gnn = !gnn_retired && !failed;  // STEP: the fallback for one step after a failed network step
      }
      rn = rn_new;
    }
    AB2_CUDA(cudaEventRecord(e1, ctx->stream));
    AB2_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    AB2_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    op_spmv(ctx, A, x->d, z, AB2_SPMV_AUTO);
    op_copy(ctx, n, b->d, r);
    op_axpy(ctx, n, -1.0, z, r);
    st->true_residual = nb > 0 ? std::sqrt(dot(r, r)) / nb : 0.0;
    st->succeeded = ok ? 1 : 0;
    st->iterations = it;
    st->solve_ms = ms;
    if (!ok && st->error == AB2_OK) st->error = AB2_ERR_NOT_CONVERGED;
    for (double* v : {r, z, pv, qv, zq_part, zq_out}) dev_free(ctx, v);
    dev_free(ctx, sc);
    dev_free(ctx, zq_counter);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (G) check_grid_wait(G);
  });
}

}  // extern "C"
