// batch.cu -- many independent systems of uneven sizes solved in ONE
// persistent launch.  No counterpart in the reference (its solvers take one
// system at a time); the per-system method is the reference's Jacobi-PCG
// (CG.h:59-150 with DiagPreconditioner.h:49-68) in FP32 inside FP64
// iterative refinement, as ab2_mixed does for one system.
//
// The systems are the diagonal blocks of one block-diagonal ab2_matrix (rows
// of system s are sys_off[s] .. sys_off[s+1]-1, columns global).  The launch
// is persistent: a grid of thread-block CLUSTERS, as many as can be resident
// at once; each cluster takes the next system from a ticket (largest first,
// so the long poles start early) and solves it completely, then takes the
// next.  Inside a cluster, CTA c owns a contiguous 1/csize of the system's
// rows; a dot product is a block tree per CTA plus the csize partials summed
// in rank order through distributed shared memory, so every CTA gets the same
// scalar; the CTAs of a cluster synchronise on the hardware cluster barrier
// (two per CG iteration, after each of the two reductions: the SpMV forms
// p = z + beta p itself at every row it reads -- from z and the previous p,
// written before the last barrier -- and stores its own rows' p in the other
// of two buffers; with the grouped-lane CSR variants a separate p pass and a
// third barrier).  Clusters never
// wait for each other, and no code spins on memory, so nothing can hang.
//
// Each system converges on its own: its cluster stops iterating when the
// system's true relative residual (FP64) is below tol -- the per-system
// convergence mask is simply which systems are finished.  Results are
// bit-reproducible (fixed trees) and restated by the oracle (orc_batch_solve).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <type_traits>
#include <vector>

#include "ab2_internal.cuh"
#include "spmv_view.cuh"

namespace cg = cooperative_groups;

namespace ab2 {
namespace {

constexpr int kMaxWarps = 32;

template <class V64, class V32>
struct BatchArgs {
  int nsys;
  const int* sys_off;    // nsys + 1 row offsets
  const int* order;      // systems, largest first
  unsigned int* ticket;
  V64 A64;
  V32 A32;
  const double* b;
  double* x;
  double* r64;           // FP64 residual scratch (N)
  float *r, *z, *p, *q, *d;  // FP32 inner CG vectors (N)
  float* p2;             // the second p buffer of the fused body (N)
  const float* inv32;    // Jacobi: 1/a_ii rounded to FP32
  double tol;
  float inner_tol;
  int max_outer, inner_max_iter;
  int* out_converged;
  int* out_outer;
  int* out_inner;
  double* out_residual;
};

// Sum of acc over the CTA (warp shuffle trees, then warp 0 over the warp sums),
// then over the cluster's CTAs in rank order via distributed shared memory.
// Every thread of every CTA of the cluster returns the same value.  `slot`
// alternates between consecutive reductions so a partial is never overwritten
// before all CTAs have read it (a cluster barrier separates reuses).
template <int NC, class T>
__device__ __forceinline__ void cluster_sum(T (&acc)[NC], T (*s_part)[4], T (*s_warp)[kMaxWarps], int slot,
                                            cg::cluster_group& cluster) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    T v = acc[c];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) s_warp[c][warp] = v;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      T v = lane < nw ? s_warp[c][lane] : T(0);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0) s_part[slot][c] = v;
    }
  }
  cluster.sync();
  const int cs = (int)cluster.num_blocks();
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    T s = T(0);
    for (int k = 0; k < cs; ++k) s = s + *cluster.map_shared_rank(&s_part[slot][c], k);
    acc[c] = s;
  }
}

template <class V64, class V32>
__global__ void k_batch_cg(BatchArgs<V64, V32> a) {
  cg::cluster_group cluster = cg::this_cluster();
  __shared__ double s_part64[2][4];
  __shared__ float s_part32[2][4];
  __shared__ double s_warp64[4][kMaxWarps];
  __shared__ float s_warp32[4][kMaxWarps];
  __shared__ int s_sys;
  const int crank = (int)cluster.block_rank();
  const int csize = (int)cluster.num_blocks();
  const int T = blockDim.x;
  int slot = 0;

  for (;;) {
    if (crank == 0 && threadIdx.x == 0) {
      const unsigned int t = atomicAdd(a.ticket, 1u);
      s_sys = t < (unsigned)a.nsys ? a.order[t] : -1;
    }
    cluster.sync();
    const int sys = *cluster.map_shared_rank(&s_sys, 0);
    // Every CTA has read the leader's s_sys before the leader may overwrite it
    // or any CTA may exit: a CTA's shared memory must outlive the remote reads
    // of it.  (All other remote reads, the partials in cluster_sum, are
    // followed by a cluster barrier before this point.)
    cluster.sync();
    if (sys < 0) break;
    const int s0 = a.sys_off[sys], s1 = a.sys_off[sys + 1];
    const int chunk = (s1 - s0 + csize - 1) / csize;
    const int lo = min(s1, s0 + crank * chunk), hi = min(s1, lo + chunk);

    // ||b||^2 of this system (FP64)
    double bb[1] = {0.0};
    for (int i = lo + threadIdx.x; i < hi; i += T) bb[0] = fma(a.b[i], a.b[i], bb[0]);
    cluster_sum<1>(bb, s_part64, s_warp64, slot, cluster);
    slot ^= 1;
    int outer = 0, inner = 0, converged = 0;
    double res = 0.0, prev = INFINITY;
    if (bb[0] == 0.0) converged = 1;
    while (!converged) {
      // r64 = b - A x, ||r||^2 (FP64)
      double rr[1] = {0.0};
      for (int i = lo + threadIdx.x; i < hi; i += T) {
        const double rv = a.b[i] - a.A64.row(i, a.x);
        a.r64[i] = rv;
        rr[0] = fma(rv, rv, rr[0]);
      }
      cluster_sum<1>(rr, s_part64, s_warp64, slot, cluster);
      slot ^= 1;
      res = sqrt(rr[0]) / sqrt(bb[0]);
      if (res < a.tol) {
        converged = 1;
        break;
      }
      if (outer >= a.max_outer || !(res < prev) || rr[0] == 0.0) break;
      prev = res;
      // inner FP32 Jacobi-PCG on A32 d = float(r / ||r||), from d = 0 (CG.h:59-150)
      const double scale = 1.0 / sqrt(rr[0]);
      float acc[2] = {0.f, 0.f};  // rho1 = r.z, r.r
      for (int i = lo + threadIdx.x; i < hi; i += T) {
        const float rv = (float)(a.r64[i] * scale);
        const float zv = __fmul_rn(a.inv32[i], rv);
        a.r[i] = rv;
        a.z[i] = zv;
        a.p[i] = zv;
        a.d[i] = 0.f;
        acc[0] = __fmaf_rn(rv, zv, acc[0]);
        acc[1] = __fmaf_rn(rv, rv, acc[1]);
      }
      cluster_sum<2>(acc, s_part32, s_warp32, slot, cluster);
      slot ^= 1;
      const float crit = a.inner_tol * a.inner_tol * acc[1];
      float rho = acc[0];
      int it = 0;
      if constexpr (lanes_per_row<V32>::value == 1) {
        // p = z + beta p formed inside the SpMV: the same fma as the p pass of
        // the loop below, so q, p.q and every scalar are the same numbers
        float beta = 0.f;
        for (;;) {
          const float* __restrict__ pold = (it & 1) ? a.p : a.p2;
          float* __restrict__ pcur = (it & 1) ? a.p2 : a.p;
          const bool first = it == 0;
          auto pval = [&](int c) { return first ? a.z[c] : __fmaf_rn(beta, pold[c], a.z[c]); };
          float pq[1] = {0.f};
          for (int i = lo + threadIdx.x; i < hi; i += T) {
            const float qv = a.A32.row_f(i, pval);
            const float pv = pval(i);
            pcur[i] = pv;
            a.q[i] = qv;
            pq[0] = __fmaf_rn(pv, qv, pq[0]);
          }
          cluster_sum<1>(pq, s_part32, s_warp32, slot, cluster);
          slot ^= 1;
          if (pq[0] == 0.f) break;  // breakdown "alpha": keep the correction so far
          const float alpha = rho / pq[0];
          float rz[2] = {0.f, 0.f};
          for (int i = lo + threadIdx.x; i < hi; i += T) {
            a.d[i] = __fmaf_rn(alpha, pcur[i], a.d[i]);
            const float rv = __fmaf_rn(-alpha, a.q[i], a.r[i]);
            a.r[i] = rv;
            const float zv = __fmul_rn(a.inv32[i], rv);
            a.z[i] = zv;
            rz[0] = __fmaf_rn(rv, zv, rz[0]);
            rz[1] = __fmaf_rn(rv, rv, rz[1]);
          }
          cluster_sum<2>(rz, s_part32, s_warp32, slot, cluster);
          slot ^= 1;
          ++it;
          if (rz[1] < crit || it >= a.inner_max_iter) break;
          beta = rz[0] / rho;
          rho = rz[0];
        }
      } else
      for (;;) {
        // q = A32 p ; alpha = rho / (p.q)   (p of every CTA written: the barrier in cluster_sum above
        // or the explicit one at the end of the previous iteration)
        float pq[1] = {0.f};
        if constexpr (lanes_per_row<V32>::value > 1) {
          // LPR lanes per row: the group's rows first, then p.q with one row per thread
          constexpr int LPR = lanes_per_row<V32>::value;
          const int g = threadIdx.x % LPR;
          for (int base = lo; base < hi; base += T / LPR) {
            const int i = base + (int)threadIdx.x / LPR;
            const bool in = i < hi;
            const float qv = a.A32.row_group(in ? i : lo, in, g, a.p);
            if (in && g == 0) a.q[i] = qv;
          }
          __syncthreads();
          for (int i = lo + threadIdx.x; i < hi; i += T) pq[0] = __fmaf_rn(a.p[i], a.q[i], pq[0]);
        } else {
          for (int i = lo + threadIdx.x; i < hi; i += T) {
            const float qv = a.A32.row(i, a.p);
            a.q[i] = qv;
            pq[0] = __fmaf_rn(a.p[i], qv, pq[0]);
          }
        }
        cluster_sum<1>(pq, s_part32, s_warp32, slot, cluster);
        slot ^= 1;
        if (pq[0] == 0.f) break;  // breakdown "alpha": keep the correction so far
        const float alpha = rho / pq[0];
        // d += alpha p ; r -= alpha q ; z = D^-1 r ; rho1 = r.z ; r.r
        float rz[2] = {0.f, 0.f};
        for (int i = lo + threadIdx.x; i < hi; i += T) {
          a.d[i] = __fmaf_rn(alpha, a.p[i], a.d[i]);
          const float rv = __fmaf_rn(-alpha, a.q[i], a.r[i]);
          a.r[i] = rv;
          const float zv = __fmul_rn(a.inv32[i], rv);
          a.z[i] = zv;
          rz[0] = __fmaf_rn(rv, zv, rz[0]);
          rz[1] = __fmaf_rn(rv, rv, rz[1]);
        }
        cluster_sum<2>(rz, s_part32, s_warp32, slot, cluster);
        slot ^= 1;
        ++it;
        if (rz[1] < crit || it >= a.inner_max_iter) break;
        // p = z + beta p
        const float beta = rz[0] / rho;
        rho = rz[0];
        for (int i = lo + threadIdx.x; i < hi; i += T) a.p[i] = __fmaf_rn(beta, a.p[i], a.z[i]);
        cluster.sync();
      }
      inner += it;
      // x += ||r|| d (FP64)
      const double sr = sqrt(rr[0]);
      for (int i = lo + threadIdx.x; i < hi; i += T) a.x[i] = fma(sr, (double)a.d[i], a.x[i]);
      cluster.sync();  // x of every CTA updated before the next residual
      ++outer;
    }
    if (crank == 0 && threadIdx.x == 0) {
      a.out_converged[sys] = converged;
      a.out_outer[sys] = outer;
      a.out_inner[sys] = inner;
      a.out_residual[sys] = res;
    }
  }
}

__global__ void k_inv32(int n, const double* __restrict__ inv, float* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = (float)inv[i];
}

}  // namespace
}  // namespace ab2

using namespace ab2;

struct ab2_batch {
  ab2_context* ctx = nullptr;
  const ab2_matrix* A = nullptr;
  ab2_batch_options opts{};
  int nsys = 0;
  int* d_off = nullptr;
  int* d_order = nullptr;
  unsigned int* d_ticket = nullptr;
  double* d_r64 = nullptr;
  float* d_vec32 = nullptr;  // r z p q d p2
  float* d_inv32 = nullptr;
  int *d_conv = nullptr, *d_outer = nullptr, *d_inner = nullptr;
  double* d_res = nullptr;
  int variant = AB2_SPMV_ELL, csize = 4, threads = 256, slice = 32, lpr = 1;
  // FP32 sliced-ELL copies with 16 and 64 rows per slice (32: the matrix's own)
  ab2::EllLayout ell16, ell64;
  int tuned = 0;
  double tune_ms = 0, setup_ms = 0, solve_ms = 0;
  std::vector<ab2_batch_trial> trials;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace ab2 {
namespace {

// Launches the persistent kernel over the first nsys_run systems of the
// largest-first order.  Returns false (nothing launched) when not even one
// cluster of this shape fits on the GPU.
template <class V64, class V32>
bool launch_batch(ab2_batch* B, V64 a64, V32 a32, int csize, int threads, const double* b, double* x, int max_outer,
                  int inner_max_iter, int nsys_run) {
  ab2_context* ctx = B->ctx;
  const size_t N = (size_t)B->A->n;
  BatchArgs<V64, V32> args;
  args.nsys = nsys_run;
  args.sys_off = B->d_off;
  args.order = B->d_order;
  args.ticket = B->d_ticket;
  args.A64 = a64;
  args.A32 = a32;
  args.b = b;
  args.x = x;
  args.r64 = B->d_r64;
  args.r = B->d_vec32;
  args.z = B->d_vec32 + N;
  args.p = B->d_vec32 + 2 * N;
  args.q = B->d_vec32 + 3 * N;
  args.d = B->d_vec32 + 4 * N;
  args.p2 = B->d_vec32 + 5 * N;
  args.inv32 = B->d_inv32;
  args.tol = B->opts.tol;
  args.inner_tol = (float)B->opts.inner_tol;
  args.max_outer = max_outer;
  args.inner_max_iter = inner_max_iter;
  args.out_converged = B->d_conv;
  args.out_outer = B->d_outer;
  args.out_inner = B->d_inner;
  args.out_residual = B->d_res;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3((unsigned)threads);
  cfg.gridDim = dim3((unsigned)csize);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = ctx->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (csize > 8)  // 16-CTA clusters are beyond the portable size
    AB2_CUDA(cudaFuncSetAttribute(k_batch_cg<V64, V32>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  int nclusters = 0;
  AB2_CUDA(cudaOccupancyMaxActiveClusters(&nclusters, (void*)k_batch_cg<V64, V32>, &cfg));
  if (nclusters < 1) return false;
  nclusters = std::min(nclusters, nsys_run);
  cfg.gridDim = dim3((unsigned)(nclusters * csize));
  AB2_CUDA(cudaMemsetAsync(B->d_ticket, 0, sizeof(unsigned int), ctx->stream));
  AB2_CUDA(cudaLaunchKernelEx(&cfg, k_batch_cg<V64, V32>, args));
  check_launch(ctx, "batch_cg");
  return true;
}

// The FP64 residual reads the CSR values (any format gives the same bits);
// the FP32 inner SpMV runs in the format under trial.
bool run_batch(ab2_batch* B, int variant, int slice, int lpr, int csize, int threads, const double* b, double* x,
               int max_outer, int inner_max_iter, int nsys_run) {
  const ab2_matrix* A = B->A;
  const CsrView<double> v64{A->d_rp, A->d_ci, A->d_v};
  auto go = [&](auto v32) { return launch_batch(B, v64, v32, csize, threads, b, x, max_outer, inner_max_iter, nsys_run); };
  if (variant == AB2_SPMV_ELL) {
    if (slice == 16) return go(EllViewS<float, 16>{B->ell16.off, B->ell16.ci, B->ell16.v});
    if (slice == 64) return go(EllViewS<float, 64>{B->ell64.off, B->ell64.ci, B->ell64.v});
    require(A->d_ell_v32 != nullptr, "batched solver: the matrix has no FP32 sliced-ELL copy");
    return go(EllViewS<float, 32>{A->d_ell_off, A->d_ell_ci, A->d_ell_v32});
  }
  switch (lpr) {
    case 2: return go(CsrGroupView<float, 2>{A->d_rp, A->d_ci, A->d_v32});
    case 4: return go(CsrGroupView<float, 4>{A->d_rp, A->d_ci, A->d_v32});
    case 8: return go(CsrGroupView<float, 8>{A->d_rp, A->d_ci, A->d_v32});
    default: return go(CsrView<float>{A->d_rp, A->d_ci, A->d_v32});
  }
}

// A shape of the inner SpMV: sliced ELL (slice rows) or CSR (lanes per row).
struct Fmt {
  int variant, slice, lpr;
};

// Scores candidates on the batch itself, from b = 1: score = (one refinement
// step of `tune_iters` FP32 iterations for every system: the throughput of the
// launch) + (4 x tune_iters iterations of the largest system alone: the
// latency of the long pole, which bounds a batch whose hardest system needs
// many iterations).  Two rounds: every SpMV format (ELL with 16 / 32 / 64
// rows per slice, CSR with 1 / 2 / 4 / 8 lanes per row) at 8 CTAs x 512
// threads (or the fixed shape), then the best format at every CTA count x
// width.  Shapes that do not fit are skipped.
void autotune(ab2_batch* B) {
  ab2_context* ctx = B->ctx;
  const int N = B->A->n;
  double* b = dev_alloc<double>(ctx, (size_t)N);
  double* x = dev_alloc<double>(ctx, (size_t)N);
  op_fill(ctx, N, 1.0, b);
  const ab2_batch_options& o = B->opts;
  std::vector<Fmt> fmts;
  const bool ell_ok = B->A->d_ell_v32 != nullptr;
  if (o.spmv_variant == AB2_SPMV_AUTO || o.spmv_variant == AB2_SPMV_ELL) {
    for (int sl : {16, 32, 64})
      if ((o.ell_slice == 0 || o.ell_slice == sl) && (sl != 32 || ell_ok)) fmts.push_back(Fmt{AB2_SPMV_ELL, sl, 0});
  }
  if (o.spmv_variant == AB2_SPMV_AUTO || o.spmv_variant == AB2_SPMV_CSR_SCALAR) {
    for (int l : {1, 2, 4, 8})
      if (o.lanes_per_row == 0 || o.lanes_per_row == l) fmts.push_back(Fmt{AB2_SPMV_CSR_SCALAR, 0, l});
  }
  const std::vector<int> csizes = o.cluster_size ? std::vector<int>{o.cluster_size} : std::vector<int>{1, 2, 4, 8, 16};
  const std::vector<int> widths = o.threads ? std::vector<int>{o.threads} : std::vector<int>{256, 512};
  const int iters = o.tune_iters > 0 ? o.tune_iters : 8;
  cudaEvent_t e0, e1;
  AB2_CUDA(cudaEventCreate(&e0));
  AB2_CUDA(cudaEventCreate(&e1));
  AB2_CUDA(cudaEventRecord(B->ev0, ctx->stream));
  float best = 1e30f;
  Fmt best_fmt = fmts.empty() ? Fmt{AB2_SPMV_CSR_SCALAR, 0, 1} : fmts[0];
  auto trial = [&](const Fmt& f, int c, int t) {
    float ms = 0;
    for (int part = 0; part < 2; ++part) {
      const int nrun = part == 0 ? B->nsys : 1;
      const int it = part == 0 ? iters : 4 * iters;
      op_fill(ctx, N, 0.0, x);
      if (!run_batch(B, f.variant, f.slice, f.lpr, c, t, b, x, 1, it, nrun)) return;  // warm; does not fit
      op_fill(ctx, N, 0.0, x);
      AB2_CUDA(cudaEventRecord(e0, ctx->stream));
      run_batch(B, f.variant, f.slice, f.lpr, c, t, b, x, 1, it, nrun);
      AB2_CUDA(cudaEventRecord(e1, ctx->stream));
      AB2_CUDA(cudaEventSynchronize(e1));
      float part_ms = 0;
      AB2_CUDA(cudaEventElapsedTime(&part_ms, e0, e1));
      ms += part_ms;
    }
    B->trials.push_back(ab2_batch_trial{f.variant, c, t, ms, f.slice, f.lpr});
    if (ms < best) {
      best = ms;
      best_fmt = f;
      B->variant = f.variant;
      B->slice = f.slice;
      B->lpr = f.lpr;
      B->csize = c;
      B->threads = t;
    }
  };
  // round 1: the format, at the reference shape
  const int c0 = o.cluster_size ? o.cluster_size : 8, t0 = o.threads ? o.threads : 512;
  for (const Fmt& f : fmts) trial(f, c0, t0);
  // round 2: the shape, for the best format
  for (int c : csizes)
    for (int t : widths)
      if (!(c == c0 && t == t0)) trial(best_fmt, c, t);
  AB2_CUDA(cudaEventRecord(B->ev1, ctx->stream));
  AB2_CUDA(cudaEventSynchronize(B->ev1));
  float ms = 0;
  AB2_CUDA(cudaEventElapsedTime(&ms, B->ev0, B->ev1));
  B->tune_ms = ms;
  B->tuned = 1;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dev_free(ctx, b);
  dev_free(ctx, x);
}

}  // namespace
}  // namespace ab2

extern "C" {

void ab2_batch_options_default(ab2_batch_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->tol = 1e-8;
  o->max_outer = 20;
  o->inner_tol = 1e-4;
  o->inner_max_iter = 5000;
  o->spmv_variant = AB2_SPMV_AUTO;
  o->cluster_size = 0;
  o->threads = 0;
  o->tune_iters = 8;
}

int ab2_batch_create(ab2_context* ctx, const ab2_matrix* A, int nsys, const int* sys_offsets,
                     const ab2_batch_options* o, ab2_batch** out) {
  if (!ctx || !A || !o || !out || nsys <= 0 || !sys_offsets) return AB2_ERR_BAD_ARG;
  *out = nullptr;
  if (!A->d_v32) {
    ctx->last_error = "batched solver needs the matrix's FP32 values (create it with AB2_FMT_F32)";
    return AB2_ERR_BAD_ARG;
  }
  if (o->spmv_variant != AB2_SPMV_AUTO && o->spmv_variant != AB2_SPMV_ELL && o->spmv_variant != AB2_SPMV_CSR_SCALAR)
    return AB2_ERR_BAD_ARG;
  if (!(o->cluster_size == 0 || o->cluster_size == 1 || o->cluster_size == 2 || o->cluster_size == 4 ||
        o->cluster_size == 8 || o->cluster_size == 16))
    return AB2_ERR_BAD_ARG;
  if (o->threads != 0 && (o->threads < 64 || o->threads > 1024 || o->threads % 32 != 0)) return AB2_ERR_BAD_ARG;
  if (!(o->ell_slice == 0 || o->ell_slice == 16 || o->ell_slice == 32 || o->ell_slice == 64)) return AB2_ERR_BAD_ARG;
  if (!(o->lanes_per_row == 0 || o->lanes_per_row == 1 || o->lanes_per_row == 2 || o->lanes_per_row == 4 ||
        o->lanes_per_row == 8))
    return AB2_ERR_BAD_ARG;
  if (!(o->tol >= 0) || !(o->inner_tol > 0 && o->inner_tol < 1) || o->max_outer < 0 || o->inner_max_iter < 1)
    return AB2_ERR_BAD_ARG;
  // systems: increasing offsets from 0 to n, each a diagonal block of A
  if (sys_offsets[0] != 0 || sys_offsets[nsys] != A->n) return AB2_ERR_BAD_ARG;
  if (const int rc = guard(ctx, [&] { host_profile(A); }); rc != AB2_OK) return rc;
  for (int s = 0; s < nsys; ++s) {
    if (sys_offsets[s + 1] <= sys_offsets[s]) return AB2_ERR_BAD_ARG;
    for (int r = sys_offsets[s]; r < sys_offsets[s + 1]; ++r)
      for (int k = A->h_rp[r]; k < A->h_rp[r + 1]; ++k)
        if (A->h_ci[k] < sys_offsets[s] || A->h_ci[k] >= sys_offsets[s + 1]) {
          ctx->last_error = "batched solver: a row couples two systems (the matrix must be block diagonal)";
          return AB2_ERR_BAD_ARG;
        }
  }
  ab2_batch* B = new (std::nothrow) ab2_batch();
  if (!B) return AB2_ERR_OOM;
  B->ctx = ctx_retain(ctx);
  int rc = guard(ctx, [&] {
    B->A = A;
    B->opts = *o;
    B->nsys = nsys;
    AB2_CUDA(cudaEventCreate(&B->ev0));
    AB2_CUDA(cudaEventCreate(&B->ev1));
    cudaEvent_t s0, s1;
    AB2_CUDA(cudaEventCreate(&s0));
    AB2_CUDA(cudaEventCreate(&s1));
    AB2_CUDA(cudaEventRecord(s0, ctx->stream));
    const size_t N = (size_t)A->n;
    std::vector<int> order(nsys);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      return sys_offsets[a + 1] - sys_offsets[a] > sys_offsets[b + 1] - sys_offsets[b];
    });
    B->d_off = dev_alloc<int>(ctx, (size_t)nsys + 1);
    B->d_order = dev_alloc<int>(ctx, (size_t)nsys);
    AB2_CUDA(cudaMemcpyAsync(B->d_off, sys_offsets, sizeof(int) * ((size_t)nsys + 1), cudaMemcpyHostToDevice,
                             ctx->stream));
    AB2_CUDA(cudaMemcpyAsync(B->d_order, order.data(), sizeof(int) * (size_t)nsys, cudaMemcpyHostToDevice,
                             ctx->stream));
    B->d_ticket = dev_alloc<unsigned int>(ctx, 1);
    B->d_r64 = dev_alloc<double>(ctx, N);
    B->d_vec32 = dev_alloc<float>(ctx, 6 * N);
    B->d_inv32 = dev_alloc<float>(ctx, N);
    double* inv = dev_alloc<double>(ctx, N);
    op_inv_diag(ctx, A, inv);
    k_inv32<<<grid_for(A->n), kThreads, 0, ctx->stream>>>(A->n, inv, B->d_inv32);
    check_launch(ctx, "inv32");
    dev_free(ctx, inv);
    B->d_conv = dev_alloc<int>(ctx, (size_t)nsys);
    B->d_outer = dev_alloc<int>(ctx, (size_t)nsys);
    B->d_inner = dev_alloc<int>(ctx, (size_t)nsys);
    B->d_res = dev_alloc<double>(ctx, (size_t)nsys);
    B->variant = o->spmv_variant == AB2_SPMV_AUTO ? (A->d_ell_v32 ? AB2_SPMV_ELL : AB2_SPMV_CSR_SCALAR)
                                                  : o->spmv_variant;
    B->slice = o->ell_slice ? o->ell_slice : 32;
    B->lpr = o->lanes_per_row ? o->lanes_per_row : 1;
    B->csize = o->cluster_size ? o->cluster_size : 4;
    B->threads = o->threads ? o->threads : 256;
    const bool tune_fmt = o->spmv_variant == AB2_SPMV_AUTO ||
                          (o->spmv_variant == AB2_SPMV_ELL && o->ell_slice == 0) ||
                          (o->spmv_variant == AB2_SPMV_CSR_SCALAR && o->lanes_per_row == 0);
    // the 16- and 64-row ELL copies, where ELL may be used with those widths
    if (o->spmv_variant != AB2_SPMV_CSR_SCALAR) {
      if (o->ell_slice == 16 || (o->ell_slice == 0 && tune_fmt)) B->ell16 = build_ell_f32(ctx, A, 16);
      if (o->ell_slice == 64 || (o->ell_slice == 0 && tune_fmt)) B->ell64 = build_ell_f32(ctx, A, 64);
    }
    if (B->variant == AB2_SPMV_ELL && B->slice == 32 && !A->d_ell_v32 && !tune_fmt)
      throw Error{AB2_ERR_BAD_ARG, "batched solver: 32-row ELL needs the matrix's ELL copy (AB2_FMT_ELL)"};
    if (tune_fmt || o->cluster_size == 0 || o->threads == 0) autotune(B);
    // the ELL copies the chosen format does not use are not kept
    if (!(B->variant == AB2_SPMV_ELL && B->slice == 16)) free_ell(ctx, B->ell16);
    if (!(B->variant == AB2_SPMV_ELL && B->slice == 64)) free_ell(ctx, B->ell64);
    AB2_CUDA(cudaEventRecord(s1, ctx->stream));
    AB2_CUDA(cudaEventSynchronize(s1));
    float ms = 0;
    AB2_CUDA(cudaEventElapsedTime(&ms, s0, s1));
    B->setup_ms = ms;
    cudaEventDestroy(s0);
    cudaEventDestroy(s1);
  });
  if (rc != AB2_OK) {
    ab2_batch_destroy(B);
    return rc;
  }
  *out = B;
  return AB2_OK;
}

int ab2_batch_solve(ab2_batch* B, const ab2_vector* b, ab2_vector* x, ab2_batch_status* status) {
  if (!B || !b || !x || !status || b->n != B->A->n || x->n != B->A->n) return AB2_ERR_BAD_ARG;
  ab2_context* ctx = B->ctx;
  PhaseScope phase_scope(ctx, "BATCH-SOLVE");
  std::memset(status, 0, sizeof(*status));
  return guard(ctx, [&] {
    AB2_CUDA(cudaEventRecord(B->ev0, ctx->stream));
    if (!run_batch(B, B->variant, B->slice, B->lpr, B->csize, B->threads, b->d, x->d, B->opts.max_outer,
                   B->opts.inner_max_iter, B->nsys))
      throw Error{AB2_ERR_UNSUPPORTED, "batched solver: no cluster of the configured shape fits on this GPU"};
    AB2_CUDA(cudaEventRecord(B->ev1, ctx->stream));
    AB2_CUDA(cudaEventSynchronize(B->ev1));
    float ms = 0;
    AB2_CUDA(cudaEventElapsedTime(&ms, B->ev0, B->ev1));
    B->solve_ms = ms;
    std::vector<int> conv(B->nsys), outer(B->nsys), inner(B->nsys);
    std::vector<double> res(B->nsys);
    AB2_CUDA(cudaMemcpy(conv.data(), B->d_conv, sizeof(int) * B->nsys, cudaMemcpyDeviceToHost));
    AB2_CUDA(cudaMemcpy(outer.data(), B->d_outer, sizeof(int) * B->nsys, cudaMemcpyDeviceToHost));
    AB2_CUDA(cudaMemcpy(inner.data(), B->d_inner, sizeof(int) * B->nsys, cudaMemcpyDeviceToHost));
    AB2_CUDA(cudaMemcpy(res.data(), B->d_res, sizeof(double) * B->nsys, cudaMemcpyDeviceToHost));
    for (int s = 0; s < B->nsys; ++s) {
      status->systems_converged += conv[s];
      status->max_outer = std::max(status->max_outer, outer[s]);
      status->inner_total += inner[s];
      status->inner_max = std::max(status->inner_max, inner[s]);
      status->max_residual = std::max(status->max_residual, res[s]);
    }
    status->solve_ms = B->solve_ms;
  });
}

int ab2_batch_results(const ab2_batch* B, int* converged, int* outer, int* inner, double* residual) {
  if (!B) return AB2_ERR_BAD_ARG;
  const size_t m = (size_t)B->nsys;
  if (converged && cudaMemcpy(converged, B->d_conv, sizeof(int) * m, cudaMemcpyDeviceToHost) != cudaSuccess)
    return AB2_ERR_CUDA;
  if (outer && cudaMemcpy(outer, B->d_outer, sizeof(int) * m, cudaMemcpyDeviceToHost) != cudaSuccess)
    return AB2_ERR_CUDA;
  if (inner && cudaMemcpy(inner, B->d_inner, sizeof(int) * m, cudaMemcpyDeviceToHost) != cudaSuccess)
    return AB2_ERR_CUDA;
  if (residual && cudaMemcpy(residual, B->d_res, sizeof(double) * m, cudaMemcpyDeviceToHost) != cudaSuccess)
    return AB2_ERR_CUDA;
  return AB2_OK;
}

int ab2_batch_get_info(const ab2_batch* B, ab2_batch_info* info) {
  if (!B || !info) return AB2_ERR_BAD_ARG;
  info->nsys = B->nsys;
  info->rows = B->A->n;
  info->spmv_variant = B->variant;
  info->cluster_size = B->csize;
  info->threads = B->threads;
  info->tuned = B->tuned;
  info->tune_ms = B->tune_ms;
  info->setup_ms = B->setup_ms;
  info->trials = (int)B->trials.size();
  info->ell_slice = B->variant == AB2_SPMV_ELL ? B->slice : 0;
  info->lanes_per_row = B->variant == AB2_SPMV_CSR_SCALAR ? B->lpr : 0;
  return AB2_OK;
}

int ab2_batch_trials(const ab2_batch* B, ab2_batch_trial* trials, int cap) {
  if (!B || (cap > 0 && !trials)) return AB2_ERR_BAD_ARG;
  const int m = std::min(cap, (int)B->trials.size());
  for (int i = 0; i < m; ++i) trials[i] = B->trials[(size_t)i];
  return AB2_OK;
}

int ab2_batch_destroy(ab2_batch* B) {
  if (!B) return AB2_ERR_BAD_ARG;
  if (B->ctx) {
    ctx_quiesce(B->ctx);
    for (void* p : {(void*)B->d_off, (void*)B->d_order, (void*)B->d_ticket, (void*)B->d_r64, (void*)B->d_vec32,
                    (void*)B->d_inv32, (void*)B->d_conv, (void*)B->d_outer, (void*)B->d_inner, (void*)B->d_res})
      dev_free(B->ctx, p);
    free_ell(B->ctx, B->ell16);
    free_ell(B->ctx, B->ell64);
  }
  if (B->ev0) cudaEventDestroy(B->ev0);
  if (B->ev1) cudaEventDestroy(B->ev1);
  if (B->ctx) ctx_release(B->ctx);
  delete B;
  return AB2_OK;
}

}  // extern "C"
