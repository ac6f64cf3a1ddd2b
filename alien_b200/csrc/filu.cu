// filu.cu -- FILU0 and Neumann-polynomial preconditioners on the device.
//
//   FILU0    FILU0Preconditioner.h:28-337 (FLUFactorisationAlgo)
//            init :60-84      factor: exact ILU(0) (nb-factor-iter = 0) or
//                             factorizeMultiIter :119-145, which init (:72)
//                             calls on the factor matrix itself: every sweep
//                             starts from the previous iterate (the first from A)
//            solve :245-267   nb-solver-iter Jacobi sweeps for L, then for U,
//                             the device-algebra branch of solveL/solveU
//                             (:161-175 / :218-226: copy, addLMult(-1) or
//                             addUMult(-1), pointwiseMult by 1/u_ii)
//   Neumann  NeumannPolyPreconditioner.h:33-190
//            solve :103-119   y = x; order x { y <- x + (y - omega A y) }; y *= omega
//            computeFactor :133-168 (power method on A, omega = 1/estimate)
//
// Arithmetic follows the reference operation by operation, so the device
// results are bit-identical to the reference templates run on a sequential
// CPU algebra: the factor sweep is the row loop of _factorizeRow (:270-300) --
// an IEEE division by the previous iterate's pivot, products and differences
// rounded apart -- and an L/U sweep is SimpleCSR's _seqAddLMult/_seqAddUMult
// row (SimpleCSRMatrixMultT.h:193-233: tmpy += (alpha a) x in CSR order with
// alpha = -1) followed by pointwiseMult.  The factor sweep is one thread per
// row, each row depending only on the previous iterate (set-up only); the
// application sweeps stream L and U from sliced ELL, one thread per row,
// coalesced, with the operand vector read through L2.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "ab2_internal.cuh"
#include "precond.cuh"
#include "spmv_view.cuh"

namespace ab2 {
namespace {

constexpr int kSlice = 32;

// One fixed-point factorisation sweep (factorizeIter + _factorizeRow): v = the
// new iterate, each row starting from a (the previous iterate: the reference's
// "matrix values" are the factor's own) and reading the copy v0 of it.  Row 0
// keeps its values (the reference starts at irow = 1).
__global__ void k_filu_factor_sweep(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                    const int* __restrict__ dcol, const double* a, const double* __restrict__ v0,
                                    double* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int kb = rp[i], ke = rp[i + 1];
    for (int k = kb; k < ke; ++k) v[k] = a[k];
    if (i == 0) continue;
    for (int k = kb; k < dcol[i]; ++k) {
      const int krow = ci[k];
      const double aik = __ddiv_rn(v[k], v0[dcol[krow]]);
      v[k] = aik;
      const int lo0 = rp[krow], hi0 = rp[krow + 1] - 1;
      for (int j = k + 1; j < ke; ++j) {
        const int jcol = ci[j];
        int lo = lo0, hi = hi0, kj = -1;  // position of jcol in row krow (sorted columns)
        while (lo <= hi) {
          const int mid = (lo + hi) >> 1;
          const int c = ci[mid];
          if (c == jcol) {
            kj = mid;
            break;
          }
          if (c < jcol) lo = mid + 1;
          else hi = mid - 1;
        }
        if (kj >= 0) v[j] = __dsub_rn(v[j], __dmul_rn(aik, v0[kj]));
      }
    }
  }
}

// Per 32-row slice: the widest strict-lower and strict-upper row.
__global__ void k_filu_widths(int n, const int* __restrict__ rp, const int* __restrict__ dcol, int* __restrict__ wl,
                              int* __restrict__ wu) {
  const int lane = threadIdx.x & 31;
  const int nslices = (n + kSlice - 1) / kSlice;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nslices; s += (gridDim.x * blockDim.x) >> 5) {
    const int i = s * kSlice + lane;
    int l = 0, u = 0;
    if (i < n) {
      l = dcol[i] - rp[i];
      u = rp[i + 1] - dcol[i] - 1;
    }
    l = __reduce_max_sync(0xffffffffu, l);
    u = __reduce_max_sync(0xffffffffu, u);
    if (lane == 0) {
      wl[s] = l;
      wu[s] = u;
    }
  }
}

// Scatters the strict L and strict U entries of the factor into sliced ELL
// (slot-major inside a slice, row order kept, column -1 pads) and 1/u_ii.
__global__ void k_filu_fill(int n, const int* __restrict__ rp, const int* __restrict__ ci, const int* __restrict__ dcol,
                            const double* __restrict__ lu, const int* __restrict__ loff, const int* __restrict__ uoff,
                            int* __restrict__ lci, double* __restrict__ lv, int* __restrict__ uci,
                            double* __restrict__ uv, double* __restrict__ inv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int s = i / kSlice, lane = i % kSlice;
    const int dk = dcol[i];
    const long long lb = (long long)loff[s] * kSlice + lane, ub = (long long)uoff[s] * kSlice + lane;
    const int lw = loff[s + 1] - loff[s], uw = uoff[s + 1] - uoff[s];
    int w = 0;
    for (int k = rp[i]; k < dk; ++k, ++w) {
      lci[lb + (long long)w * kSlice] = ci[k];
      lv[lb + (long long)w * kSlice] = lu[k];
    }
    for (; w < lw; ++w) {
      lci[lb + (long long)w * kSlice] = -1;
      lv[lb + (long long)w * kSlice] = 0.0;
    }
    w = 0;
    for (int k = dk + 1; k < rp[i + 1]; ++k, ++w) {
      uci[ub + (long long)w * kSlice] = ci[k];
      uv[ub + (long long)w * kSlice] = lu[k];
    }
    for (; w < uw; ++w) {
      uci[ub + (long long)w * kSlice] = -1;
      uv[ub + (long long)w * kSlice] = 0.0;
    }
    inv[i] = __ddiv_rn(1.0, lu[dk]);  // computeInvDiag on the factor
  }
}

// One Jacobi sweep: out_i = rhs_i - sum_k t_k xk[c_k] (CSR order, product and
// difference rounded apart), times inv_i for U.
template <class T, bool UPPER>
__global__ void __launch_bounds__(kThreads) k_filu_sweep(int n, const int* __restrict__ off, const int* __restrict__ ci,
                                                         const T* __restrict__ v, const T* __restrict__ rhs,
                                                         const T* __restrict__ xk, const T* __restrict__ inv,
                                                         T* __restrict__ out) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const int s = row / kSlice;
  const long long b = (long long)off[s] * kSlice + row % kSlice;
  const int w = off[s + 1] - off[s];
  T acc = rhs[row];
  for (int k = 0; k < w; ++k) {
    const int c = ci[b + (long long)k * kSlice];
    if (c >= 0) acc = add_rn(acc, -mul_rn(v[b + (long long)k * kSlice], xk[c]));
  }
  if (UPPER) acc = mul_rn(inv[row], acc);
  out[row] = acc;
}

// Neumann step: out = x + (cur - omega A cur) as copy + axpy(-omega) + axpy(1);
// the last step also applies scal(omega).
template <class View, class T>
__global__ void __launch_bounds__(kThreads) k_neumann_step(int n, View A, const T* __restrict__ x,
                                                           const T* __restrict__ cur, T* __restrict__ out, T omega,
                                                           int last) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const T ay = A.row(row, cur);
  T v = fma_rn(-omega, ay, cur[row]);
  v = fma_rn(T(1), x[row], v);
  out[row] = last ? mul_rn(omega, v) : v;
}

template <class T>
__global__ void k_scale_copy(int n, T a, const T* __restrict__ x, T* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = mul_rn(a, x[i]);
}

// Slice offsets (prefix of the widths) on the host; returns the total slots.
long long slice_offsets(ab2_context* ctx, const int* d_w, int nslices, int* d_off) {
  std::vector<int> w((size_t)nslices), off((size_t)nslices + 1, 0);
  AB2_CUDA(cudaMemcpyAsync(w.data(), d_w, sizeof(int) * (size_t)nslices, cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  long long total = 0;
  for (int s = 0; s < nslices; ++s) {
    total += w[(size_t)s];
    require(total < (1LL << 31), "FILU0: too many ELL slots for 32-bit offsets");
    off[(size_t)s + 1] = (int)total;
  }
  AB2_CUDA(cudaMemcpyAsync(d_off, off.data(), sizeof(int) * ((size_t)nslices + 1), cudaMemcpyHostToDevice, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  return total * kSlice;
}

template <class T>
struct FiluArrays;
template <>
struct FiluArrays<double> {
  const double *lv, *uv, *inv;
  double* t[2];
  explicit FiluArrays(const FiluData& f) : lv(f.d_l_v), uv(f.d_u_v), inv(f.d_inv), t{f.d_t[0], f.d_t[1]} {}
};
template <>
struct FiluArrays<float> {
  const float *lv, *uv, *inv;
  float* t[2];
  FiluArrays(const FiluData& f, int n) : lv(f.d_l_v32), uv(f.d_u_v32), inv(f.d_inv32), t{f.d_t32, f.d_t32 + n} {}
};

}  // namespace

void filu_init(ab2_context* ctx, ab2_precond* pc, const ab2_precond_options* o) {
  require(o->filu_factor_iter >= 0 && o->filu_solver_iter >= 0, "FILU0 iteration counts must be >= 0");
  const ab2_matrix* A = pc->A;
  const int n = A->n;
  FiluData& f = pc->fil;
  f.factor_iter = o->filu_factor_iter;
  f.solver_iter = o->filu_solver_iter;
  f.tol = o->filu_tol;
  Ilu0Data& d = pc->ilu;
  if (f.factor_iter == 0) {
    // init :67-68 -> factorize(): the exact ILU(0) factor (the sequential
    // branch does not depend on the block-Jacobi flag)
    ilu_init(ctx, pc, AB2_ILU_AUTO);
    ilu_drop_schedule(ctx, d);
  } else {
    d.d_lu = dev_alloc<double>(ctx, (size_t)A->nnz);
    double* tmp = dev_alloc<double>(ctx, (size_t)A->nnz);
    // baseInit clones A: the first iterate is A itself
    AB2_CUDA(cudaMemcpyAsync(tmp, A->d_v, sizeof(double) * (size_t)A->nnz, cudaMemcpyDeviceToDevice, ctx->stream));
    double* prev = tmp;
    double* cur = d.d_lu;
    for (int it = 0; it < f.factor_iter; ++it) {
      k_filu_factor_sweep<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, A->d_dcol, prev, prev,
                                                                      cur);
      check_launch(ctx, "filu_factor_sweep");
      std::swap(prev, cur);
    }
    if (prev != d.d_lu)  // the latest iterate is in `prev`
      AB2_CUDA(cudaMemcpyAsync(d.d_lu, prev, sizeof(double) * (size_t)A->nnz, cudaMemcpyDeviceToDevice, ctx->stream));
    dev_free(ctx, tmp);
  }
  const int nslices = (n + kSlice - 1) / kSlice;
  int* wl = dev_alloc<int>(ctx, (size_t)nslices);
  int* wu = dev_alloc<int>(ctx, (size_t)nslices);
  k_filu_widths<<<grid_for((long long)nslices * 32), kThreads, 0, ctx->stream>>>(n, A->d_rp, A->d_dcol, wl, wu);
  check_launch(ctx, "filu_widths");
  f.d_l_off = dev_alloc<int>(ctx, (size_t)nslices + 1);
  f.d_u_off = dev_alloc<int>(ctx, (size_t)nslices + 1);
  const long long lslots = slice_offsets(ctx, wl, nslices, f.d_l_off);
  const long long uslots = slice_offsets(ctx, wu, nslices, f.d_u_off);
  dev_free(ctx, wl);
  dev_free(ctx, wu);
  f.d_l_ci = dev_alloc<int>(ctx, (size_t)std::max(lslots, 1LL));
  f.d_l_v = dev_alloc<double>(ctx, (size_t)std::max(lslots, 1LL));
  f.d_u_ci = dev_alloc<int>(ctx, (size_t)std::max(uslots, 1LL));
  f.d_u_v = dev_alloc<double>(ctx, (size_t)std::max(uslots, 1LL));
  f.d_inv = dev_alloc<double>(ctx, (size_t)n);
  f.d_t[0] = dev_alloc<double>(ctx, (size_t)n);
  f.d_t[1] = dev_alloc<double>(ctx, (size_t)n);
  k_filu_fill<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, A->d_dcol, d.d_lu, f.d_l_off, f.d_u_off,
                                                         f.d_l_ci, f.d_l_v, f.d_u_ci, f.d_u_v, f.d_inv);
  check_launch(ctx, "filu_fill");
}

template <class T>
void filu_apply(ab2_context* ctx, const ab2_precond* pc, const T* x, T* y) {
  const int n = pc->A->n;
  const FiluData& f = pc->fil;
  const int S = f.solver_iter;
  if (S == 0) {  // m_x = x, y = m_x
    if (x != y) AB2_CUDA(cudaMemcpyAsync(y, x, sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
    return;
  }
  FiluArrays<T> w = [&] {
    if constexpr (sizeof(T) == 8) return FiluArrays<T>(f);
    else return FiluArrays<T>(f, n);
  }();
  const int g = (n + kThreads - 1) / kThreads;
  // L: m_x = x, then m_x <- x - L m_x, S times (ping-pong in t0/t1)
  const T* xk = x;
  for (int it = 0; it < S; ++it) {
    T* out = w.t[it & 1];
    k_filu_sweep<T, false><<<g, kThreads, 0, ctx->stream>>>(n, f.d_l_off, f.d_l_ci, w.lv, x, xk, nullptr, out);
    check_launch(ctx, "filu_lsweep");
    xk = out;
  }
  const T* mx = xk;              // L result, the right-hand side of every U sweep
  T* other = w.t[(S & 1)];       // the work vector mx is not in
  // U: y = m_x, then y <- inv (m_x - U y), S times; the last sweep lands in y
  const T* yk = mx;
  for (int it = 0; it < S; ++it) {
    T* out = ((S - 1 - it) % 2 == 0) ? y : other;
    k_filu_sweep<T, true><<<g, kThreads, 0, ctx->stream>>>(n, f.d_u_off, f.d_u_ci, w.uv, mx, yk, w.inv, out);
    check_launch(ctx, "filu_usweep");
    yk = out;
  }
}

void neumann_init(ab2_context* ctx, ab2_precond* pc, const ab2_precond_options* o) {
  const ab2_matrix* A = pc->A;
  const int n = A->n;
  NeumannData& nd = pc->neu;
  require(o->poly_order >= 0, "Neumann polynomial order must be >= 0");
  nd.order = o->poly_order;
  for (double*& t : nd.d_t) t = dev_alloc<double>(ctx, (size_t)n);
  nd.omega = o->poly_factor;
  if (nd.omega != 0.0) return;
  // computeFactor :133-168: |lambda_max| of A by the power method, omega = 1/it
  require(o->poly_factor_max_iter >= 1, "Neumann power method needs poly_factor_max_iter >= 1");
  std::vector<double> h((size_t)n);
  std::mt19937 gen;
  std::uniform_real_distribution<> dis(-1., 1.);
  for (int i = 0; i < n; ++i) h[(size_t)i] = dis(gen);
  double* x = nd.d_t[0];
  double* y = nd.d_t[1];
  double* s = red_slot(ctx, 0).result;
  AB2_CUDA(cudaMemcpyAsync(x, h.data(), sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
  op_spmv(ctx, A, x, y, pc->variant);
  op_dot(ctx, n, y, y, s);
  double nk = std::sqrt(read_scalar(ctx, s));
  double factor = 0.0;
  for (int it = 0; it < o->poly_factor_max_iter; ++it) {
    op_copy(ctx, n, y, x);
    op_spmv(ctx, A, x, y, pc->variant);
    op_dot(ctx, n, y, y, s);
    const double nrm = std::sqrt(read_scalar(ctx, s));
    factor = nrm / nk;
    nk = nrm;
  }
  nd.omega = 1. / factor;
}

template <class T>
void neumann_apply(ab2_context* ctx, const ab2_precond* pc, const T* x, T* y) {
  const int n = pc->A->n;
  const NeumannData& nd = pc->neu;
  T* t[3];
  if constexpr (sizeof(T) == 8) {
    for (int k = 0; k < 3; ++k) t[k] = nd.d_t[k];
  } else {
    for (int k = 0; k < 3; ++k) t[k] = nd.d_t32 + (size_t)k * n;
  }
  const T omega = (T)nd.omega;
  if (nd.order == 0) {  // copy then scal
    k_scale_copy<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, omega, x, y);
    check_launch(ctx, "neumann_scal");
    return;
  }
  const T* xin = x;
  if (x == y) {  // the last step writes y while others still read x as the iterate
    AB2_CUDA(cudaMemcpyAsync(t[2], x, sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
    xin = t[2];
  }
  const T* cur = xin;  // y = x
  for (int i = 0; i < nd.order; ++i) {
    const bool last = i + 1 == nd.order;
    T* out = last ? y : t[i & 1];
    with_view<T>(pc->A, pc->variant, [&](auto view) {
      k_neumann_step<<<(n + kThreads - 1) / kThreads, kThreads, 0, ctx->stream>>>(n, view, xin, cur, out, omega,
                                                                                  last ? 1 : 0);
    });
    check_launch(ctx, "neumann_step");
    cur = out;
  }
}

template void filu_apply<double>(ab2_context*, const ab2_precond*, const double*, double*);
template void filu_apply<float>(ab2_context*, const ab2_precond*, const float*, float*);
template void neumann_apply<double>(ab2_context*, const ab2_precond*, const double*, double*);
template void neumann_apply<float>(ab2_context*, const ab2_precond*, const float*, float*);

void filu_enable_f32(ab2_context* ctx, ab2_precond* pc) {
  FiluData& f = pc->fil;
  const int n = pc->A->n;
  const int nslices = (n + kSlice - 1) / kSlice;
  int lo = 0, uo = 0;
  AB2_CUDA(cudaMemcpyAsync(&lo, f.d_l_off + nslices, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaMemcpyAsync(&uo, f.d_u_off + nslices, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  const long long ls = std::max((long long)lo * kSlice, 1LL), us = std::max((long long)uo * kSlice, 1LL);
  f.d_l_v32 = dev_alloc<float>(ctx, (size_t)ls);
  f.d_u_v32 = dev_alloc<float>(ctx, (size_t)us);
  f.d_inv32 = dev_alloc<float>(ctx, (size_t)n);
  f.d_t32 = dev_alloc<float>(ctx, 2 * (size_t)n);
  op_to_f32(ctx, ls, f.d_l_v, f.d_l_v32);
  op_to_f32(ctx, us, f.d_u_v, f.d_u_v32);
  op_to_f32(ctx, n, f.d_inv, f.d_inv32);
}

void neumann_enable_f32(ab2_context* ctx, ab2_precond* pc) {
  require(pc->A->d_v32 != nullptr, "FP32 Neumann needs the matrix's FP32 values (AB2_FMT_F32)");
  pc->neu.d_t32 = dev_alloc<float>(ctx, 3 * (size_t)pc->A->n);
}

void filu_neumann_release(ab2_context* ctx, ab2_precond* pc) {
  FiluData& f = pc->fil;
  for (void* p : {(void*)f.d_l_off, (void*)f.d_l_ci, (void*)f.d_l_v, (void*)f.d_u_off, (void*)f.d_u_ci, (void*)f.d_u_v,
                  (void*)f.d_inv, (void*)f.d_t[0], (void*)f.d_t[1], (void*)f.d_l_v32, (void*)f.d_u_v32,
                  (void*)f.d_inv32, (void*)f.d_t32})
    dev_free(ctx, p);
  f = FiluData{};
  NeumannData& nd = pc->neu;
  for (double* t : nd.d_t) dev_free(ctx, t);
  dev_free(ctx, nd.d_t32);
  nd = NeumannData{};
}

}  // namespace ab2
