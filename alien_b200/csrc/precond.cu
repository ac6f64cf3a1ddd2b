// precond.cu -- Diag, ILU(0) and Chebyshev preconditioners on the device.
//
//   Diag       DiagPreconditioner.h:49-68            z = (1/a_ii) . r
//   ILU(0)     ILU0Preconditioner.h:71-248           IKJ factorisation, forward
//              (sequential branch)                   unit-L sweep, backward U sweep
//   Chebyshev  ChebyshevPreconditioner.h:73-202,     power-method bounds, then the
//              392-434 (_algo2)                      Ifpack2-style polynomial
//   FILU0, Neumann: filu.cu
//
// ILU(0): the factorisation and both sweeps keep the reference's arithmetic row
// by row (same column order, product and difference rounded apart, an IEEE
// division by the pivot),
// so the factor and every application are bit-identical to the sequential CPU
// code.  Parallelism comes from the wavefronts of the triangular graphs: rows
// in the same wavefront are independent.  The factorisation runs one launch
// per wavefront (set-up only).  The sweeps run as ONE launch each with no
// grid-wide barrier: warps take 32-row chunks in wavefront order from an
// atomic ticket and wait, per dependency, until the producer's value has been
// stored.  The value itself is the flag: the output vector is pre-filled with
// a signalling-NaN sentinel that arithmetic never produces, and a consumer
// polls the 8-byte word with ld.relaxed.gpu until it changes.  Tickets are
// handed out in order, so the chunk a warp waits on was taken earlier by a
// running warp, and every wait is bounded (clock64 budget) -- on expiry the
// kernel records an error and finishes instead of hanging.
//
// Chebyshev: each polynomial step is one fused SpMV kernel whose epilogue forms
// r = x - A y, z = D^-1 r, p = beta p + z and y' = y + a p in registers, with the
// reference's rounding (scal then axpy for p, fma for y).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <random>

#include "ab2_internal.cuh"
#include "precond.cuh"
#include "sentinel.cuh"
#include "spmv_view.cuh"

namespace ab2 {

namespace {

// acc - sum_{k in [kb, ke)} a_k x[c_k], k ascending, waiting for each x value to
// be produced.  Up to 8 dependencies are loaded at once, so a row whose inputs
// are ready costs one round trip to L2 instead of one per dependency; only the
// values still at the sentinel are polled again.
template <class T>
__device__ __forceinline__ T sweep_row(T acc, int kb, int ke, const int* __restrict__ ci, const T* __restrict__ lu,
                                       const T* x, int* err) {
  for (int k0 = kb; k0 < ke; k0 += 8) {
    T a[8], v[8];
    int c[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const bool in = k0 + u < ke;
      c[u] = in ? ci[k0 + u] : 0;
      a[u] = in ? lu[k0 + u] : T(0);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = k0 + u < ke ? ld_relaxed(x + c[u]) : T(0);
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (k0 + u < ke && is_sentinel(v[u])) v[u] = wait_value(x + c[u], err);
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (k0 + u < ke) acc = mul_sub_rn(a[u], v[u], acc);
  }
  return acc;
}

// One wavefront of the IKJ factorisation (ILU0Preconditioner.h:156-178): for
// each k left of the diagonal, a_ik /= a_kk, then a_ij -= a_ik a_kj for every
// j > k present in both rows (two-pointer merge of the sorted rows).
__global__ void k_ilu_factor_level(const int* __restrict__ rows, int count, const int* __restrict__ rp,
                                   const int* __restrict__ ci, const int* __restrict__ dcol, double* __restrict__ lu) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const int i = rows[t];
  if (i < 0) return;
  const int end = rp[i + 1];
  const int di = dcol[i];
  for (int k = rp[i]; k < di; ++k) {
    const int kr = ci[k];
    const int dk = dcol[kr];
    const double piv = dk < rp[kr + 1] ? lu[dk] : 0.0;
    const double aik = lu[k] / piv;
    lu[k] = aik;
    int l = rp[kr];
    const int le = rp[kr + 1];
    for (int j = k + 1; j < end; ++j) {
      const int cj = ci[j];
      while (l < le && ci[l] < cj) ++l;
      if (l == le) break;
      if (ci[l] == cj) lu[j] = mul_sub_rn(aik, lu[l], lu[j]);
    }
  }
}

// Forward sweep x_i = y_i - sum_{k<dcol} l_ik x_k (solveL, ILU0Preconditioner.h:181-198).
// Also leaves z at the sentinel for the backward sweep (after y_i was read, so
// y and z may be the same vector).
template <class T>
__global__ void __launch_bounds__(256) k_ilu_lsweep(int len, const int* __restrict__ perm, const int* __restrict__ rp,
                                                    const int* __restrict__ ci, const int* __restrict__ dcol,
                                                    const T* __restrict__ lu, const T* y, T* t, T* z,
                                                    unsigned int* tickets, int* err) {
  const int lane = threadIdx.x & 31;
  const int nchunks = len >> 5;
  for (;;) {
    int chunk = 0;
    if (lane == 0) chunk = (int)atomicAdd(tickets, 1u);
    chunk = __shfl_sync(0xffffffffu, chunk, 0);
    if (chunk >= nchunks) break;
    const int row = perm[chunk * 32 + lane];
    if (row >= 0) {
      const T acc = sweep_row(y[row], rp[row], dcol[row], ci, lu, t, err);
      z[row] = sentinel_of<T>();
      st_relaxed(t + row, not_sentinel(acc));
    }
  }
  // The backward sweep's ticket is reset here: it is not in use while this runs.
  if (blockIdx.x == 0 && threadIdx.x == 0) tickets[1] = 0u;
}

// Backward sweep x_i = (y_i - sum_{k>dcol} u_ik x_k) / u_ii (solveU, :200-231).
// Puts t back to the sentinel for the next forward sweep.
template <class T>
__global__ void __launch_bounds__(256) k_ilu_usweep(int len, const int* __restrict__ perm, const int* __restrict__ rp,
                                                    const int* __restrict__ ci, const int* __restrict__ dcol,
                                                    const T* __restrict__ lu, T* t, T* z,
                                                    unsigned int* tickets, int* err) {
  const int lane = threadIdx.x & 31;
  const int nchunks = len >> 5;
  for (;;) {
    int chunk = 0;
    if (lane == 0) chunk = (int)atomicAdd(tickets + 1, 1u);
    chunk = __shfl_sync(0xffffffffu, chunk, 0);
    if (chunk >= nchunks) break;
    const int row = perm[chunk * 32 + lane];
    if (row >= 0) {
      const int dk = dcol[row];
      const int e = rp[row + 1];
      const T acc = sweep_row(t[row], dk + 1, e, ci, lu, z, err);
      const T piv = dk < e ? lu[dk] : T(0);
      t[row] = sentinel_of<T>();
      st_relaxed(z + row, not_sentinel(acc / piv));
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) tickets[0] = 0u;
}

// Chebyshev step (ChebyshevPreconditioner.h:392-434 with y_cur the iterate):
//   r = x - A y_cur ; z = D^-1 r ; p = first ? z : beta*p + z ; y_next = y_cur + a p
template <class View, class T>
__global__ void __launch_bounds__(kThreads) k_cheb_step(int n, View A, const T* __restrict__ x, const T* __restrict__ ycur,
                                                        const T* __restrict__ inv, T* __restrict__ p,
                                                        T* __restrict__ ynext, T a, T bcoef, int first) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const T ay = A.row(row, ycur);
  const T r = fma_rn(T(-1), ay, x[row]);
  const T z = mul_rn(inv[row], r);
  const T pn = first ? z : add_rn(mul_rn(bcoef, p[row]), z);
  p[row] = pn;
  ynext[row] = fma_rn(a, pn, ycur[row]);
}

// _algo1 start (ChebyshevPreconditioner.h:329-336): r = D^-1 x ; w = r / theta ; y = w.
// x and y may be the same vector (x_i is read before y_i is written).
template <class T>
__global__ void k_cheb1_start(int n, const T* x, const T* __restrict__ inv, T inv_theta, T* __restrict__ r,
                              T* __restrict__ w, T* y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T rv = mul_rn(inv[i], x[i]);
    const T wv = mul_rn(inv_theta, rv);
    r[i] = rv;
    w[i] = wv;
    y[i] = wv;
  }
}

// _algo1 step (:342-354): r -= D^-1 A w ; w = c1 w + c2 r ; y += w, with the
// rounding of pointwiseMult, axpy(-1), scal, axpy(c2), axpy(1).
template <class View, class T>
__global__ void __launch_bounds__(kThreads) k_cheb1_step(int n, View A, const T* __restrict__ inv, T* __restrict__ r,
                                                         const T* __restrict__ wcur, T* __restrict__ wnext,
                                                         T* __restrict__ y, T c1, T c2) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  // mul_rn: the products are rounded on their own, as pointwiseMult and
  // scal round them; a plain '*' could be fused into the following update.
  const T my = mul_rn(inv[row], A.row(row, wcur));
  const T rv = fma_rn(T(-1), my, r[row]);
  r[row] = rv;
  const T wv = fma_rn(c2, rv, mul_rn(c1, wcur[row]));
  wnext[row] = wv;
  y[row] = fma_rn(T(1), wv, y[row]);
}

__global__ void k_sqrt(int n, const double* __restrict__ a, double* __restrict__ s) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s[i] = sqrt(a[i]);
}

// Smallest and largest eigenvalue of the symmetric tridiagonal matrix with
// diagonal a[0..m) and off-diagonal b[0..m-1): bisection on Sturm counts,
// 128 halvings of the Gershgorin interval.
void tridiag_extremes(const std::vector<double>& a, const std::vector<double>& b, double* lmin, double* lmax) {
  const int m = (int)a.size();
  double lo = a[0], hi = a[0];
  for (int i = 0; i < m; ++i) {
    const double rad = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < m ? std::fabs(b[i]) : 0.0);
    lo = std::min(lo, a[i] - rad);
    hi = std::max(hi, a[i] + rad);
  }
  auto below = [&](double x) {
    int cnt = 0;
    double d = 1.0;
    for (int i = 0; i < m; ++i) {
      d = (a[i] - x) - (i > 0 ? b[i - 1] * b[i - 1] / d : 0.0);
      if (d == 0.0) d = -1e-300;
      cnt += d < 0.0;
    }
    return cnt;
  };
  auto kth = [&](int k) {
    double l = lo, h = hi;
    for (int it = 0; it < 128; ++it) {
      const double mid = 0.5 * (l + h);
      if (below(mid) >= k) h = mid;
      else l = mid;
    }
    return h;
  };
  *lmin = kth(1);
  *lmax = kth(m);
}

template <class T>
__global__ void k_pmult2(int n, const T* __restrict__ a, const T* x, T* y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = mul_rn(a[i], x[i]);
}

void ilu_symbolic(const ab2_matrix* A, Ilu0Data& d) {
  host_profile(A);
  const int n = A->n;
  const int* rp = A->h_rp.data();
  const int* ci = A->h_ci.data();
  std::vector<int> dc(n);
  for (int i = 0; i < n; ++i) {
    int k = rp[i];
    while (k < rp[i + 1] && ci[k] < i) ++k;
    dc[i] = k;
  }
  std::vector<int> lev_l(n, 0), lev_u(n, 0);
  int max_l = -1, max_u = -1;
  for (int i = 0; i < n; ++i) {
    int lv = 0;
    for (int k = rp[i]; k < dc[i]; ++k) lv = std::max(lv, lev_l[ci[k]] + 1);
    lev_l[i] = lv;
    max_l = std::max(max_l, lv);
  }
  for (int i = n - 1; i >= 0; --i) {
    int lv = 0;
    for (int k = dc[i] + 1; k < rp[i + 1]; ++k) lv = std::max(lv, lev_u[ci[k]] + 1);
    lev_u[i] = lv;
    max_u = std::max(max_u, lv);
  }
  auto build = [n](const std::vector<int>& lev, int nlev, bool descending, std::vector<int>& perm,
                   std::vector<int>& ptr) {
    std::vector<int> cnt(nlev, 0);
    for (int i = 0; i < n; ++i) cnt[lev[i]]++;
    ptr.assign(nlev + 1, 0);
    for (int l = 0; l < nlev; ++l) ptr[l + 1] = ptr[l] + ((cnt[l] + 31) / 32) * 32;
    perm.assign(ptr[nlev], -1);
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    if (!descending) {
      for (int i = 0; i < n; ++i) perm[fill[lev[i]]++] = i;
    } else {
      for (int i = n - 1; i >= 0; --i) perm[fill[lev[i]]++] = i;
    }
  };
  std::vector<int> perm_u, ptr_u;
  d.levels_l = max_l + 1;
  d.levels_u = max_u + 1;
  build(lev_l, d.levels_l, false, d.h_perm_l, d.lev_ptr_l);
  build(lev_u, d.levels_u, true, perm_u, ptr_u);
  d.widest_l = d.widest_u = 1;
  for (int l = 0; l < d.levels_l; ++l) d.widest_l = std::max(d.widest_l, (d.lev_ptr_l[l + 1] - d.lev_ptr_l[l]) / 32);
  for (int l = 0; l < d.levels_u; ++l) d.widest_u = std::max(d.widest_u, (ptr_u[l + 1] - ptr_u[l]) / 32);
  d.len_l = (int)d.h_perm_l.size();
  d.len_u = (int)perm_u.size();
  d.d_perm_l = dev_alloc<int>(A->ctx, d.h_perm_l.size());
  d.d_perm_u = dev_alloc<int>(A->ctx, perm_u.size());
  AB2_CUDA(cudaMemcpy(d.d_perm_l, d.h_perm_l.data(), sizeof(int) * d.h_perm_l.size(), cudaMemcpyHostToDevice));
  AB2_CUDA(cudaMemcpy(d.d_perm_u, perm_u.data(), sizeof(int) * perm_u.size(), cudaMemcpyHostToDevice));
}

// Warps of a sweep: a few wavefronts' worth.  Every warp beyond the ones the
// current wavefront can use only polls, and polling traffic slows the L2 the
// producers write through, so the grid is sized to keep about three
// wavefronts in flight (the AB2_ILU_WINDOW environment variable overrides the
// three, for tuning).
int sweep_blocks(ab2_context* ctx, int len, int widest_chunks) {
  static const int window = [] {
    const char* e = std::getenv("AB2_ILU_WINDOW");
    return e ? std::max(1, std::atoi(e)) : 3;
  }();
  const long long warps = std::min<long long>((long long)widest_chunks * window, len / 32);
  const int blocks = (int)((warps + 7) / 8);
  return std::max(1, std::min(blocks, ctx->num_sms * 8));
}

}  // namespace

void ilu_init(ab2_context* ctx, ab2_precond* pc, int schedule, const double* lu) {
  const ab2_matrix* A = pc->A;
  Ilu0Data& d = pc->ilu;
  d.d_lu = dev_alloc<double>(ctx, (size_t)A->nnz);
  d.d_tmp = dev_alloc<double>(ctx, (size_t)A->n);
  d.d_counters = dev_alloc<unsigned int>(ctx, 2);
  d.d_err = dev_alloc<int>(ctx, 1);
  AB2_CUDA(cudaMemsetAsync(d.d_counters, 0, 2 * sizeof(unsigned int), ctx->stream));
  AB2_CUDA(cudaMemsetAsync(d.d_err, 0, sizeof(int), ctx->stream));
  AB2_CUDA(cudaMemcpyAsync(d.d_lu, lu ? lu : A->d_v, sizeof(double) * (size_t)A->nnz, cudaMemcpyDeviceToDevice,
                           ctx->stream));
  k_fill_bits<<<grid_for(A->n), kThreads, 0, ctx->stream>>>(A->n, kSentinel, d.d_tmp);
  check_launch(ctx, "ilu_fill");
  if (schedule != AB2_ILU_WAVEFRONT && ilu_stencil_setup(ctx, A, d, lu != nullptr, schedule)) return;
  require(schedule != AB2_ILU_STENCIL && schedule != AB2_ILU_STENCIL_CLUSTER,
          "ILU0 tile schedule requested but the matrix is not a 3-D 7-point matrix in lexicographic order");
  ilu_symbolic(A, d);
  if (lu) return;
  for (int l = 1; l < d.levels_l; ++l) {  // wavefront 0 rows have nothing left of the diagonal
    const int a = d.lev_ptr_l[l], b = d.lev_ptr_l[l + 1];
    const int cnt = b - a;
    if (cnt == 0) continue;
    k_ilu_factor_level<<<(cnt + 127) / 128, 128, 0, ctx->stream>>>(d.d_perm_l + a, cnt, A->d_rp, A->d_ci, A->d_dcol,
                                                                   d.d_lu);
    check_launch(ctx, "ilu_factor");
  }
}

void ilu_drop_schedule(ab2_context* ctx, Ilu0Data& d) {
  for (void* p : {(void*)d.d_perm_l, (void*)d.d_perm_u, (void*)d.d_tmp, (void*)d.d_counters, (void*)d.d_err,
                  (void*)d.d_bands, (void*)d.d_walk, (void*)d.d_walk32, (void*)d.d_tile_tickets})
    dev_free(ctx, p);
  double* lu = d.d_lu;
  d = Ilu0Data{};
  d.d_lu = lu;
}

namespace {

void cheb_init(ab2_context* ctx, ab2_precond* pc, const ab2_precond_options* o) {
  const ab2_matrix* A = pc->A;
  const int n = A->n;
  ChebData& c = pc->cheb;
  c.order = o->poly_order;
  c.d_p = dev_alloc<double>(ctx, (size_t)n);
  c.d_y[0] = dev_alloc<double>(ctx, (size_t)n);
  c.d_y[1] = dev_alloc<double>(ctx, (size_t)n);
  c.d_xcopy = dev_alloc<double>(ctx, (size_t)n);
  double* x = dev_alloc<double>(ctx, (size_t)n);
  double* y = c.d_y[0];
  double* s = red_slot(ctx, 0).result;
  double* s_out = s;
  c.saad = o->cheb_saad != 0;
  op_fill(ctx, n, 0.0, y);
  op_fill(ctx, n, 0.0, c.d_p);
  // Both power methods draw their start vector from a default-seeded
  // std::mt19937 with U(-1,1), index order (computeBeta :124-129, computeAlpha :166-172).
  std::vector<double> h(n);
  auto power = [&](bool shift, double b) {
    std::mt19937 gen;
    std::uniform_real_distribution<> dis(-1., 1.);
    for (int i = 0; i < n; ++i) h[i] = dis(gen);
    AB2_CUDA(cudaMemcpyAsync(x, h.data(), sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    op_dot(ctx, n, x, x, s);
    const double nrm = std::sqrt(read_scalar(ctx, s));
    op_scal(ctx, n, 1 / nrm, x);
    double est = 0.0;
    for (int it = 0; it < o->poly_factor_max_iter; ++it) {
      op_spmv(ctx, A, x, y, pc->variant);
      op_pmult(ctx, n, pc->d_inv, y, y);
      if (shift) op_axpy(ctx, n, -b, x, y);
      op_dot(ctx, n, y, x, s);
      const double xax = read_scalar(ctx, s);
      op_dot(ctx, n, x, x, s);
      const double xdx = read_scalar(ctx, s);
      est = xax / xdx;
      op_dot(ctx, n, y, y, s);
      const double nr = std::sqrt(read_scalar(ctx, s));
      op_scal(ctx, n, 1 / nr, y);
      op_copy(ctx, n, y, x);
    }
    return shift ? est + b : est;
  };
  // Lanczos on S A S, S = diag(sqrt(1/a_ii)), from the same start vector:
  // alpha = smallest Ritz value, beta = 1.1 x the largest.
  auto lanczos = [&](int steps) {
    double* s = dev_alloc<double>(ctx, (size_t)n);
    double* vp = dev_alloc<double>(ctx, (size_t)n);
    double* t = dev_alloc<double>(ctx, (size_t)n);
    double* w = c.d_xcopy;  // free until the first application
    k_sqrt<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, pc->d_inv, s);
    check_launch(ctx, "sqrt");
    std::mt19937 gen;
    std::uniform_real_distribution<> dis(-1., 1.);
    for (int i = 0; i < n; ++i) h[i] = dis(gen);
    AB2_CUDA(cudaMemcpyAsync(x, h.data(), sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    op_dot(ctx, n, x, x, s_out);
    const double nrm = std::sqrt(read_scalar(ctx, s_out));
    op_scal(ctx, n, 1 / nrm, x);
    std::vector<double> ta, tb;
    double bprev = 0.0;
    const int m = std::max(steps, 1);
    for (int j = 0; j < m; ++j) {
      op_pmult(ctx, n, s, x, t);
      op_spmv(ctx, A, t, w, pc->variant);
      op_pmult(ctx, n, s, w, w);
      if (j > 0) op_axpy(ctx, n, -bprev, vp, w);
      op_dot(ctx, n, w, x, s_out);
      const double aj = read_scalar(ctx, s_out);
      op_axpy(ctx, n, -aj, x, w);
      op_dot(ctx, n, w, w, s_out);
      const double bj = std::sqrt(read_scalar(ctx, s_out));
      ta.push_back(aj);
      if (bj == 0.0 || j + 1 == m) break;
      tb.push_back(bj);
      op_copy(ctx, n, x, vp);
      op_copy(ctx, n, w, x);
      op_scal(ctx, n, 1 / bj, x);
      bprev = bj;
    }
    double lmin = 0.0, lmax = 0.0;
    tridiag_extremes(ta, tb, &lmin, &lmax);
    c.alpha = lmin;
    c.beta = 1.1 * lmax;
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    dev_free(ctx, s);
    dev_free(ctx, vp);
    dev_free(ctx, t);
  };
  if (o->cheb_lanczos) {
    lanczos(o->poly_factor_max_iter);
  } else {
    c.beta = power(false, 0.0);
    c.alpha = power(true, c.beta);
  }
  if (o->poly_factor != 0.) c.alpha = c.beta / o->poly_factor;
  dev_free(ctx, x);
  op_fill(ctx, n, 0.0, y);
  const int steps = std::max(1, c.order);
  c.a.assign(steps, 0.0);
  c.b.assign(steps, 0.0);
  if (c.saad) {
    // _algo1 scalars (ChebyshevPreconditioner.h:316-351), in the reference's order.
    const double delta = (c.beta - c.alpha) / 2;
    const double theta = (c.beta + c.alpha) / 2;
    const double sigma = theta / delta;
    double rho_old = 1. / sigma;
    c.inv_theta = 1 / theta;
    for (int k = 1; k < steps; ++k) {
      const double rho = 1. / (2 * sigma - rho_old);
      c.a[k] = rho * rho_old;
      c.b[k] = 2 * rho / delta;
      rho_old = rho;
    }
    return;
  }
  // Step coefficients of _algo2, evaluated in the reference's order.
  const double dd = (c.beta + c.alpha) / 2;
  const double cc = (c.beta - c.alpha) / 2;
  double a = 2 / dd;
  c.a[0] = a;
  for (int i = 1; i < steps; ++i) {
    const double beta = a * (cc / 2.) * (cc / 2.);
    a = 1. / (dd - beta);
    c.b[i] = beta;
    c.a[i] = a;
  }
}

}  // namespace

namespace {

// The FP64 or FP32 arrays of a preconditioner.
template <class T>
struct PcArrays;
template <>
struct PcArrays<double> {
  const double* inv;
  const double* lu;
  double* tmp;
  double *p, *y0, *y1, *xcopy;
  explicit PcArrays(const ab2_precond* pc)
      : inv(pc->d_inv), lu(pc->ilu.d_lu), tmp(pc->ilu.d_tmp), p(pc->cheb.d_p), y0(pc->cheb.d_y[0]),
        y1(pc->cheb.d_y[1]), xcopy(pc->cheb.d_xcopy) {}
};
template <>
struct PcArrays<float> {
  const float* inv;
  const float* lu;
  float* tmp;
  float *p, *y0, *y1, *xcopy;
  explicit PcArrays(const ab2_precond* pc) : inv(pc->d_inv32), lu(pc->d_lu32), tmp(pc->d_tmp32) {
    const size_t n = (size_t)pc->A->n;
    float* c = pc->d_cheb32;
    p = c;
    y0 = c ? c + n : nullptr;
    y1 = c ? c + 2 * n : nullptr;
    xcopy = c ? c + 3 * n : nullptr;
  }
};

template <class T>
void copy_t(ab2_context* ctx, int n, const T* x, T* y) {
  if (x == y) return;
  AB2_CUDA(cudaMemcpyAsync(y, x, sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
}

template <class T>
void apply_t(ab2_context* ctx, const ab2_precond* pc, const T* x, T* y) {
  const int n = pc->A->n;
  if (n == 0) return;
  const PcArrays<T> w(pc);
  switch (pc->kind) {
    case AB2_PC_NONE: copy_t(ctx, n, x, y); break;
    case AB2_PC_DIAG:
      k_pmult2<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, w.inv, x, y);
      check_launch(ctx, "diag_apply");
      break;
    case AB2_PC_ILU0: {
      const Ilu0Data& d = pc->ilu;
      const ab2_matrix* A = pc->A;
      if (d.stencil) {
        if constexpr (sizeof(T) == 8) ilu_stencil_apply(ctx, A, d, x, y);
        else ilu_stencil_apply_f32(ctx, d, x, y);
        break;
      }
      k_ilu_lsweep<T><<<sweep_blocks(ctx, d.len_l, d.widest_l), 256, 0, ctx->stream>>>(
          d.len_l, d.d_perm_l, A->d_rp, A->d_ci, A->d_dcol, w.lu, x, w.tmp, y, d.d_counters, d.d_err);
      check_launch(ctx, "ilu_lsweep");
      k_ilu_usweep<T><<<sweep_blocks(ctx, d.len_u, d.widest_u), 256, 0, ctx->stream>>>(
          d.len_u, d.d_perm_u, A->d_rp, A->d_ci, A->d_dcol, w.lu, w.tmp, y, d.d_counters, d.d_err);
      check_launch(ctx, "ilu_usweep");
      break;
    }
    case AB2_PC_CHEB: {
      const ChebData& c = pc->cheb;
      const int steps = std::max(1, c.order);
      if (c.saad) {
        T* r = w.p;
        T* wv[2] = {w.y0, w.y1};
        k_cheb1_start<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, x, w.inv, (T)c.inv_theta, r, wv[0], y);
        check_launch(ctx, "cheb1_start");
        for (int k = 1; k < steps; ++k) {
          const T* wcur = wv[(k - 1) & 1];
          T* wnext = wv[k & 1];
          with_view<T>(pc->A, pc->variant, [&](auto view) {
            k_cheb1_step<<<(n + kThreads - 1) / kThreads, kThreads, 0, ctx->stream>>>(n, view, w.inv, r, wcur, wnext,
                                                                                      y, (T)c.a[k], (T)c.b[k]);
          });
          check_launch(ctx, "cheb1_step");
        }
        break;
      }
      const T* xin = x;
      if (x == y) {
        copy_t(ctx, n, x, w.xcopy);
        xin = w.xcopy;
      }
      const T* cur = xin;
      T* ys[2] = {w.y0, w.y1};
      for (int i = 0; i < steps; ++i) {
        T* next = (i == steps - 1) ? y : ys[i & 1];
        with_view<T>(pc->A, pc->variant, [&](auto view) {
          k_cheb_step<<<(n + kThreads - 1) / kThreads, kThreads, 0, ctx->stream>>>(n, view, xin, cur, w.inv, w.p, next,
                                                                                   (T)c.a[i], (T)c.b[i], i == 0);
        });
        check_launch(ctx, "cheb_step");
        cur = next;
      }
      break;
    }
    case AB2_PC_FILU0: filu_apply<T>(ctx, pc, x, y); break;
    case AB2_PC_NEUMANN: neumann_apply<T>(ctx, pc, x, y); break;
    default: throw Error{AB2_ERR_BAD_ARG, "unknown preconditioner"};
  }
}

}  // namespace

void pc_apply(ab2_context* ctx, const ab2_precond* pc, const double* x, double* y) { apply_t(ctx, pc, x, y); }

void pc_enable_f32(ab2_context* ctx, ab2_precond* pc) {
  if (pc->f32) return;
  const ab2_matrix* A = pc->A;
  const int n = A->n;
  if (pc->d_inv) {
    pc->d_inv32 = dev_alloc<float>(ctx, (size_t)n);
    op_to_f32(ctx, n, pc->d_inv, pc->d_inv32);
  }
  if (pc->kind == AB2_PC_CHEB) {
    require(A->d_v32 != nullptr, "FP32 Chebyshev needs the matrix's FP32 values (AB2_FMT_F32)");
    pc->d_cheb32 = dev_alloc<float>(ctx, 4 * (size_t)std::max(n, 1));
    AB2_CUDA(cudaMemsetAsync(pc->d_cheb32, 0, sizeof(float) * 4 * (size_t)std::max(n, 1), ctx->stream));
  }
  if (pc->kind == AB2_PC_ILU0) {
    if (pc->ilu.stencil) {
      ilu_stencil_enable_f32(ctx, pc->ilu);
    } else {
      pc->d_lu32 = dev_alloc<float>(ctx, (size_t)A->nnz);
      op_to_f32(ctx, A->nnz, pc->ilu.d_lu, pc->d_lu32);
      pc->d_tmp32 = dev_alloc<float>(ctx, (size_t)n);
      k_fill_bits32<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, kSentinel32, pc->d_tmp32);
      check_launch(ctx, "ilu_fill32");
    }
  }
  if (pc->kind == AB2_PC_FILU0) filu_enable_f32(ctx, pc);
  if (pc->kind == AB2_PC_NEUMANN) neumann_enable_f32(ctx, pc);
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  pc->f32 = true;
}

void pc_apply_f32(ab2_context* ctx, const ab2_precond* pc, const float* x, float* y) {
  require(pc->f32, "preconditioner has no FP32 form (pc_enable_f32)");
  apply_t(ctx, pc, x, y);
}

void pc_reset(ab2_context* ctx, const ab2_precond* pc) {
  if (pc->kind != AB2_PC_ILU0) return;
  const Ilu0Data& d = pc->ilu;
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  k_fill_bits<<<grid_for(pc->A->n), kThreads, 0, ctx->stream>>>(pc->A->n, kSentinel, d.d_tmp);
  check_launch(ctx, "ilu_fill");
  if (pc->d_tmp32) {
    k_fill_bits32<<<grid_for(pc->A->n), kThreads, 0, ctx->stream>>>(pc->A->n, kSentinel32, pc->d_tmp32);
    check_launch(ctx, "ilu_fill32");
  }
  AB2_CUDA(cudaMemsetAsync(d.d_counters, 0, 2 * sizeof(unsigned int), ctx->stream));
  if (d.d_tile_tickets) AB2_CUDA(cudaMemsetAsync(d.d_tile_tickets, 0, 3 * sizeof(unsigned int), ctx->stream));
  if (d.stencil) ilu_stencil_reset(ctx, d);
  AB2_CUDA(cudaMemsetAsync(d.d_err, 0, sizeof(int), ctx->stream));
}

int pc_error(ab2_context* ctx, const ab2_precond* pc) {
  if (pc->kind != AB2_PC_ILU0) return 0;
  int e = 0;
  AB2_CUDA(cudaMemcpyAsync(&e, pc->ilu.d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  return e;
}

}  // namespace ab2

using namespace ab2;

extern "C" {

int ab2_precond_create(ab2_context* ctx, const ab2_matrix* A, const ab2_precond_options* o, ab2_precond** out) {
  if (!ctx || !A || !o || !out) return AB2_ERR_BAD_ARG;
  *out = nullptr;
  if (o->kind < AB2_PC_NONE || o->kind > AB2_PC_NEUMANN) return AB2_ERR_BAD_ARG;
  ab2_precond* pc = new (std::nothrow) ab2_precond();
  if (!pc) return AB2_ERR_OOM;
  pc->ctx = ctx_retain(ctx);
  int rc = guard(ctx, [&] {
    pc->A = A;
    pc->kind = o->kind;
    if (o->kind == AB2_PC_DIAG || o->kind == AB2_PC_CHEB) {
      pc->d_inv = dev_alloc<double>(ctx, (size_t)A->n);
      // init(): assign(inv, 1) then computeInvDiag (DiagPreconditioner.h:49-54)
      op_inv_diag(ctx, A, pc->d_inv);
    }
    if (o->kind == AB2_PC_ILU0) {
      require(o->ilu_schedule >= AB2_ILU_AUTO && o->ilu_schedule <= AB2_ILU_STENCIL_CLUSTER, "unknown ILU0 schedule");
      ilu_init(ctx, pc, o->ilu_schedule);
    }
    if (o->kind == AB2_PC_CHEB) {
      require(o->poly_factor_max_iter >= 0, "poly_factor_max_iter must be >= 0");
      cheb_init(ctx, pc, o);
    }
    if (o->kind == AB2_PC_FILU0) filu_init(ctx, pc, o);
    if (o->kind == AB2_PC_NEUMANN) neumann_init(ctx, pc, o);
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  });
  if (rc != AB2_OK) {
    ab2_precond_destroy(pc);
    return rc;
  }
  *out = pc;
  return AB2_OK;
}

int ab2_precond_apply(ab2_context* ctx, const ab2_precond* pc, const ab2_vector* x, ab2_vector* y) {
  if (!ctx || !pc || !x || !y || x->n != pc->A->n || y->n != pc->A->n) return AB2_ERR_BAD_ARG;
  static const char* const kPhase[] = {"PRECOND-NONE", "PRECOND-DIAG", "PRECOND-ILU0", "PRECOND-CHEB", "PRECOND-FILU0",
                                       "PRECOND-NEUMANN"};
  PhaseScope phase_scope(ctx, kPhase[pc->kind]);
  return guard(ctx, [&] { pc_apply(ctx, pc, x->d, y->d); });
}

int ab2_precond_destroy(ab2_precond* pc) {
  if (!pc) return AB2_ERR_BAD_ARG;
  if (pc->ctx) ctx_quiesce(pc->ctx);
  dev_free(pc->ctx, pc->d_inv);
  dev_free(pc->ctx, pc->ilu.d_lu);
  dev_free(pc->ctx, pc->ilu.d_perm_l);
  dev_free(pc->ctx, pc->ilu.d_perm_u);
  dev_free(pc->ctx, pc->ilu.d_tmp);
  dev_free(pc->ctx, pc->ilu.d_counters);
  dev_free(pc->ctx, pc->ilu.d_err);
  dev_free(pc->ctx, pc->ilu.d_bands);
  dev_free(pc->ctx, pc->ilu.d_walk);
  dev_free(pc->ctx, pc->ilu.d_walk32);
  dev_free(pc->ctx, pc->ilu.d_tile_tickets);
  dev_free(pc->ctx, pc->cheb.d_p);
  dev_free(pc->ctx, pc->cheb.d_y[0]);
  dev_free(pc->ctx, pc->cheb.d_y[1]);
  dev_free(pc->ctx, pc->cheb.d_xcopy);
  dev_free(pc->ctx, pc->d_inv32);
  dev_free(pc->ctx, pc->d_lu32);
  dev_free(pc->ctx, pc->d_tmp32);
  dev_free(pc->ctx, pc->d_cheb32);
  filu_neumann_release(pc->ctx, pc);
  if (pc->ctx) ctx_release(pc->ctx);
  delete pc;
  return AB2_OK;
}

int ab2_precond_get_info(const ab2_precond* pc, ab2_precond_info* info) {
  if (!pc || !info) return AB2_ERR_BAD_ARG;
  info->kind = pc->kind;
  info->cheb_alpha = pc->cheb.alpha;
  info->cheb_beta = pc->cheb.beta;
  info->ilu_levels_lower = pc->ilu.levels_l;
  info->ilu_levels_upper = pc->ilu.levels_u;
  info->ilu_schedule = pc->kind != AB2_PC_ILU0 ? 0
                      : pc->ilu.stencil ? (pc->ilu.walk_cluster ? AB2_ILU_STENCIL_CLUSTER : AB2_ILU_STENCIL)
                                        : AB2_ILU_WAVEFRONT;
  info->neumann_factor = pc->neu.omega;
  return AB2_OK;
}

int ab2_precond_ilu0_values(ab2_context* ctx, const ab2_precond* pc, double* lu) {
  if (!ctx || !pc || !lu || (pc->kind != AB2_PC_ILU0 && pc->kind != AB2_PC_FILU0)) return AB2_ERR_BAD_ARG;
  return guard(ctx, [&] {
    AB2_CUDA(cudaMemcpyAsync(lu, pc->ilu.d_lu, sizeof(double) * (size_t)pc->A->nnz, cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

}  // extern "C"
