// ab2_oracle.cpp -- CPU oracle for the alien-b200 hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: it is loaded by the
// tests, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg, and by
// nothing else.  The product (libab2) never links or calls it.
//
// It restates, sequentially and in plain C++, the arithmetic of Alien's
// SimpleCSR internal algebra and of the header-only Krylov templates:
//
//   SpMV            src/core/alien/kernels/simple_csr/algebra/SimpleCSRMatrixMultT.h:172-191
//   addL/UMult      SimpleCSRMatrixMultT.h:193-233
//   invdiag         SimpleCSRMatrixMultT.h:494-509, dcol from CSRStructInfo.h:291-309
//   BLAS-1          src/core/alien/kernels/simple_csr/algebra/CBLASMPIKernel.h:37-125
//                   (norm2 = sqrt(dot), SimpleCSRInternalLinearAlgebra.cc:102-108)
//   Iteration       src/core/alien/expression/krylov/Iteration.h:44-90
//   CG              src/core/alien/expression/krylov/CG.h:59-150
//   BiCGStab        src/core/alien/expression/krylov/BiCGStab.h:45-136 (its Iteration), 152-300
//   Diag            src/core/alien/expression/krylov/DiagPreconditioner.h:49-68
//   ILU0            src/core/alien/expression/krylov/ILU0Preconditioner.h:71-248 (sequential branch)
//   Chebyshev       src/core/alien/expression/krylov/ChebyshevPreconditioner.h:73-202, 392-434
//   BEllPack layout src/core/alien/kernels/sycl/data/SYCLBEllPackMatrix.cc:70-88 (slice S)
//
// Floating-point conventions (the GPU path follows the same ones, so it can
// match bit for bit wherever the reference's own order is sequential):
//   * loops written in Alien's sources as `a += b*c` / `a -= b*c` (SpMV,
//     addL/UMult, ILU0 factorisation and sweeps) round the product and the sum
//     separately: that is how the stock build compiles them (ISO -std=c++17
//     turns contraction off; without -march there is no FMA anyway).  The
//     reference templates built by oracle/Makefile confirm it bit for bit;
//   * BLAS-1 (cblas_daxpy etc.) is one fma per element, as CBLAS kernels on
//     FMA hardware compute it;
//   * dot products sum sequentially with fma, which is one admissible order of
//     cblas_ddot; the GPU uses a fixed tree, so dots agree to rounding only.
// The file is compiled with -ffp-contract=off so that only explicit std::fma
// calls fuse.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>
#include <algorithm>

#include "simplecsr_kernels.h"

extern "C" {

// Codes shared with include/ab2.h (same numeric values).
enum {
  ORC_OK = 0,
  ORC_ERR_BREAKDOWN = -3,
  ORC_ERR_NOT_CONVERGED = -4,
  ORC_ERR_BAD_ARG = -6,
};
enum { ORC_SOLVER_CG = 0, ORC_SOLVER_BICGSTAB = 1 };
enum { ORC_PC_NONE = 0, ORC_PC_DIAG = 1, ORC_PC_ILU0 = 2, ORC_PC_CHEB = 3, ORC_PC_FILU0 = 4, ORC_PC_NEUMANN = 5 };
// Which scalar broke down (the string passed to NullValueException).
enum { ORC_BD_NONE = 0, ORC_BD_ALPHA = 1, ORC_BD_BETA = 2, ORC_BD_RHO = 3 };

typedef struct {
  int solver;               // ORC_SOLVER_*
  int precond;              // ORC_PC_*
  double tol;
  int max_iter;
  double poly_factor;       // Chebyshev "factor" (0 = computed bounds)
  int poly_order;           // Chebyshev polynomial order
  int poly_factor_max_iter; // power-method steps for each bound
  // Summation order of every dot product: 0 = sequential (one admissible
  // cblas_ddot order, the reference templates' shim uses it); 1 = libab2's
  // device tree with `tree_blocks` blocks at most (bit-exact GPU checks).
  int dot_mode;
  int tree_blocks;
  int cheb_saad;     // 1: ChebyshevPreconditioner<AlgebraT, true> (_algo1)
  int cheb_lanczos;  // 1: bounds from poly_factor_max_iter Lanczos steps
  int filu_factor_iter;  // FILU0 nb-factor-iter (0: exact ILU(0) factor)
  int filu_solver_iter;  // FILU0 nb-solver-iter
} orc_options;

typedef struct {
  int iterations;        // Iteration::operator()()
  int converged;         // Iteration::getStatus()
  int error;             // ORC_OK or ORC_ERR_BREAKDOWN
  int breakdown;         // ORC_BD_*
  double nrm2_b;         // b.b
  double last_rr;        // last value the stop test compared (r.r or s.s)
  double cheb_alpha;     // Chebyshev bounds actually used
  double cheb_beta;
  int history_len;       // entries written into hist
} orc_result;

// Mixed-precision refinement (libab2's ab2_mixed, no reference counterpart):
// FP64 residual and update, FP32 inner CG/BiCGStab from the reference
// templates' arithmetic instantiated in float.
typedef struct {
  int solver;               // inner ORC_SOLVER_*
  int precond;              // inner ORC_PC_* (FP64 set-up, applied in float)
  double tol;               // true relative residual, FP64
  int max_outer;
  double inner_tol;
  int inner_max_iter;
  double poly_factor;
  int poly_order;
  int poly_factor_max_iter;
  int cheb_saad;
  int cheb_lanczos;
  int dot_mode;             // as orc_options, for the FP64 and the FP32 dots
  int tree_blocks;
  int filu_factor_iter;
  int filu_solver_iter;
  int jacobi_scaled;        // CG + Diag in the scaled form (mixed.cu's AB2_MIXED_JACOBI_SCALED)
} orc_mixed_options;

typedef struct {
  int succeeded;
  int outer_iterations;
  int inner_iterations;
  int error;                // ORC_OK, ORC_ERR_NOT_CONVERGED, ORC_ERR_BREAKDOWN
  double true_residual;
  int history_len;          // true relative residuals written into hist
} orc_mixed_result;

}  // extern "C"

namespace {

using namespace ab2_oracle;

// One warp's __shfl_down_sync tree (offsets 16..1): lane l adds lane l+off's
// value when l+off < 32; the result is lane 0's.
template <class T>
T warp_tree(const T* in) {
  T v[32], w[32];
  for (int l = 0; l < 32; ++l) v[l] = in[l];
  for (int off = 16; off > 0; off >>= 1) {
    for (int l = 0; l < 32; ++l) w[l] = v[l] + (l + off < 32 ? v[l + off] : v[l]);
    for (int l = 0; l < 32; ++l) v[l] = w[l];
  }
  return v[0];
}

// libab2's deterministic grid reduction (reduce.cuh), restated: G blocks of
// 256 threads, G = min(max(ceil(n/256), 1), max_blocks); thread g sums
// x_i y_i for i = g, g + 256G, ... with fma; each warp's values go through
// warp_tree, the 8 warp sums through another; then lane l of the last block
// adds the block partials l, l+32, ... in order and a final warp_tree.  In T
// throughout (float for the FP32 inner solves).
template <class T>
T tree_dot(int n, const T* x, const T* y, int max_blocks) {
  const int TH = 256;
  long long g = ((long long)n + TH - 1) / TH;
  if (g < 1) g = 1;
  if (g > max_blocks) g = max_blocks;
  const int G = (int)g;
  const long long stride = (long long)G * TH;
  std::vector<T> partial(G);
  T th[256], ws[32];
  for (int b = 0; b < G; ++b) {
    for (int t = 0; t < TH; ++t) {
      T acc = 0;
      for (long long i = (long long)b * TH + t; i < n; i += stride) acc = std::fma(x[i], y[i], acc);
      th[t] = acc;
    }
    for (int l = 0; l < 32; ++l) ws[l] = l < TH / 32 ? warp_tree(th + 32 * l) : T(0);
    partial[b] = warp_tree(ws);
  }
  T lanes[32];
  for (int l = 0; l < 32; ++l) {
    T s = 0;
    for (int b = l; b < G; b += 32) s = s + partial[b];
    lanes[l] = s;
  }
  return warp_tree(lanes);
}

thread_local int g_dot_mode = 0;
thread_local int g_tree_blocks = 1184;
thread_local bool g_cheb_saad = false;
thread_local bool g_cheb_lanczos = false;

// Row-block distribution in effect (orc_dist_solve): every dot is each rank's
// local dot over its rows, summed over the ranks left to right (CBLASMPIKernel
// dot + mpAllReduce; MPI leaves the order of that sum open, libab2 fixes this one).
thread_local const std::vector<int>* g_dist_off = nullptr;

template <class T>
T local_dot(int n, const T* x, const T* y) {
  return g_dot_mode == 1 ? tree_dot(n, x, y, g_tree_blocks) : dot(n, x, y);
}

template <class T>
T vdot(int n, const T* x, const T* y) {
  if (!g_dist_off) return local_dot(n, x, y);
  const std::vector<int>& off = *g_dist_off;
  T s = 0;
  for (size_t r = 0; r + 1 < off.size(); ++r) {
    const T p = local_dot(off[r + 1] - off[r], x + off[r], y + off[r]);
    s = r == 0 ? p : s + p;
  }
  return s;
}

// Stop test shared by CG (Iteration.h) and BiCGStab (its nested Iteration).
template <class T>
struct StopTest {
  int n;
  int max_iter;
  int iter = 0;
  T criteria;
  T nrm2_b;
  bool status = false;
  T last = 0;
  T* hist;
  int hist_cap;
  int hist_len = 0;

  // weight (the mixed solver's scaled Jacobi form): the stop test and b.b
  // become sum (v_i w_i) v_i, the residual's norm before the scaling.
  const T* weight = nullptr;
  std::vector<T> vw;

  StopTest(int n_, const T* b, T tol, int max_it, T* h, int cap, const T* w = nullptr)
      : n(n_), max_iter(max_it), hist(h), hist_cap(cap), weight(w) {
    nrm2_b = wdot(b);
    criteria = tol * tol * nrm2_b;
    status = (nrm2_b == 0);
  }
  T wdot(const T* v) {
    if (!weight) return vdot(n, v, v);
    vw.resize((size_t)n);
    for (int i = 0; i < n; ++i) vw[(size_t)i] = v[i] * weight[i];
    return vdot(n, vw.data(), v);
  }
  bool null_rhs() const { return nrm2_b == 0; }
  bool stop(const T* r) {
    if (iter >= max_iter) return true;
    last = wdot(r);
    if (hist && hist_len < hist_cap) hist[hist_len] = last;
    ++hist_len;
    status = last < criteria;
    return status;
  }
  void next() { ++iter; }
};

struct Breakdown {
  int which;
};

// ---------------------------------------------------------------- preconditioners
// Set up in FP64 from the FP64 matrix (as the reference does); applied in T:
// the FP32 form rounds the FP64 set-up's results, as libab2's pc_enable_f32.
template <class T>
struct Precond {
  virtual ~Precond() {}
  virtual void apply(const T* x, T* y) = 0;
};

template <class T>
struct Identity : Precond<T> {
  int n;
  explicit Identity(int n_) : n(n_) {}
  void apply(const T* x, T* y) override { copy(n, x, y); }
};

template <class T>
struct Diag : Precond<T> {
  int n;
  std::vector<T> inv;
  explicit Diag(const Csr& A) : n(A.n), inv(A.n, T(1)) {
    std::vector<int> d = diag_offsets(A);
    for (int i = 0; i < n; ++i) inv[i] = (T)(1.0 / A.v[d[i]]);
  }
  void apply(const T* x, T* y) override { pmult(n, inv.data(), x, y); }
};

// In-place IKJ ILU(0) (ILU0Preconditioner.h:156-178), in FP64.
void ilu0_factor_inplace(const Csr& A, const std::vector<int>& d, std::vector<double>& lu64) {
  const int n = A.n;
  const int* rp = A.rp;
  const int* ci = A.ci;
  std::vector<int> work(n, -1);
  for (int i = 1; i < n; ++i) {
    for (int k = rp[i]; k < d[i]; ++k) {
      const int kr = ci[k];
      const double aik = lu64[k] / lu64[d[kr]];
      lu64[k] = aik;
      for (int l = rp[kr]; l < rp[kr + 1]; ++l) work[ci[l]] = l;
      for (int j = k + 1; j < rp[i + 1]; ++j) {
        const int kj = work[ci[j]];
        if (kj != -1) lu64[j] = lu64[j] - aik * lu64[kj];
      }
      for (int l = rp[kr]; l < rp[kr + 1]; ++l) work[ci[l]] = -1;
    }
  }
}

// ILU(0) on a copy of the values, in FP64, then the forward/backward sweeps
// of solveL/solveU (ILU0Preconditioner.h:181-231) in T.
template <class T>
struct Ilu0 : Precond<T> {
  int n;
  const int* rp;
  const int* ci;
  std::vector<int> d;
  std::vector<double> lu64;
  std::vector<T> lu;
  std::vector<T> tmp;

  explicit Ilu0(const Csr& A) : n(A.n), rp(A.rp), ci(A.ci), lu64(A.v, A.v + A.rp[A.n]), tmp(A.n) {
    d = diag_offsets(A);
    ilu0_factor_inplace(A, d, lu64);
    lu.assign(lu64.begin(), lu64.end());
  }
  void solve_l(const T* y, T* x) const {
    for (int i = 0; i < n; ++i) {
      T v = y[i];
      for (int k = rp[i]; k < d[i]; ++k) v = v - lu[k] * x[ci[k]];
      x[i] = v;
    }
  }
  void solve_u(const T* y, T* x) const {
    for (int i = n - 1; i >= 0; --i) {
      const int dk = d[i];
      T v = y[i];
      for (int k = dk + 1; k < rp[i + 1]; ++k) v = v - lu[k] * x[ci[k]];
      x[i] = v / lu[dk];
    }
  }
  void apply(const T* y, T* x) override {
    solve_l(y, tmp.data());
    solve_u(tmp.data(), x);
  }
};

// FILU0 (FILU0Preconditioner.h, FLUFactorisationAlgo): the factor is the
// exact ILU(0) one (nb-factor-iter = 0, init :67-68) or factor_iter
// fixed-point sweeps (factorizeMultiIter :119-145, called on the factor
// matrix itself by init :72, so "matrix values" and the iterate are the same
// storage: each sweep starts from the previous iterate, not from A) updating
// every row i >= 1 against a copy v0 of the previous iterate
// (_factorizeRow :270-300: aik = v[k] / v0[pivot of row k]; v[j] -= aik v0[kj]).
// Application (solve :245-267), the device-algebra branch of solveL/solveU
// (:161-175, :218-226): m_x = x; solver_iter times m_x <- x - L m_x
// (copy, copy, addLMult(-1): SimpleCSRMatrixMultT.h:193-212 with alpha = -1);
// y = m_x; solver_iter times y <- (1/u_ii) (m_x - U y) (addUMult(-1),
// pointwiseMult).  Factor in FP64; the FP32 form rounds factor and 1/u_ii.
template <class T>
struct Filu0 : Precond<T> {
  int n;
  const int* rp;
  const int* ci;
  int S;
  std::vector<int> d;
  std::vector<double> lu64;
  std::vector<T> lu, inv, mx, xk;

  Filu0(const Csr& A, int factor_iter, int solver_iter)
      : n(A.n), rp(A.rp), ci(A.ci), S(solver_iter), lu64(A.v, A.v + A.rp[A.n]), mx(A.n), xk(A.n) {
    d = diag_offsets(A);
    if (factor_iter == 0) {
      ilu0_factor_inplace(A, d, lu64);
    } else {
      std::vector<double> prev(A.v, A.v + A.rp[A.n]);
      std::vector<int> work(n, -1);
      for (int it = 0; it < factor_iter; ++it) {
        std::vector<double> cur(prev);
        for (int i = 1; i < n; ++i) {
          for (int k = rp[i]; k < d[i]; ++k) {
            const int kr = ci[k];
            const double aik = cur[k] / prev[d[kr]];
            cur[k] = aik;
            for (int l = rp[kr]; l < rp[kr + 1]; ++l) work[ci[l]] = l;
            for (int j = k + 1; j < rp[i + 1]; ++j) {
              const int kj = work[ci[j]];
              if (kj != -1) cur[j] = cur[j] - aik * prev[kj];
            }
            for (int l = rp[kr]; l < rp[kr + 1]; ++l) work[ci[l]] = -1;
          }
        }
        prev.swap(cur);
      }
      lu64.swap(prev);
    }
    lu.assign(lu64.begin(), lu64.end());
    inv.resize(n);
    for (int i = 0; i < n; ++i) inv[i] = (T)(1.0 / lu64[d[i]]);
  }
  void apply(const T* x, T* y) override {
    if (S == 0) {
      copy(n, x, y);
      return;
    }
    copy(n, x, mx.data());
    for (int it = 0; it < S; ++it) {
      copy(n, mx.data(), xk.data());
      for (int i = 0; i < n; ++i) {
        T v = x[i];
        for (int k = rp[i]; k < d[i]; ++k) v = v + (T(-1) * lu[k]) * xk[ci[k]];
        mx[i] = v;
      }
    }
    copy(n, mx.data(), y);
    for (int it = 0; it < S; ++it) {
      copy(n, y, xk.data());
      for (int i = 0; i < n; ++i) {
        T v = mx[i];
        for (int k = d[i] + 1; k < rp[i + 1]; ++k) v = v + (T(-1) * lu[k]) * xk[ci[k]];
        y[i] = inv[i] * v;
      }
    }
  }
};

// Neumann polynomial (NeumannPolyPreconditioner.h): solve (:103-119)
// y = x; order times { t = A y; m = y; m = fma(-omega, t, m) (axpy);
// m = fma(1, x, m) (axpy); y = m }; y = omega y (scal).  omega = factor, or
// (factor = 0) computeFactor (:133-168): x random, y = A x, then
// max_iter times x = y, y = A x, est = |y| / |y_prev|; omega = 1/est.  The
// reference draws x from std::random_device; here (as libab2) from a
// default-seeded std::mt19937, U(-1,1) in index order.
template <class T>
struct Neumann : Precond<T> {
  CsrT<T> A;
  int n, order;
  double omega;
  std::vector<T> y, t, ay;

  Neumann(const Csr& A64, const T* vals, double factor, int order_, int max_iter)
      : A{A64.n, A64.rp, A64.ci, vals}, n(A64.n), order(order_), omega(factor), y(A64.n), t(A64.n), ay(A64.n) {
    if (omega != 0.0) return;
    std::vector<double> x(n), yy(n);
    std::mt19937 gen;
    std::uniform_real_distribution<> dis(-1., 1.);
    for (int i = 0; i < n; ++i) x[i] = dis(gen);
    spmv(A64, x.data(), yy.data());
    double nk = std::sqrt(vdot(n, yy.data(), yy.data()));
    double f = 0.0;
    for (int it = 0; it < max_iter; ++it) {
      copy(n, yy.data(), x.data());
      spmv(A64, x.data(), yy.data());
      const double nrm = std::sqrt(vdot(n, yy.data(), yy.data()));
      f = nrm / nk;
      nk = nrm;
    }
    omega = 1. / f;
  }
  void apply(const T* x, T* out) override {
    const T w = (T)omega;
    copy(n, x, y.data());
    for (int i = 0; i < order; ++i) {
      spmv(A, y.data(), ay.data());
      copy(n, y.data(), t.data());
      axpy(n, -w, ay.data(), t.data());
      axpy(n, T(1), x, t.data());
      copy(n, t.data(), y.data());
    }
    copy(n, y.data(), out);
    scal(n, w, out);
  }
};

// Chebyshev polynomial preconditioner, non-Saad branch (_algo2).
// Smallest and largest eigenvalue of the symmetric tridiagonal matrix with
// diagonal a[0..m) and off-diagonal b[0..m-1), by bisection on Sturm counts
// (128 halvings of the Gershgorin interval).
void tridiag_extremes(const std::vector<double>& a, const std::vector<double>& b, double* lmin, double* lmax) {
  const int m = (int)a.size();
  double lo = a[0], hi = a[0];
  for (int i = 0; i < m; ++i) {
    const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < m ? std::fabs(b[i]) : 0.0);
    lo = std::min(lo, a[i] - r);
    hi = std::max(hi, a[i] + r);
  }
  auto below = [&](double x) {  // eigenvalues < x
    int cnt = 0;
    double d = 1.0;
    for (int i = 0; i < m; ++i) {
      d = (a[i] - x) - (i > 0 ? b[i - 1] * b[i - 1] / d : 0.0);
      if (d == 0.0) d = -1e-300;
      cnt += d < 0.0;
    }
    return cnt;
  };
  auto kth = [&](int k) {  // smallest x with below(x) >= k
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
struct Cheb : Precond<T> {
  const Csr A64;     // bounds are estimated in FP64 on the FP64 matrix
  const CsrT<T> A;   // the matrix the application multiplies by
  int n;
  int order;
  bool saad;
  std::vector<double> inv64, y64;
  std::vector<T> inv, y_, r_, p_, z_, w_;
  double alpha = 0.0, beta = 0.0;
  // step coefficients, evaluated in FP64 in the reference's order
  std::vector<double> ca, cb;  // _algo2: alpha_i, beta_i ; _algo1: rho rho_old, 2 rho / delta
  double inv_theta = 0.0;      // _algo1: 1 / theta

  // saad: ChebyshevPreconditioner<AlgebraT, true> (_algo1, zero start, a
  // symmetric operator); otherwise the default _algo2.  lanczos: bounds from
  // `max_iter` Lanczos steps on D^-1/2 A D^-1/2 (this repo's addition)
  // instead of the reference's two power methods.  vT: the matrix values in T.
  Cheb(const Csr& A_, const T* vT, double factor, int order_, int max_iter, bool saad_ = false, bool lanczos = false)
      : A64(A_), A{A_.n, A_.rp, A_.ci, vT}, n(A_.n), order(order_), saad(saad_), inv64(A_.n, 1.0), y64(A_.n, 0.0),
        inv(A_.n, T(1)), y_(A_.n, T(0)), r_(A_.n, T(0)), p_(A_.n, T(0)), z_(A_.n, T(0)), w_(A_.n, T(0)) {
    std::vector<int> d = diag_offsets(A64);
    for (int i = 0; i < n; ++i) inv64[i] = 1.0 / A64.v[d[i]];
    for (int i = 0; i < n; ++i) inv[i] = (T)inv64[i];
    if (lanczos) {
      lanczos_bounds(max_iter);
    } else {
      beta = power_bound(max_iter, /*shift=*/false, 0.0);
      alpha = power_bound(max_iter, /*shift=*/true, beta);
    }
    if (factor != 0.0) alpha = beta / factor;
    coefficients();
  }

  void coefficients() {
    const int steps = std::max(1, order);
    ca.assign(steps, 0.0);
    cb.assign(steps, 0.0);
    if (saad) {  // ChebyshevPreconditioner.h:316-351
      const double delta = (beta - alpha) / 2;
      const double theta = (beta + alpha) / 2;
      const double sigma = theta / delta;
      double rho_old = 1. / sigma;
      inv_theta = 1 / theta;
      for (int k = 1; k < steps; ++k) {
        const double rho = 1. / (2 * sigma - rho_old);
        ca[k] = rho * rho_old;
        cb[k] = 2 * rho / delta;
        rho_old = rho;
      }
      return;
    }
    const double dd = (beta + alpha) / 2;  // :392-434
    const double c = (beta - alpha) / 2;
    double a = 2 / dd;
    ca[0] = a;
    for (int i = 1; i < steps; ++i) {
      const double bcoef = a * (c / 2.) * (c / 2.);
      a = 1. / (dd - bcoef);
      cb[i] = bcoef;
      ca[i] = a;
    }
  }

  // Lanczos on B = S A S, S = diag(sqrt(1/a_ii)), from the same mt19937 start
  // vector as the power methods; alpha = smallest Ritz value, beta = 1.1 x the
  // largest (Ritz values lie inside the spectrum; the margin keeps the
  // polynomial positive on all of it).
  void lanczos_bounds(int steps) {
    std::vector<double> s(n), v(n), vp(n, 0.0), t(n), w(n);
    for (int i = 0; i < n; ++i) s[i] = std::sqrt(inv64[i]);
    std::mt19937 gen;
    std::uniform_real_distribution<> dis(-1., 1.);
    for (int i = 0; i < n; ++i) v[i] = dis(gen);
    const double nrm = std::sqrt(vdot(n, v.data(), v.data()));
    scal(n, 1 / nrm, v.data());
    std::vector<double> a, b;
    double bprev = 0.0;
    for (int j = 0; j < std::max(steps, 1); ++j) {
      pmult(n, s.data(), v.data(), t.data());
      spmv(A64, t.data(), w.data());
      pmult(n, s.data(), w.data(), w.data());
      if (j > 0) axpy(n, -bprev, vp.data(), w.data());
      const double aj = vdot(n, w.data(), v.data());
      axpy(n, -aj, v.data(), w.data());
      const double bj = std::sqrt(vdot(n, w.data(), w.data()));
      a.push_back(aj);
      if (bj == 0.0 || j + 1 == std::max(steps, 1)) break;
      b.push_back(bj);
      copy(n, v.data(), vp.data());
      copy(n, w.data(), v.data());
      scal(n, 1 / bj, v.data());
      bprev = bj;
    }
    double lmin = 0.0, lmax = 0.0;
    tridiag_extremes(a, b, &lmin, &lmax);
    alpha = lmin;
    beta = 1.1 * lmax;
  }

  // computeBeta (:118-156) when shift is false, computeAlpha (:158-202) otherwise.
  // Both draw their start vector from a default-constructed std::mt19937 with
  // U(-1,1) in index order, which makes them deterministic.
  double power_bound(int max_iter, bool shift, double b) {
    std::vector<double> x(n);
    std::mt19937 gen;
    std::uniform_real_distribution<> dis(-1., 1.);
    for (int i = 0; i < n; ++i) x[i] = dis(gen);
    double nrm = std::sqrt(vdot(n, x.data(), x.data()));
    scal(n, 1 / nrm, x.data());
    double est = 0.0;
    for (int it = 0; it < max_iter; ++it) {
      spmv(A64, x.data(), y64.data());
      pmult(n, inv64.data(), y64.data(), y64.data());
      if (shift) axpy(n, -b, x.data(), y64.data());
      const double xax = vdot(n, y64.data(), x.data());
      const double xdx = vdot(n, x.data(), x.data());
      est = xax / xdx;
      const double nr = std::sqrt(vdot(n, y64.data(), y64.data()));
      scal(n, 1 / nr, y64.data());
      copy(n, y64.data(), x.data());
    }
    if (shift) est += b;
    return est;
  }

  // _algo2 (ChebyshevPreconditioner.h:392-434), the default.
  void apply_default(const T* x, T* y) {
    copy(n, x, y);
    spmv(A, y, y_.data());
    copy(n, x, r_.data());
    axpy(n, T(-1), y_.data(), r_.data());
    pmult(n, inv.data(), r_.data(), z_.data());
    copy(n, z_.data(), p_.data());
    axpy(n, (T)ca[0], p_.data(), y);
    for (int i = 1; i < order; ++i) {
      spmv(A, y, y_.data());
      copy(n, x, r_.data());
      axpy(n, T(-1), y_.data(), r_.data());
      pmult(n, inv.data(), r_.data(), z_.data());
      scal(n, (T)cb[i], p_.data());
      axpy(n, T(1), z_.data(), p_.data());
      axpy(n, (T)ca[i], p_.data(), y);
    }
  }

  void apply(const T* x, T* y) override {
    if (saad) apply_saad(x, y);
    else apply_default(x, y);
  }

  // _algo1 (ChebyshevPreconditioner.h:286-360): r = D^-1 x, w = r / theta,
  // y = w, then order-1 steps of the three-term recurrence.
  void apply_saad(const T* x, T* y) {
    pmult(n, inv.data(), x, r_.data());
    copy(n, r_.data(), w_.data());
    scal(n, (T)inv_theta, w_.data());
    copy(n, w_.data(), y);
    for (int k = 1; k < order; ++k) {
      spmv(A, w_.data(), y_.data());
      pmult(n, inv.data(), y_.data(), y_.data());
      axpy(n, T(-1), y_.data(), r_.data());
      scal(n, (T)ca[k], w_.data());
      axpy(n, (T)cb[k], r_.data(), w_.data());
      axpy(n, T(1), w_.data(), y);
    }
  }
};

// ---------------------------------------------------------------- row-block distribution
// One rank's rows in the layout of DistStructInfo::compute
// (kernels/simple_csr/DistStructInfo.cc:44-233) after sortGhostCols
// (SimpleCSRMatrix.h:215-258): in each row the local columns first (local id =
// global id - base), then the ghost columns (id n + g, ghosts numbered by
// owning rank, ascending global id inside each owner); lrs = local entries per
// row; interface rows = rows with a ghost entry.
struct DistLocal {
  int n = 0, base = 0, nghost = 0;
  std::vector<int> rp, ci, lrs, ghost_uids, iface;
  std::vector<double> v;
};

DistLocal dist_local(const Csr& A, const std::vector<int>& off, int r) {
  DistLocal L;
  L.base = off[r];
  L.n = off[r + 1] - off[r];
  const int np = (int)off.size() - 1;
  auto owner = [&](int c) {
    int q = 0;
    while (c >= off[q + 1]) ++q;
    return q;
  };
  std::vector<std::vector<int>> gids(np);
  L.rp.assign(1, 0);
  for (int i = 0; i < L.n; ++i) {
    const int g = L.base + i;
    int nl = 0;
    for (int k = A.rp[g]; k < A.rp[g + 1]; ++k)
      if (owner(A.ci[k]) == r) {
        L.ci.push_back(A.ci[k] - L.base);
        L.v.push_back(A.v[k]);
        ++nl;
      }
    for (int k = A.rp[g]; k < A.rp[g + 1]; ++k)
      if (owner(A.ci[k]) != r) {
        L.ci.push_back(-1 - A.ci[k]);  // global id, numbered below
        L.v.push_back(A.v[k]);
        gids[owner(A.ci[k])].push_back(A.ci[k]);
      }
    L.lrs.push_back(nl);
    L.rp.push_back((int)L.ci.size());
    if (L.rp[i + 1] - L.rp[i] > nl) L.iface.push_back(i);
  }
  for (auto& v : gids) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    L.ghost_uids.insert(L.ghost_uids.end(), v.begin(), v.end());
  }
  L.nghost = (int)L.ghost_uids.size();
  for (auto& c : L.ci)
    if (c < 0) c = L.n + (int)(std::lower_bound(L.ghost_uids.begin(), L.ghost_uids.end(), -1 - c) - L.ghost_uids.begin());
  return L;
}

struct DistCsr {
  int n = 0;  // global rows
  std::vector<int> off;
  std::vector<DistLocal> ranks;
  DistCsr(const Csr& A, const std::vector<int>& o) : n(A.n), off(o) {
    for (size_t r = 0; r + 1 < off.size(); ++r) ranks.push_back(dist_local(A, off, (int)r));
  }
};

// SimpleCSRMatrixMultT::_parallelMult (:85-128): each row's local entries
// summed (tmpy from 0, a*x rounded apart), then the interface rows add the sum
// of their ghost entries; ghost values are the owners' entries of x.
void spmv(const DistCsr& A, const double* x, double* y) {
  for (const DistLocal& L : A.ranks) {
    std::vector<double> xe(L.n + L.nghost);
    for (int i = 0; i < L.n; ++i) xe[i] = x[L.base + i];
    for (int g = 0; g < L.nghost; ++g) xe[L.n + g] = x[L.ghost_uids[g]];
    for (int i = 0; i < L.n; ++i) {
      double t = 0.;
      for (int k = L.rp[i]; k < L.rp[i] + L.lrs[i]; ++k) t += L.v[k] * xe[L.ci[k]];
      y[L.base + i] = t;
    }
    for (int i : L.iface) {
      double t = 0.;
      for (int k = L.rp[i] + L.lrs[i]; k < L.rp[i + 1]; ++k) t += L.v[k] * xe[L.ci[k]];
      y[L.base + i] += t;
    }
  }
}

// DistStructInfo::computeUpperDiagOffset: first local position not below the row.
std::vector<int> dist_dcol(const DistLocal& L) {
  std::vector<int> d(L.n);
  for (int i = 0; i < L.n; ++i) {
    int k = L.rp[i];
    while (k < L.rp[i] + L.lrs[i] && L.ci[k] < i) ++k;
    d[i] = k;
  }
  return d;
}

// The parallel block-Jacobi factorisation of ILU0Preconditioner.h:93-119,
// loop bounds as written there: row i is eliminated by row krow = col(k) only
// at positions j in (k, kcol[krow] + lrs[i]), with krow's local columns marked.
// With a single rank the matrix is not parallel (m_is_parallel = nproc > 1)
// and the sequential branch runs: rows eliminated up to their end (:156-178).
void bj_ilu0_factor(const DistLocal& L, const std::vector<int>& d, std::vector<double>& lu, bool parallel) {
  std::vector<int> work(L.n + L.nghost, -1);
  const int nnz = L.rp[L.n];
  for (int i = 1; i < L.n; ++i)
    for (int k = L.rp[i]; k < d[i]; ++k) {
      const int kr = L.ci[k];
      const double aik = lu[k] / (d[kr] < nnz ? lu[d[kr]] : 0.0);
      lu[k] = aik;
      for (int l = L.rp[kr]; l < L.rp[kr] + L.lrs[kr]; ++l) work[L.ci[l]] = l;
      const int bound = parallel ? L.rp[kr] + L.lrs[i] : L.rp[i + 1];
      for (int j = k + 1; j < bound; ++j) {
        const int kj = work[L.ci[j]];
        if (kj != -1) lu[j] = lu[j] - aik * lu[kj];
      }
      for (int l = L.rp[kr]; l < L.rp[kr] + L.lrs[kr]; ++l) work[L.ci[l]] = -1;
    }
}

// Block-Jacobi ILU(0): every rank factorises its rows (local columns only;
// one rank: the sequential ILU(0)) and sweeps them (solveL over local entries left of dcol, solveU over local
// entries right of it: ILU0Preconditioner.h:181-231, parallel branches).
struct BjIlu0 : Precond<double> {
  const DistCsr& A;
  std::vector<std::vector<int>> d;
  std::vector<std::vector<double>> lu;
  std::vector<double> t;
  explicit BjIlu0(const DistCsr& M) : A(M), t(M.n) {
    for (const DistLocal& L : A.ranks) {
      d.push_back(dist_dcol(L));
      lu.push_back(L.v);
      bj_ilu0_factor(L, d.back(), lu.back(), A.ranks.size() > 1);
    }
  }
  void apply(const double* y, double* x) override {
    for (size_t r = 0; r < A.ranks.size(); ++r) {
      const DistLocal& L = A.ranks[r];
      const std::vector<int>& dc = d[r];
      const std::vector<double>& f = lu[r];
      double* tt = t.data() + L.base;
      for (int i = 0; i < L.n; ++i) {
        double v = y[L.base + i];
        for (int k = L.rp[i]; k < dc[i]; ++k) v = v - f[k] * tt[L.ci[k]];
        tt[i] = v;
      }
      double* xx = x + L.base;
      for (int i = L.n - 1; i >= 0; --i) {
        double v = tt[i];
        for (int k = dc[i] + 1; k < L.rp[i] + L.lrs[i]; ++k) v = v - f[k] * xx[L.ci[k]];
        xx[i] = v / f[dc[i]];
      }
    }
  }
};

// ---------------------------------------------------------------- solvers
template <class T, class Mat>
void cg(const Mat& A, Precond<T>& M, StopTest<T>& it, const T* b, T* x) {
  if (it.null_rhs()) return;
  const int n = A.n;
  std::vector<T> p(n), z(n), q(n), r(n);
  T rho = 0, rho1 = 0, alpha = 0;
  copy(n, b, r.data());
  spmv(A, x, p.data());
  axpy(n, T(-1), p.data(), r.data());

  M.apply(r.data(), z.data());
  rho1 = vdot(n,r.data(), z.data());
  copy(n, z.data(), p.data());
  spmv(A, p.data(), q.data());
  alpha = vdot(n,p.data(), q.data());
  if (alpha == 0) {
    if (it.stop(r.data())) { it.next(); return; }
    throw Breakdown{ORC_BD_ALPHA};
  }
  alpha = rho1 / alpha;
  axpy(n, alpha, p.data(), x);
  axpy(n, -alpha, q.data(), r.data());
  rho = rho1;
  it.next();

  while (!it.stop(r.data())) {
    M.apply(r.data(), z.data());
    rho1 = vdot(n,r.data(), z.data());
    alpha = rho1 / rho;
    axpy(n, alpha, p.data(), z.data());
    copy(n, z.data(), p.data());
    spmv(A, p.data(), q.data());
    alpha = vdot(n,q.data(), p.data());
    if (alpha == 0) {
      if (it.stop(r.data())) { it.next(); return; }
      throw Breakdown{ORC_BD_ALPHA};
    }
    alpha = rho1 / alpha;
    axpy(n, alpha, p.data(), x);
    axpy(n, -alpha, q.data(), r.data());
    rho = rho1;
    it.next();
  }
}

template <class T, class Mat>
void bicgstab(const Mat& A, Precond<T>& M, StopTest<T>& it, const T* b, T* x) {
  if (it.null_rhs()) return;
  const int n = A.n;
  std::vector<T> p(n), phat(n), s(n), shat(n), t(n), v(n), r(n), r0(n);
  T rho = 0, rho1 = 0, alpha = 0, beta = 0, omega = 0;

  copy(n, b, r.data());
  spmv(A, x, r0.data());
  axpy(n, T(-1), r0.data(), r.data());
  copy(n, r.data(), r0.data());
  copy(n, r.data(), p.data());
  rho1 = vdot(n,r.data(), r0.data());

  M.apply(p.data(), phat.data());
  spmv(A, phat.data(), v.data());
  alpha = vdot(n,v.data(), r0.data());
  if (alpha == 0) throw Breakdown{ORC_BD_ALPHA};
  alpha = rho1 / alpha;
  copy(n, r.data(), s.data());
  axpy(n, -alpha, v.data(), s.data());

  if (it.stop(s.data())) {
    it.next();
    axpy(n, alpha, phat.data(), x);
    return;
  }

  M.apply(s.data(), shat.data());
  spmv(A, shat.data(), t.data());
  omega = vdot(n,t.data(), s.data());
  beta = vdot(n,t.data(), t.data());
  if (beta == 0) {
    if (it.stop(r.data())) {
      it.next();
      axpy(n, alpha, phat.data(), x);
      return;
    }
    throw Breakdown{ORC_BD_BETA};
  }
  omega = omega / beta;
  axpy(n, omega, shat.data(), x);
  axpy(n, alpha, phat.data(), x);
  copy(n, s.data(), r.data());
  axpy(n, -omega, t.data(), r.data());
  rho = rho1;
  it.next();

  while (!it.stop(r.data())) {
    rho1 = vdot(n,r.data(), r0.data());
    beta = (rho1 / rho) * (alpha / omega);
    axpy(n, -omega, v.data(), p.data());
    scal(n, beta, p.data());
    axpy(n, T(1), r.data(), p.data());
    if (rho == 0) throw Breakdown{ORC_BD_RHO};

    M.apply(p.data(), phat.data());
    spmv(A, phat.data(), v.data());
    alpha = vdot(n,v.data(), r0.data());
    if (alpha == 0) throw Breakdown{ORC_BD_ALPHA};
    alpha = rho1 / alpha;
    copy(n, r.data(), s.data());
    axpy(n, -alpha, v.data(), s.data());
    // Early exit on ||s|| without ++iter (BiCGStab.h:259-263).
    if (it.stop(s.data())) {
      axpy(n, alpha, phat.data(), x);
      return;
    }

    M.apply(s.data(), shat.data());
    spmv(A, shat.data(), t.data());
    omega = vdot(n,t.data(), s.data());
    beta = vdot(n,t.data(), t.data());
    if (beta == 0) {
      if (it.stop(s.data())) {
        axpy(n, alpha, phat.data(), x);
        return;
      }
      throw Breakdown{ORC_BD_BETA};
    }
    omega = omega / beta;
    axpy(n, omega, shat.data(), x);
    axpy(n, alpha, phat.data(), x);
    copy(n, s.data(), r.data());
    axpy(n, -omega, t.data(), r.data());
    rho = rho1;
    it.next();
  }
}

}  // namespace

extern "C" {

int orc_spmv(int n, const int* rp, const int* ci, const double* v, const double* x, double* y) {
  if (n < 0) return ORC_ERR_BAD_ARG;
  spmv(Csr{n, rp, ci, v}, x, y);
  return ORC_OK;
}

// y += alpha * (strict lower part of A) x   (SimpleCSRMatrixMultT.h:193-212)
int orc_add_lmult(int n, const int* rp, const int* ci, const double* v, double alpha, const double* x,
                  double* y) {
  Csr A{n, rp, ci, v};
  std::vector<int> d = diag_offsets(A);
  for (int i = 0; i < n; ++i) {
    double acc = y[i];
    for (int k = rp[i]; k < d[i]; ++k) acc = acc + alpha * v[k] * x[ci[k]];
    y[i] = acc;
  }
  return ORC_OK;
}

// y += alpha * (strict upper part of A) x   (SimpleCSRMatrixMultT.h:214-233)
int orc_add_umult(int n, const int* rp, const int* ci, const double* v, double alpha, const double* x,
                  double* y) {
  Csr A{n, rp, ci, v};
  std::vector<int> d = diag_offsets(A);
  for (int i = 0; i < n; ++i) {
    double acc = y[i];
    for (int k = d[i] + 1; k < rp[i + 1]; ++k) acc = acc + alpha * v[k] * x[ci[k]];
    y[i] = acc;
  }
  return ORC_OK;
}

int orc_diag_offsets(int n, const int* rp, const int* ci, int* dcol) {
  std::vector<int> d = diag_offsets(Csr{n, rp, ci, nullptr});
  std::copy(d.begin(), d.end(), dcol);
  return ORC_OK;
}

int orc_inv_diag(int n, const int* rp, const int* ci, const double* v, double* inv) {
  Csr A{n, rp, ci, v};
  std::vector<int> d = diag_offsets(A);
  for (int i = 0; i < n; ++i) inv[i] = 1. / v[d[i]];
  return ORC_OK;
}

double orc_dot(int n, const double* x, const double* y) { return dot(n, x, y); }

// The device's reduction tree (see tree_dot), for bit-exact checks of libab2.
double orc_dot_tree(int n, const double* x, const double* y, int max_blocks) { return tree_dot(n, x, y, max_blocks); }

// y += a x (cblas_daxpy, CBLASMPIKernel.h:48-53)
int orc_axpy(int n, double a, const double* x, double* y) {
  axpy(n, a, x, y);
  return ORC_OK;
}

// y = a y + x, one fma per element (the aypx the algebra interface names)
int orc_aypx(int n, double a, double* y, const double* x) {
  for (int i = 0; i < n; ++i) y[i] = std::fma(a, y[i], x[i]);
  return ORC_OK;
}

// ILU(0) factor values, written into lu (nnz entries).
int orc_ilu0_factor(int n, const int* rp, const int* ci, const double* v, double* lu) {
  Ilu0<double> f(Csr{n, rp, ci, v});
  std::copy(f.lu.begin(), f.lu.end(), lu);
  return ORC_OK;
}

int orc_ilu0_apply(int n, const int* rp, const int* ci, const double* v, const double* y, double* x) {
  Ilu0<double> f(Csr{n, rp, ci, v});
  f.apply(y, x);
  return ORC_OK;
}

// Dot summation order for the calls that take no options (Chebyshev set-up
// and application); orc_solve sets it from its options.
int orc_set_dot_mode(int mode, int tree_blocks) {
  g_dot_mode = mode;
  g_tree_blocks = tree_blocks > 0 ? tree_blocks : 1184;
  return ORC_OK;
}

// Chebyshev bounds (alpha = lambda_min estimate, beta = lambda_max estimate).
int orc_cheb_bounds(int n, const int* rp, const int* ci, const double* v, double factor, int max_iter,
                    double* alpha, double* beta) {
  Cheb<double> c(Csr{n, rp, ci, v}, v, factor, 1, max_iter, g_cheb_saad, g_cheb_lanczos);
  *alpha = c.alpha;
  *beta = c.beta;
  return ORC_OK;
}

int orc_cheb_apply(int n, const int* rp, const int* ci, const double* v, double factor, int order,
                   int max_iter, const double* x, double* y) {
  Cheb<double> c(Csr{n, rp, ci, v}, v, factor, order, max_iter, g_cheb_saad, g_cheb_lanczos);
  c.apply(x, y);
  return ORC_OK;
}

// Chebyshev variant for the two calls above (orc_solve takes it as options).
int orc_set_cheb_variant(int saad, int lanczos) {
  g_cheb_saad = saad != 0;
  g_cheb_lanczos = lanczos != 0;
  return ORC_OK;
}

// Full solve: x holds the initial guess on entry and the solution on exit.
// hist (optional, hist_cap entries) receives every value the stop test compares.
int orc_solve(int n, const int* rp, const int* ci, const double* v, const double* b, double* x,
              const orc_options* o, orc_result* res, double* hist, int hist_cap) {
  if (!o || !res || n < 0) return ORC_ERR_BAD_ARG;
  std::memset(res, 0, sizeof(*res));
  g_dot_mode = o->dot_mode;
  g_tree_blocks = o->tree_blocks > 0 ? o->tree_blocks : 1184;
  Csr A{n, rp, ci, v};
  Identity<double> pid(n);
  Diag<double>* pd = nullptr;
  Ilu0<double>* pi = nullptr;
  Cheb<double>* pc = nullptr;
  Precond<double>* pother = nullptr;
  Precond<double>* M = &pid;
  switch (o->precond) {
    case ORC_PC_NONE: break;
    case ORC_PC_DIAG: M = pd = new Diag<double>(A); break;
    case ORC_PC_ILU0: M = pi = new Ilu0<double>(A); break;
    case ORC_PC_CHEB:
      M = pc = new Cheb<double>(A, v, o->poly_factor, o->poly_order, o->poly_factor_max_iter, o->cheb_saad != 0,
                                o->cheb_lanczos != 0);
      res->cheb_alpha = pc->alpha;
      res->cheb_beta = pc->beta;
      break;
    case ORC_PC_FILU0: M = pother = new Filu0<double>(A, o->filu_factor_iter, o->filu_solver_iter); break;
    case ORC_PC_NEUMANN: {
      auto* pn = new Neumann<double>(A, v, o->poly_factor, o->poly_order, o->poly_factor_max_iter);
      M = pother = pn;
      res->cheb_alpha = pn->omega;  // the omega used, reported in the first bound's slot
      break;
    }
    default: return ORC_ERR_BAD_ARG;
  }
  StopTest<double> it(n, b, o->tol, o->max_iter, hist, hist_cap);
  int rc = ORC_OK;
  try {
    if (o->solver == ORC_SOLVER_CG) cg(A, *M, it, b, x);
    else if (o->solver == ORC_SOLVER_BICGSTAB) bicgstab(A, *M, it, b, x);
    else rc = ORC_ERR_BAD_ARG;
  } catch (const Breakdown& e) {
    rc = ORC_ERR_BREAKDOWN;
    res->breakdown = e.which;
  }
  res->iterations = it.iter;
  res->converged = it.status ? 1 : 0;
  res->error = rc;
  res->nrm2_b = it.nrm2_b;
  res->last_rr = it.last;
  res->history_len = it.hist_len;
  delete pd;
  delete pi;
  delete pc;
  delete pother;
  return rc;
}

// One FILU0 application (the device-algebra branch), FP64; lu (optional)
// receives the factor in CSR order.
int orc_filu0_apply(int n, const int* rp, const int* ci, const double* v, int factor_iter, int solver_iter,
                    const double* y, double* x, double* lu) {
  Filu0<double> M(Csr{n, rp, ci, v}, factor_iter, solver_iter);
  M.apply(y, x);
  if (lu) std::memcpy(lu, M.lu64.data(), sizeof(double) * (size_t)rp[n]);
  return ORC_OK;
}

// One Neumann application; omega (optional) receives the factor used.
int orc_neumann_apply(int n, const int* rp, const int* ci, const double* v, double factor, int order, int max_iter,
                      const double* x, double* y, double* omega) {
  Neumann<double> M(Csr{n, rp, ci, v}, v, factor, order, max_iter);
  M.apply(x, y);
  if (omega) *omega = M.omega;
  return ORC_OK;
}

// ---------------------------------------------------------------- FP32 pieces
// y = A32 x in float (the FP64 values rounded), products and sums rounded apart.
int orc_spmv32(int n, const int* rp, const int* ci, const float* v32, const float* x, float* y) {
  spmv(CsrT<float>{n, rp, ci, v32}, x, y);
  return ORC_OK;
}

// The device tree in float (FP32 dots of the mixed solver's inner solves).
float orc_dot_tree32(int n, const float* x, const float* y, int max_blocks) { return tree_dot(n, x, y, max_blocks); }

// ILU(0): the FP64 factor rounded to float, sweeps in float.
int orc_ilu0_apply32(int n, const int* rp, const int* ci, const double* v, const float* y, float* x) {
  Ilu0<float> f(Csr{n, rp, ci, v});
  f.apply(y, x);
  return ORC_OK;
}

// Chebyshev in float: bounds and coefficients in FP64 (dot order from
// orc_set_dot_mode), application in float on the FP32 values.
int orc_cheb_apply32(int n, const int* rp, const int* ci, const double* v, const float* v32, double factor, int order,
                     int max_iter, const float* x, float* y) {
  Cheb<float> c(Csr{n, rp, ci, v}, v32, factor, order, max_iter, g_cheb_saad, g_cheb_lanczos);
  c.apply(x, y);
  return ORC_OK;
}

// One refinement step at a time, as libab2's ab2_mixed_solve: r = b - A x and
// ||r|| in FP64; stop below tol; inner FP32 solve of A32 d = float(r/||r||)
// from d = 0; x += ||r|| d.  Stops without success after max_outer steps or
// when a step does not reduce the true residual.
int orc_mixed_solve(int n, const int* rp, const int* ci, const double* v, const double* b, double* x,
                    const orc_mixed_options* o, orc_mixed_result* res, double* hist, int hist_cap) {
  if (!o || !res || n < 0) return ORC_ERR_BAD_ARG;
  std::memset(res, 0, sizeof(*res));
  g_dot_mode = o->dot_mode;
  g_tree_blocks = o->tree_blocks > 0 ? o->tree_blocks : 1184;
  const Csr A{n, rp, ci, v};
  std::vector<float> v32(v, v + (n > 0 ? rp[n] : 0));
  const CsrT<float> A32{n, rp, ci, v32.data()};
  Identity<float> pid(n);
  Diag<float>* pd = nullptr;
  Ilu0<float>* pi = nullptr;
  Cheb<float>* pc = nullptr;
  Precond<float>* pother = nullptr;
  Precond<float>* M = &pid;
  switch (o->precond) {
    case ORC_PC_NONE: break;
    case ORC_PC_DIAG: M = pd = new Diag<float>(A); break;
    case ORC_PC_ILU0: M = pi = new Ilu0<float>(A); break;
    case ORC_PC_CHEB:
      M = pc = new Cheb<float>(A, v32.data(), o->poly_factor, o->poly_order, o->poly_factor_max_iter,
                               o->cheb_saad != 0, o->cheb_lanczos != 0);
      break;
    case ORC_PC_FILU0: M = pother = new Filu0<float>(A, o->filu_factor_iter, o->filu_solver_iter); break;
    case ORC_PC_NEUMANN:
      M = pother = new Neumann<float>(A, v32.data(), o->poly_factor, o->poly_order, o->poly_factor_max_iter);
      break;
    default: return ORC_ERR_BAD_ARG;
  }
  // The scaled Jacobi form: plain CG on S A S, S = diag(1/sqrt(a_ii)), unit
  // diagonal, each off-diagonal value (a_rc s_r) s_c rounded once from the
  // upper triangle's entry (the lower one mirrors it), as mixed.cu builds it;
  // its stop test weighs r^2 by float(a_ii), the unscaled residual's norm.
  const bool scaled = o->jacobi_scaled && o->solver == ORC_SOLVER_CG && o->precond == ORC_PC_DIAG;
  std::vector<double> sc;
  std::vector<float> vhat;
  std::vector<float> w32;  // the stop test's weight: float(a_ii)
  CsrT<float> Ahat{n, rp, ci, nullptr};
  if (scaled) {
    sc.assign(n, 0.0);
    w32.assign(n, 0.0f);
    for (int r = 0; r < n; ++r)
      for (int k = rp[r]; k < rp[r + 1]; ++k)
        if (ci[k] == r) {
          sc[r] = 1.0 / std::sqrt(v[k]);
          w32[r] = (float)v[k];
        }
    auto entry = [&](int row, int col) {
      for (int k = rp[row]; k < rp[row + 1]; ++k)
        if (ci[k] == col) return v[k];
      return 0.0;
    };
    vhat.assign(v32.size(), 0.0f);
    for (int r = 0; r < n; ++r)
      for (int k = rp[r]; k < rp[r + 1]; ++k) {
        const int c = ci[k];
        vhat[k] = c == r ? 1.0f : c > r ? (float)((v[k] * sc[r]) * sc[c]) : (float)((entry(c, r) * sc[c]) * sc[r]);
      }
    Ahat.v = vhat.data();
    M = &pid;
  }
  const CsrT<float>& Ain = scaled ? Ahat : A32;
  std::vector<double> r(n), ax(n);
  std::vector<float> r32(n), d32(n);
  const double bb = vdot(n, b, b);
  int outer = 0, inner = 0, rc = ORC_OK;
  bool ok = false;
  double resid = 0.0;
  auto push = [&](double val) {
    if (hist && res->history_len < hist_cap) hist[res->history_len] = val;
    res->history_len += 1;
  };
  if (bb == 0.0) {
    ok = true;
  } else {
    const double nb = std::sqrt(bb);
    double prev = INFINITY;
    for (;;) {
      spmv(A, x, ax.data());
      for (int i = 0; i < n; ++i) r[i] = b[i] - ax[i];
      const double rr = vdot(n, r.data(), r.data());
      resid = std::sqrt(rr) / nb;
      push(resid);
      if (resid < o->tol) {
        ok = true;
        break;
      }
      if (outer >= o->max_outer || !(resid < prev) || rr == 0.0) {
        rc = ORC_ERR_NOT_CONVERGED;
        break;
      }
      prev = resid;
      const double scn = 1.0 / std::sqrt(rr);
      for (int i = 0; i < n; ++i) r32[i] = scaled ? (float)((r[i] * scn) * sc[i]) : (float)(r[i] * scn);
      std::fill(d32.begin(), d32.end(), 0.0f);
      StopTest<float> it(n, r32.data(), (float)o->inner_tol, o->inner_max_iter, nullptr, 0,
                         scaled ? w32.data() : nullptr);
      try {
        if (o->solver == ORC_SOLVER_CG) cg(Ain, *M, it, r32.data(), d32.data());
        else bicgstab(Ain, *M, it, r32.data(), d32.data());
      } catch (const Breakdown&) {
        if (it.iter == 0) {
          inner += it.iter;
          rc = ORC_ERR_BREAKDOWN;
          break;
        }
      }
      inner += it.iter;
      const double s = std::sqrt(rr);
      for (int i = 0; i < n; ++i) x[i] = std::fma(s, scaled ? (double)d32[i] * sc[i] : (double)d32[i], x[i]);
      ++outer;
    }
  }
  res->succeeded = ok ? 1 : 0;
  res->outer_iterations = outer;
  res->inner_iterations = inner;
  res->error = ok ? ORC_OK : rc;
  res->true_residual = resid;
  delete pd;
  delete pi;
  delete pc;
  delete pother;
  return ORC_OK;
}

// ---------------------------------------------------------------- batched systems
// libab2's ab2_batch restated (batch.cu, no reference counterpart): per system,
// FP32 Jacobi-PCG (CG.h's loop) inside FP64 refinement, every dot reduced the
// way one thread-block cluster does it -- CTA c of `csize` owns rows
// [lo_c, hi_c) (a contiguous 1/csize share), thread t of `threads` sums rows
// lo_c + t, lo_c + t + threads, ... with fma, warps and then warp 0 reduce with
// the shuffle tree, and the csize CTA partials are added in rank order.
}  // extern "C"

namespace {

template <class T, int NC, class RowFn>
void cluster_reduce(int s0, int s1, int csize, int threads, RowFn fn, T (&out)[NC]) {
  const int chunk = (s1 - s0 + csize - 1) / csize;
  const int nw = (threads + 31) / 32;
  T total[NC];
  for (int c = 0; c < NC; ++c) total[c] = T(0);
  std::vector<T> acc((size_t)threads * NC);
  for (int cta = 0; cta < csize; ++cta) {
    const int lo = std::min(s1, s0 + cta * chunk), hi = std::min(s1, lo + chunk);
    std::fill(acc.begin(), acc.end(), T(0));
    for (int t = 0; t < threads; ++t)
      for (int i = lo + t; i < hi; i += threads) fn(i, &acc[(size_t)t * NC]);
    for (int c = 0; c < NC; ++c) {
      T ws[32];
      for (int w = 0; w < 32; ++w) {
        if (w < nw) {
          T lanes[32];
          for (int l = 0; l < 32; ++l) lanes[l] = w * 32 + l < threads ? acc[(size_t)(w * 32 + l) * NC + c] : T(0);
          ws[w] = warp_tree(lanes);
        } else {
          ws[w] = T(0);
        }
      }
      total[c] = total[c] + warp_tree(ws);
    }
  }
  for (int c = 0; c < NC; ++c) out[c] = total[c];
}

}  // namespace

extern "C" {

int orc_batch_solve(int n, const int* rp, const int* ci, const double* v, int nsys, const int* off, const double* b,
                    double* x, double tol, int max_outer, double inner_tol, int inner_max_iter, int csize, int threads,
                    int lanes_per_row, int* conv_out, int* outer_out, int* inner_out, double* res_out) {
  if (n < 0 || nsys < 0 || csize < 1 || threads < 32) return ORC_ERR_BAD_ARG;
  const int lpr = lanes_per_row > 1 ? lanes_per_row : 1;
  if (lpr > 32 || (lpr & (lpr - 1)) != 0) return ORC_ERR_BAD_ARG;
  const Csr A{n, rp, ci, v};
  std::vector<float> v32(v, v + (n > 0 ? rp[n] : 0));
  std::vector<int> d = diag_offsets(A);
  std::vector<float> inv32(n);
  for (int i = 0; i < n; ++i) inv32[i] = (float)(1.0 / v[d[i]]);
  std::vector<double> r64(n);
  std::vector<float> r(n), z(n), p(n), q(n), dd(n);
  auto row64 = [&](int i) {  // row i of A x, product and sum rounded apart
    double acc = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) acc = acc + v[k] * x[ci[k]];
    return acc;
  };
  // FP32 row sum: in column order, or (lpr > 1, batch.cu's CsrGroupView)
  // lane g of lpr summing entries g, g + lpr, ... in order, then the xor
  // butterfly over the lanes (offsets lpr/2 .. 1); lane 0's value.
  auto row32 = [&](int i, const float* y) {
    if (lpr == 1) {
      float acc = 0.f;
      for (int k = rp[i]; k < rp[i + 1]; ++k) acc = acc + v32[k] * y[ci[k]];
      return acc;
    }
    float part[32], nxt[32];
    for (int g = 0; g < lpr; ++g) {
      float acc = 0.f;
      for (int k = rp[i] + g; k < rp[i + 1]; k += lpr) acc = acc + v32[k] * y[ci[k]];
      part[g] = acc;
    }
    for (int o = lpr / 2; o > 0; o >>= 1) {
      for (int g = 0; g < lpr; ++g) nxt[g] = part[g] + part[g ^ o];
      for (int g = 0; g < lpr; ++g) part[g] = nxt[g];
    }
    return part[0];
  };
  const float itol = (float)inner_tol;
  for (int s = 0; s < nsys; ++s) {
    const int s0 = off[s], s1 = off[s + 1];
    double bb[1];
    cluster_reduce<double, 1>(s0, s1, csize, threads, [&](int i, double* a) { a[0] = std::fma(b[i], b[i], a[0]); }, bb);
    int outer = 0, inner = 0, converged = bb[0] == 0.0 ? 1 : 0;
    double res = 0.0, prev = INFINITY;
    while (!converged) {
      double rr[1];
      cluster_reduce<double, 1>(s0, s1, csize, threads, [&](int i, double* a) {
        const double rv = b[i] - row64(i);
        r64[i] = rv;
        a[0] = std::fma(rv, rv, a[0]);
      }, rr);
      res = std::sqrt(rr[0]) / std::sqrt(bb[0]);
      if (res < tol) {
        converged = 1;
        break;
      }
      if (outer >= max_outer || !(res < prev) || rr[0] == 0.0) break;
      prev = res;
      const double scale = 1.0 / std::sqrt(rr[0]);
      float acc[2];
      cluster_reduce<float, 2>(s0, s1, csize, threads, [&](int i, float* a) {
        const float rv = (float)(r64[i] * scale);
        const float zv = inv32[i] * rv;
        r[i] = rv;
        z[i] = zv;
        p[i] = zv;
        dd[i] = 0.f;
        a[0] = std::fma(rv, zv, a[0]);
        a[1] = std::fma(rv, rv, a[1]);
      }, acc);
      const float crit = itol * itol * acc[1];
      float rho = acc[0];
      int it = 0;
      for (;;) {
        float pq[1];
        cluster_reduce<float, 1>(s0, s1, csize, threads, [&](int i, float* a) {
          const float qv = row32(i, p.data());
          q[i] = qv;
          a[0] = std::fma(p[i], qv, a[0]);
        }, pq);
        if (pq[0] == 0.f) break;
        const float alpha = rho / pq[0];
        float rz[2];
        cluster_reduce<float, 2>(s0, s1, csize, threads, [&](int i, float* a) {
          dd[i] = std::fma(alpha, p[i], dd[i]);
          const float rv = std::fma(-alpha, q[i], r[i]);
          r[i] = rv;
          const float zv = inv32[i] * rv;
          z[i] = zv;
          a[0] = std::fma(rv, zv, a[0]);
          a[1] = std::fma(rv, rv, a[1]);
        }, rz);
        ++it;
        if (rz[1] < crit || it >= inner_max_iter) break;
        const float beta = rz[0] / rho;
        rho = rz[0];
        for (int i = s0; i < s1; ++i) p[i] = std::fma(beta, p[i], z[i]);
      }
      inner += it;
      const double sr = std::sqrt(rr[0]);
      for (int i = s0; i < s1; ++i) x[i] = std::fma(sr, (double)dd[i], x[i]);
      ++outer;
    }
    if (conv_out) conv_out[s] = converged;
    if (outer_out) outer_out[s] = outer;
    if (inner_out) inner_out[s] = inner;
    if (res_out) res_out[s] = res;
  }
  return ORC_OK;
}

// BEllPack layout with slice S (SYCLBEllPackMatrix.cc:70-88 computes the slice
// widths; the value at (slice s, slot j, lane l) lives at off[s]*S + j*S + l,
// padding uses column 0 and value 0).
int orc_ell_layout(int n, const int* rp, const int* ci, const double* v, int S, int* slice_off,
                   int* ell_cols, double* ell_vals) {
  const int ns = (n + S - 1) / S;
  int off = 0;
  for (int s = 0; s < ns; ++s) {
    slice_off[s] = off;
    int w = 0;
    for (int l = 0; l < S && s * S + l < n; ++l) w = std::max(w, rp[s * S + l + 1] - rp[s * S + l]);
    off += w;
  }
  slice_off[ns] = off;
  if (!ell_cols) return ORC_OK;
  for (int s = 0; s < ns; ++s) {
    const int w = slice_off[s + 1] - slice_off[s];
    for (int l = 0; l < S; ++l) {
      const int row = s * S + l;
      const int len = row < n ? rp[row + 1] - rp[row] : 0;
      for (int j = 0; j < w; ++j) {
        const size_t at = (size_t)slice_off[s] * S + (size_t)j * S + l;
        ell_cols[at] = j < len ? ci[rp[row] + j] : 0;
        ell_vals[at] = j < len ? v[rp[row] + j] : 0.0;
      }
    }
  }
  return ORC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- row-block distribution (C)
extern "C" {

// One rank's layout: sizes[0..3] = local rows, ghosts, interface rows, entries;
// the arrays (any may be null) as ab2_dist_matrix_layout fills them.
int orc_dist_layout(int n, const int* rp, const int* ci, const double* v, int nranks, const int* offsets, int rank,
                    int* sizes, int* out_rp, int* out_ci, double* out_v, int* lrs, int* ghost_uids, int* iface) {
  if (nranks < 1 || rank < 0 || rank >= nranks || offsets[0] != 0 || offsets[nranks] != n) return ORC_ERR_BAD_ARG;
  const std::vector<int> off(offsets, offsets + nranks + 1);
  const DistLocal L = dist_local(Csr{n, rp, ci, v}, off, rank);
  if (sizes) {
    sizes[0] = L.n;
    sizes[1] = L.nghost;
    sizes[2] = (int)L.iface.size();
    sizes[3] = L.rp[L.n];
  }
  if (out_rp) std::copy(L.rp.begin(), L.rp.end(), out_rp);
  if (out_ci) std::copy(L.ci.begin(), L.ci.end(), out_ci);
  if (out_v) std::copy(L.v.begin(), L.v.end(), out_v);
  if (lrs) std::copy(L.lrs.begin(), L.lrs.end(), lrs);
  if (ghost_uids) std::copy(L.ghost_uids.begin(), L.ghost_uids.end(), ghost_uids);
  if (iface) std::copy(L.iface.begin(), L.iface.end(), iface);
  return ORC_OK;
}

// y = A x with A distributed by offsets (each rank's _parallelMult).
int orc_dist_spmv(int n, const int* rp, const int* ci, const double* v, int nranks, const int* offsets, const double* x,
                  double* y) {
  if (nranks < 1 || offsets[0] != 0 || offsets[nranks] != n) return ORC_ERR_BAD_ARG;
  spmv(DistCsr(Csr{n, rp, ci, v}, std::vector<int>(offsets, offsets + nranks + 1)), x, y);
  return ORC_OK;
}

// Sum over ranks of the local dots (dot_mode / tree_blocks as orc_options).
double orc_dist_dot(int nranks, const int* offsets, const double* x, const double* y, int dot_mode, int tree_blocks) {
  const std::vector<int> off(offsets, offsets + nranks + 1);
  g_dot_mode = dot_mode;
  g_tree_blocks = tree_blocks > 0 ? tree_blocks : 1184;
  g_dist_off = &off;
  const double s = vdot(offsets[nranks], x, y);
  g_dist_off = nullptr;
  return s;
}

// Block-Jacobi ILU(0): x = M^-1 y over all ranks; lu (optional) receives each
// rank's factor on its local entries, rank after rank, in the diagonal
// block's CSR order (what ab2_precond_ilu0_values returns on that rank).
int orc_bj_ilu0_apply(int n, const int* rp, const int* ci, const double* v, int nranks, const int* offsets,
                      const double* y, double* x, double* lu) {
  if (nranks < 1 || offsets[0] != 0 || offsets[nranks] != n) return ORC_ERR_BAD_ARG;
  const DistCsr A(Csr{n, rp, ci, v}, std::vector<int>(offsets, offsets + nranks + 1));
  BjIlu0 M(A);
  M.apply(y, x);
  if (lu) {
    size_t o = 0;
    for (size_t r = 0; r < A.ranks.size(); ++r) {
      const DistLocal& L = A.ranks[r];
      for (int i = 0; i < L.n; ++i)
        for (int p = 0; p < L.lrs[i]; ++p) lu[o++] = M.lu[r][L.rp[i] + p];
    }
  }
  return ORC_OK;
}

// The solve every rank runs on the distributed algebra: CG or BiCGStab with
// NONE, DIAG or ILU0 (block Jacobi).  Same conventions as orc_solve.
int orc_dist_solve(int n, const int* rp, const int* ci, const double* v, int nranks, const int* offsets, const double* b,
                   double* x, const orc_options* o, orc_result* res, double* hist, int hist_cap) {
  if (!o || !res || nranks < 1 || offsets[0] != 0 || offsets[nranks] != n) return ORC_ERR_BAD_ARG;
  std::memset(res, 0, sizeof(*res));
  g_dot_mode = o->dot_mode;
  g_tree_blocks = o->tree_blocks > 0 ? o->tree_blocks : 1184;
  const std::vector<int> off(offsets, offsets + nranks + 1);
  const Csr G{n, rp, ci, v};
  const DistCsr A(G, off);
  Identity<double> pid(n);
  Precond<double>* M = &pid;
  Diag<double>* pd = nullptr;
  BjIlu0* pb = nullptr;
  switch (o->precond) {
    case ORC_PC_NONE: break;
    case ORC_PC_DIAG: M = pd = new Diag<double>(G); break;
    case ORC_PC_ILU0: M = pb = new BjIlu0(A); break;
    default: return ORC_ERR_BAD_ARG;
  }
  g_dist_off = &off;
  int rc = ORC_OK;
  StopTest<double> it(n, b, o->tol, o->max_iter, hist, hist_cap);
  try {
    if (o->solver == ORC_SOLVER_CG) cg(A, *M, it, b, x);
    else if (o->solver == ORC_SOLVER_BICGSTAB) bicgstab(A, *M, it, b, x);
    else rc = ORC_ERR_BAD_ARG;
  } catch (const Breakdown& e) {
    rc = ORC_ERR_BREAKDOWN;
    res->breakdown = e.which;
  }
  g_dist_off = nullptr;
  res->iterations = it.iter;
  res->converged = it.status ? 1 : 0;
  res->error = rc;
  res->nrm2_b = it.nrm2_b;
  res->last_rr = it.last;
  res->history_len = it.hist_len;
  delete pd;
  delete pb;
  return rc;
}

}  // extern "C"
