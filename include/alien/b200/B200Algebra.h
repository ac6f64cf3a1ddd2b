// B200Algebra.h -- Alien's AlgebraT concept on libab2 (header-only C++17).
//
// The drop-in point for Alien's Krylov layer: the header-only templates
// (expression/krylov/Iteration.h, CG.h, BiCGStab.h, DiagPreconditioner.h,
// ChebyshevPreconditioner.h) are written against an "AlgebraT" with the
// method set of SimpleCSRInternalLinearAlgebra
// (kernels/simple_csr/algebra/SimpleCSRInternalLinearAlgebra.h:55-173) and its
// SYCL peer (kernels/sycl/algebra/SYCLInternalLinearAlgebra.h:46-141).
// Alien::B200::Algebra provides that method set over the C ABI of
// include/ab2.h, so those templates run unmodified with every vector
// operation, SpMV and dot product on the GPU:
//
//   Alien::B200::Algebra algebra(ctx);
//   Alien::CG<Alien::B200::Algebra> solver(algebra, trace_mng);
//   Alien::DiagPreconditioner<Alien::B200::Algebra> diag(algebra, A);
//   diag.init();
//   Alien::Iteration<Alien::B200::Algebra> it(algebra, b, tol, max_iter, trace_mng);
//   solver.solve(diag, it, A, b, x);
//
// ILU(0): the reference's ILU0Preconditioner.h factorises and sweeps on host
// arrays (LUFactorisationAlgo, :71-248), so the GPU form is
// Alien::B200::ILU0Preconditioner below (same interface, same factor and
// sweeps bit for bit, run by ab2_precond_*).  The fused device-resident
// solvers (ab2_solver_*, ab2_mixed_*) are wrapped by Alien::B200::Solver.
//
// Errors from the C ABI become Alien::B200::Error (a std::runtime_error with
// the code and ab2_last_error_message); breakdowns inside the templates throw
// Algebra::NullValueException as the reference's algebras do.
#pragma once

#include <ab2.h>

#include <cmath>
#include <cstddef>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace Alien {
namespace B200 {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what) : std::runtime_error(what), m_code(code) {}
  int code() const { return m_code; }

 private:
  int m_code;
};

// One GPU, one CUDA stream (ab2_context); shared by everything created on it.
class Context {
 public:
  Context() = default;  // empty; a usable context comes from Context(device)
  explicit Context(int device) {
    ab2_context* h = nullptr;
    const int rc = ab2_context_create(device, &h);
    if (rc != AB2_OK) throw Error(rc, "ab2_context_create failed");
    m_h = std::shared_ptr<ab2_context>(h, [](ab2_context* c) { ab2_context_destroy(c); });
  }
  ab2_context* handle() const { return m_h.get(); }
  void check(int rc, const char* what) const {
    if (rc != AB2_OK) throw Error(rc, std::string(what) + ": " + ab2_last_error_message(m_h.get()));
  }
  void synchronize() const { check(ab2_synchronize(m_h.get()), "ab2_synchronize"); }

  // Phase timers, the reference's StdTimer under ALIEN_USE_PERF_TIMER
  // (utils/StdTimer.h): device seconds per operation ("CSR-SPMV", "CSR-DOT",
  // ...) since timing was turned on.
  void setPhaseTiming(bool on) const { check(ab2_context_set_phase_timing(m_h.get(), on ? 1 : 0), "set_phase_timing"); }
  std::vector<std::pair<std::string, double>> phaseTimes() const {
    int n = 0;
    check(ab2_context_phase_times(m_h.get(), nullptr, 0, &n), "phase_times");
    std::vector<ab2_phase_time> t((std::size_t)n);
    if (n) check(ab2_context_phase_times(m_h.get(), t.data(), n, &n), "phase_times");
    std::vector<std::pair<std::string, double>> out;
    for (auto const& e : t) out.emplace_back(e.name, e.ms * 1e-3);
    return out;
  }
  // StdTimer::printInfo's layout: phase:seconds between rules.
  void printInfo(std::ostream& os, const std::string& msg) const {
    os << "================================\n" << "PERF INFO : " << msg << "\n";
    for (auto const& p : phaseTimes()) os << p.first << ":" << p.second << "\n";
    os << "================================" << std::endl;
  }

 private:
  std::shared_ptr<ab2_context> m_h;
};

// CSR matrix on the device (plus sliced ELL, and FP32 values on request).
// The host arrays are copied; the caller keeps them.
class Matrix {
 public:
  typedef double ValueType;

  Matrix() = default;
  Matrix(const Context& ctx, int n, const int* row_ptr, const int* cols, const double* vals,
         int formats = AB2_FMT_CSR | AB2_FMT_ELL)
      : m_ctx(ctx), m_n(n) {
    ab2_matrix* h = nullptr;
    ctx.check(ab2_matrix_create_csr(ctx.handle(), n, row_ptr, cols, vals, formats, &h), "ab2_matrix_create_csr");
    m_h = std::shared_ptr<ab2_matrix>(h, [](ab2_matrix* m) { ab2_matrix_destroy(m); });
  }
  // Same profile, new values (Alien's notifyChanges / endUpdate path).
  void updateValues(const double* vals) {
    m_ctx.check(ab2_matrix_update_values(m_ctx.handle(), m_h.get(), vals), "ab2_matrix_update_values");
  }
  int rows() const { return m_n; }
  ab2_matrix* handle() const { return m_h.get(); }
  const Context& context() const { return m_ctx; }

 private:
  Context m_ctx;
  std::shared_ptr<ab2_matrix> m_h;
  int m_n = 0;
};

// Device vector of doubles.  Default-constructible (the templates declare
// vectors first and allocate them from a matrix's resource afterwards);
// copies share the device array.
class Vector {
 public:
  Vector() = default;
  Vector(const Context& ctx, int n) { allocate(ctx, n); }
  void allocate(const Context& ctx, int n) {
    ab2_vector* h = nullptr;
    ctx.check(ab2_vector_create(ctx.handle(), n, &h), "ab2_vector_create");
    m_h = std::shared_ptr<ab2_vector>(h, [](ab2_vector* v) { ab2_vector_destroy(v); });
    m_ctx = ctx.handle();
    m_n = n;
  }
  void release() {
    m_h.reset();
    m_n = 0;
  }
  // Takes ownership of a vector made elsewhere in the C ABI (e.g. a
  // distributed vector with room for ghost values).
  void adopt(const Context& ctx, ab2_vector* h, int n) {
    m_h = std::shared_ptr<ab2_vector>(h, [](ab2_vector* v) { ab2_vector_destroy(v); });
    m_ctx = ctx.handle();
    m_n = n;
  }
  void upload(const double* host) { check(ab2_vector_upload(m_ctx, m_h.get(), host), "ab2_vector_upload"); }
  void download(double* host) const { check(ab2_vector_download(m_ctx, m_h.get(), host), "ab2_vector_download"); }
  std::vector<double> download() const {
    std::vector<double> out((std::size_t)m_n);
    if (m_n) download(out.data());
    return out;
  }
  int size() const { return m_n; }
  ab2_vector* handle() const { return m_h.get(); }

 private:
  void check(int rc, const char* what) const {
    if (rc != AB2_OK) throw Error(rc, std::string(what) + ": " + ab2_last_error_message(m_ctx));
  }
  std::shared_ptr<ab2_vector> m_h;
  ab2_context* m_ctx = nullptr;
  int m_n = 0;
};

class Algebra {
 public:
  typedef B200::Matrix Matrix;
  typedef B200::Vector Vector;
  typedef double ValueType;

  // AlgebraT::resource(A): what allocate() needs to size vectors like A's rows.
  struct ResourceType {
    Context ctx;
    int n;
  };

  // Thrown by the templates on a zero pivot scalar ("alpha", "beta", "rho").
  struct NullValueException {
    std::string which;
    explicit NullValueException(std::string const& w) : which(w) {}
  };

  // The asynchronous form of dot (SimpleCSRInternalLinearAlgebra.h:74-98):
  // dot(x, y, f) queues x.y into a device scalar; get() waits for it and
  // stores it in the value the future was built on.
  template <typename T>
  class Future {
   public:
    explicit Future(T& value) : m_value(value) {}
    T& operator()() { return m_value; }
    T get() {
      if (m_pending) {
        double v = 0.0;
        const int rc = ab2_scalar_get(m_ctx, m_slot.get(), &v);
        if (rc != AB2_OK) throw Error(rc, std::string("ab2_scalar_get: ") + ab2_last_error_message(m_ctx));
        m_value = (T)v;
        m_pending = false;
      }
      return m_value;
    }

   private:
    friend class Algebra;
    void arm(ab2_context* ctx) {
      if (!m_slot || m_ctx != ctx) {
        ab2_scalar* s = nullptr;
        const int rc = ab2_scalar_create(ctx, &s);
        if (rc != AB2_OK) throw Error(rc, "ab2_scalar_create");
        m_slot = std::shared_ptr<ab2_scalar>(s, [](ab2_scalar* p) { ab2_scalar_destroy(p); });
        m_ctx = ctx;
      }
      m_pending = true;
    }
    T& m_value;
    std::shared_ptr<ab2_scalar> m_slot;
    ab2_context* m_ctx = nullptr;
    bool m_pending = false;
  };
  typedef Future<double> FutureType;

  explicit Algebra(const Context& ctx) : m_ctx(ctx) {}
  const Context& context() const { return m_ctx; }

  static ResourceType resource(Matrix const& A) { return ResourceType{A.context(), A.rows()}; }

  void allocate(ResourceType const& r, Vector& v) const { v.allocate(r.ctx, r.n); }
  template <typename T0, typename... T>
  void allocate(ResourceType const& r, T0& v0, T&... rest) const {
    allocate(r, v0);
    allocate(r, rest...);
  }
  void free(Vector& v) const { v.release(); }
  template <typename T0, typename... T>
  void free(T0& v0, T&... rest) const {
    free(v0);
    free(rest...);
  }

  // ------------------------------------------------------------ BLAS-1
  void copy(Vector const& x, Vector& y) const { chk(ab2_copy(h(), x.handle(), y.handle()), "ab2_copy"); }
  void axpy(double a, Vector const& x, Vector& y) const { chk(ab2_axpy(h(), a, x.handle(), y.handle()), "ab2_axpy"); }
  void aypx(double a, Vector& y, Vector const& x) const { chk(ab2_aypx(h(), a, y.handle(), x.handle()), "ab2_aypx"); }
  void scal(double a, Vector& x) const { chk(ab2_scal(h(), a, x.handle()), "ab2_scal"); }
  double dot(Vector const& x, Vector const& y) const {
    double r = 0.0;
    chk(ab2_dot(h(), x.handle(), y.handle(), &r), "ab2_dot");
    return r;
  }
  void dot(Vector const& x, Vector const& y, FutureType& f) const {
    f.arm(h());
    chk(ab2_dot_async(h(), x.handle(), y.handle(), f.m_slot.get()), "ab2_dot_async");
  }
  double norm0(Vector const& x) const {
    double r = 0.0;
    chk(ab2_norm0(h(), x.handle(), &r), "ab2_norm0");
    return r;
  }
  double norm1(Vector const& x) const {
    double r = 0.0;
    chk(ab2_norm1(h(), x.handle(), &r), "ab2_norm1");
    return r;
  }
  double norm2(Vector const& x) const {
    double r = 0.0;
    chk(ab2_norm2(h(), x.handle(), &r), "ab2_norm2");
    return r;
  }
  void pointwiseMult(Vector const& x, Vector const& y, Vector& w) const {
    chk(ab2_pointwise_mult(h(), x.handle(), y.handle(), w.handle()), "ab2_pointwise_mult");
  }
  void assign(Vector& x, double a) const { chk(ab2_assign(h(), x.handle(), a), "ab2_assign"); }
  // assign(x, f): x_i = f(i), evaluated on the host in index order (the
  // reference calls it with a random generator, so the order matters), then
  // uploaded.
  template <typename LambdaT>
  void assign(Vector& x, LambdaT const& f) const {
    std::vector<double> v((std::size_t)x.size());
    for (std::size_t i = 0; i < v.size(); ++i) v[i] = f(i);
    x.upload(v.data());
  }
  void reciprocal(Vector& x) const { chk(ab2_reciprocal(h(), x.handle()), "ab2_reciprocal"); }

  // ------------------------------------------------------------ matrix
  void mult(Matrix const& A, Vector const& x, Vector& y) const {
    chk(ab2_mult(h(), A.handle(), x.handle(), y.handle()), "ab2_mult");
  }
  void addLMult(double alpha, Matrix const& A, Vector const& x, Vector& y) const {
    chk(ab2_add_lmult(h(), alpha, A.handle(), x.handle(), y.handle()), "ab2_add_lmult");
  }
  void addUMult(double alpha, Matrix const& A, Vector const& x, Vector& y) const {
    chk(ab2_add_umult(h(), alpha, A.handle(), x.handle(), y.handle()), "ab2_add_umult");
  }
  void computeInvDiag(Matrix const& A, Vector& d) const {
    chk(ab2_compute_inv_diag(h(), A.handle(), d.handle()), "ab2_compute_inv_diag");
  }
  void multInvDiag(Matrix const& A, Vector& y) const {
    chk(ab2_mult_inv_diag(h(), A.handle(), y.handle()), "ab2_mult_inv_diag");
  }
  void diagonal(Matrix const& A, Vector& d) const { chk(ab2_diagonal(h(), A.handle(), d.handle()), "ab2_diagonal"); }

  template <typename PrecondT>
  void exec(PrecondT& precond, Vector const& x, Vector& y) {
    precond.solve(*this, x, y);
  }

 private:
  ab2_context* h() const { return m_ctx.handle(); }
  void chk(int rc, const char* what) const { m_ctx.check(rc, what); }
  Context m_ctx;
};

// ILU(0) on the GPU with the interface of ILU0Preconditioner.h:273-323
// (constructor (algebra, matrix[, trace]), init(), solve(algebra, y, x)).
template <typename AlgebraT = Algebra>
class ILU0Preconditioner {
 public:
  typedef AlgebraT AlgebraType;
  typedef typename AlgebraType::Matrix MatrixType;
  typedef typename AlgebraType::Vector VectorType;
  typedef typename MatrixType::ValueType ValueType;

  template <typename TraceT = void>
  ILU0Preconditioner(AlgebraType& algebra, MatrixType const& matrix, TraceT* = nullptr, int schedule = AB2_ILU_AUTO)
      : m_algebra(algebra), m_matrix(matrix), m_schedule(schedule) {}

  void init() {
    ab2_precond_options o{};
    o.kind = AB2_PC_ILU0;
    o.ilu_schedule = m_schedule;
    ab2_precond* p = nullptr;
    const Context& ctx = m_algebra.context();
    ctx.check(ab2_precond_create(ctx.handle(), m_matrix.handle(), &o, &p), "ab2_precond_create");
    m_pc = std::shared_ptr<ab2_precond>(p, [](ab2_precond* q) { ab2_precond_destroy(q); });
  }
  void update() {}
  void solve(AlgebraType& algebra, VectorType const& y, VectorType& x) const {
    const Context& ctx = algebra.context();
    ctx.check(ab2_precond_apply(ctx.handle(), m_pc.get(), y.handle(), x.handle()), "ab2_precond_apply");
  }
  void solve(VectorType const& y, VectorType& x) const { solve(m_algebra, y, x); }

 private:
  AlgebraType& m_algebra;
  MatrixType const& m_matrix;
  int m_schedule;
  std::shared_ptr<ab2_precond> m_pc;
};

// FILU0 on the GPU: the interface of FILU0Preconditioner.h:320-430
// (setParameter "nb-factor-iter" / "nb-solver-iter" / "tol", init, solve) over
// ab2_precond.  The reference's FLUFactorisationAlgo factorises on host
// arrays; here the factor sweeps run on the device with the same arithmetic
// and the application is the device-algebra branch of solveL/solveU, bit for
// bit.  (NeumannPolyPreconditioner.h needs nothing beyond the algebra: the
// reference template runs on Alien::B200::Algebra as it is.)
template <typename AlgebraT = Algebra>
class FILU0Preconditioner {
 public:
  typedef AlgebraT AlgebraType;
  typedef typename AlgebraType::Matrix MatrixType;
  typedef typename AlgebraType::Vector VectorType;
  typedef typename MatrixType::ValueType ValueType;

  template <typename TraceT = void>
  FILU0Preconditioner(AlgebraType& algebra, MatrixType const& matrix, TraceT* = nullptr)
      : m_algebra(algebra), m_matrix(matrix) {}

  void setParameter(std::string param, int value) {
    if (param.compare("nb-factor-iter") == 0) m_factor_iter = value;
    else if (param.compare("nb-solver-iter") == 0) m_solver_iter = value;
  }
  void setParameter(std::string param, double value) {
    if (param.compare("tol") == 0) m_tol = value;
  }
  void init() {
    ab2_precond_options o{};
    o.kind = AB2_PC_FILU0;
    o.filu_factor_iter = m_factor_iter;
    o.filu_solver_iter = m_solver_iter;
    o.filu_tol = m_tol;
    ab2_precond* p = nullptr;
    const Context& ctx = m_algebra.context();
    ctx.check(ab2_precond_create(ctx.handle(), m_matrix.handle(), &o, &p), "ab2_precond_create");
    m_pc = std::shared_ptr<ab2_precond>(p, [](ab2_precond* q) { ab2_precond_destroy(q); });
  }
  void solve(AlgebraType& algebra, VectorType const& y, VectorType& x) const {
    const Context& ctx = algebra.context();
    ctx.check(ab2_precond_apply(ctx.handle(), m_pc.get(), y.handle(), x.handle()), "ab2_precond_apply");
  }
  void solve(VectorType const& y, VectorType& x) const { solve(m_algebra, y, x); }

 private:
  AlgebraType& m_algebra;
  MatrixType const& m_matrix;
  int m_factor_iter = 0, m_solver_iter = 0;
  double m_tol = 0;
  std::shared_ptr<ab2_precond> m_pc;
};

// The fused device-resident solvers: the whole Krylov loop on the GPU
// (ab2_solver_*), or FP32 Krylov inside FP64 refinement (ab2_mixed_*).
class Solver {
 public:
  Solver(const Context& ctx, const Matrix& A, const ab2_solver_options& opts) : m_ctx(ctx) {
    ab2_solver* s = nullptr;
    ctx.check(ab2_solver_create(ctx.handle(), A.handle(), &opts, &s), "ab2_solver_create");
    m_s = std::shared_ptr<ab2_solver>(s, [](ab2_solver* p) { ab2_solver_destroy(p); });
  }
  ab2_status solve(const Vector& b, Vector& x) {
    ab2_status st{};
    m_ctx.check(ab2_solver_solve(m_s.get(), b.handle(), x.handle(), &st), "ab2_solver_solve");
    return st;
  }

 private:
  Context m_ctx;
  std::shared_ptr<ab2_solver> m_s;
};

}  // namespace B200
}  // namespace Alien
