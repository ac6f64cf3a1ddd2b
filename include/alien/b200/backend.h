// backend.h -- libab2 as an Alien back end: the b200 tag, its AlgebraTraits,
// and the internal algebra and solver that Alien's LinearAlgebra and
// LinearSolver facades call.
//
// Alien reaches a back end through AlgebraTraits<Tag> (declared in
// core/backend/BackEnd.h:29-31): LinearAlgebra<Tag> asks algebra_factory() for
// an IInternalLinearAlgebra<Matrix, Vector> (LinearAlgebra.h:72-75,
// IInternalLinearAlgebraT.h:49-188) and LinearSolver<Tag> asks
// solver_factory(options) for an IInternalLinearSolver<Matrix, Vector>
// (LinearSolver.h:78-82, IInternalLinearSolverT.h:59-125).  This header
// supplies both for BackEnd::tag::b200, in the shape of the Ginkgo plugin's
// (plugins/ginkgo/include/alien/ginkgo/backend.h:51-76):
//
//   * InternalLinearAlgebra: every IInternalLinearAlgebra operation (norm0/1/2,
//     mult, axpy, aypx, copy, dot, scal, diagonal, reciprocal, pointwiseMult)
//     runs on the GPU through the C ABI of include/ab2.h, with the rounding of
//     SimpleCSRInternalLinearAlgebra (see B200Algebra.h);
//   * InternalLinearSolver: solve(A, b, x) is the device-resident CG or
//     BiCGStab of ab2_solver_* with the preconditioner the options name (or,
//     with Options::mixed, FP32 Krylov inside FP64 refinement, ab2_mixed_*);
//     it fills SolverStatus (succeeded, final relative residual, iterations,
//     error) as the plugins' solvers do (ginkgo_linear_solver.cpp:177-186) and
//     SolverStat's counters and timers as SolverStater does;
//   * fromSimpleCSR / toSimpleCSR: the data side of the simplecsr <-> b200
//     converters -- the device matrix from the arrays a SimpleCSRMatrix holds
//     (CSRStructInfo row offsets and columns, the value array: what
//     SimpleCSRtoSYCLMatrixConverter.cc:74-104 reads), and a device vector
//     downloaded into a host view (SYCLtoSimpleCSRVectorConverter.cc:60-70).
//
// Unlike B200Algebra.h and ab2.h, this header includes Alien's own headers
// (alien/core/backend/*.h, alien/expression/solver/*.h) and through them
// Arccore's; Alien's SolverStat.cc is linked in as a library source.
#pragma once

#include <alien/core/backend/BackEnd.h>
#include <alien/core/backend/IInternalLinearAlgebraT.h>
#include <alien/core/backend/IInternalLinearSolverT.h>
#include <alien/expression/solver/ILinearSolver.h>
#include <alien/expression/solver/SolverStat.h>

#include <alien/b200/B200Algebra.h>

#include <chrono>
#include <string>

namespace Alien {
namespace B200 {

// The solver settings, named as the krylov example's options (solver,
// precond, tol, max-iter, poly-*, nb-factor-iter / nb-solver-iter).
struct Options {
  int device = 0;                // GPU of the context the factories create
  std::string solver = "cg";     // "cg" or "bicgs"
  std::string precond = "diag";  // "none", "diag", "ilu0", "cheb", "filu0", "neumann"
  double tol = 1e-8;             // Iteration's relative residual (recursive)
  int max_iter = 1000;
  double poly_factor = 0.0;      // Chebyshev / Neumann settings
  int poly_order = 3;
  int poly_factor_max_iter = 10;
  bool cheb_saad = false;
  bool cheb_lanczos = false;
  int filu_factor_iter = 0;
  int filu_solver_iter = 3;
  double filu_tol = 0.0;
  bool use_graph = true;         // the iteration loop as one CUDA graph
  bool mixed = false;            // FP32 Krylov inside FP64 refinement (tol: the true residual)
  double inner_tol = 1e-4;       // mixed: relative residual of each FP32 solve
  int max_outer = 20;            // mixed: refinement steps

  int solverKind() const {
    if (solver == "cg") return AB2_SOLVER_CG;
    if (solver == "bicgs" || solver == "bicgstab") return AB2_SOLVER_BICGSTAB;
    throw Error(AB2_ERR_BAD_ARG, "unknown solver '" + solver + "'");
  }
  int precondKind() const {
    if (precond == "none") return AB2_PC_NONE;
    if (precond == "diag") return AB2_PC_DIAG;
    if (precond == "ilu0") return AB2_PC_ILU0;
    if (precond == "cheb" || precond == "poly") return AB2_PC_CHEB;
    if (precond == "filu0") return AB2_PC_FILU0;
    if (precond == "neumann") return AB2_PC_NEUMANN;
    throw Error(AB2_ERR_BAD_ARG, "unknown preconditioner '" + precond + "'");
  }
  ab2_solver_options solverOptions() const {
    ab2_solver_options o;
    ab2_solver_options_default(&o);
    o.solver = solverKind();
    o.precond = precondKind();
    o.tol = tol;
    o.max_iter = max_iter;
    o.poly_factor = poly_factor;
    o.poly_order = poly_order;
    o.poly_factor_max_iter = poly_factor_max_iter;
    o.cheb_saad = cheb_saad ? 1 : 0;
    o.cheb_lanczos = cheb_lanczos ? 1 : 0;
    o.filu_factor_iter = filu_factor_iter;
    o.filu_solver_iter = filu_solver_iter;
    o.filu_tol = filu_tol;
    o.use_graph = use_graph ? 1 : 0;
    return o;
  }
  ab2_mixed_options mixedOptions() const {
    ab2_mixed_options o;
    ab2_mixed_options_default(&o);
    o.solver = solverKind();
    o.precond = precondKind();
    o.tol = tol;
    o.max_outer = max_outer;
    o.inner_tol = inner_tol;
    o.inner_max_iter = max_iter;
    o.poly_factor = poly_factor;
    o.poly_order = poly_order;
    o.poly_factor_max_iter = poly_factor_max_iter;
    o.cheb_saad = cheb_saad ? 1 : 0;
    o.cheb_lanczos = cheb_lanczos ? 1 : 0;
    o.filu_factor_iter = filu_factor_iter;
    o.filu_solver_iter = filu_solver_iter;
    o.filu_tol = filu_tol;
    o.use_graph = use_graph ? 1 : 0;
    return o;
  }
};

// IInternalLinearAlgebra over libab2.  The operations are those of
// Alien::B200::Algebra (B200Algebra.h), which also serves Alien's Krylov
// templates as their AlgebraT: algebra() hands it out.
class InternalLinearAlgebra : public IInternalLinearAlgebra<Matrix, Vector> {
 public:
  explicit InternalLinearAlgebra(const Context& ctx) : m_algebra(ctx) {}

  Real norm0(const Vector& x) const override { return m_algebra.norm0(x); }
  Real norm1(const Vector& x) const override { return m_algebra.norm1(x); }
  Real norm2(const Vector& x) const override { return m_algebra.norm2(x); }
  void mult(const Matrix& a, const Vector& x, Vector& r) const override { m_algebra.mult(a, x, r); }
  void axpy(Real alpha, const Vector& x, Vector& y) const override { m_algebra.axpy(alpha, x, y); }
  void aypx(Real alpha, Vector& y, const Vector& x) const override { m_algebra.aypx(alpha, y, x); }
  void copy(const Vector& x, Vector& r) const override { m_algebra.copy(x, r); }
  Real dot(const Vector& x, const Vector& y) const override { return m_algebra.dot(x, y); }
  void scal(Real alpha, Vector& x) const override { m_algebra.scal(alpha, x); }
  void diagonal(const Matrix& a, Vector& x) const override { m_algebra.diagonal(a, x); }
  void reciprocal(Vector& x) const override { m_algebra.reciprocal(x); }
  void pointwiseMult(const Vector& x, const Vector& y, Vector& w) const override { m_algebra.pointwiseMult(x, y, w); }

  const Algebra& algebra() const { return m_algebra; }
  Algebra& algebra() { return m_algebra; }
  const Context& context() const { return m_algebra.context(); }

 private:
  Algebra m_algebra;
};

// IInternalLinearSolver over the device-resident solvers.  One GPU, no
// distribution: hasParallelSupport() is false (the row-block distribution is
// B200DistAlgebra.h's).
class InternalLinearSolver : public IInternalLinearSolver<Matrix, Vector> {
 public:
  explicit InternalLinearSolver(const Options& options = Options()) : m_options(options) {}

  void init() override {}
  void end() override {}

  // Set-up (preconditioner, graph) and solve from the x given; false when the
  // solve did not converge (status.error says why: AB2_ERR_NOT_CONVERGED,
  // AB2_ERR_BREAKDOWN, ...).  ABI failures other than those throw Error.
  bool solve(const Matrix& A, const Vector& b, Vector& x) override {
    const Context& ctx = A.context();
    const auto t0 = std::chrono::steady_clock::now();
    double setup_ms = 0, solve_ms = 0;
    if (m_options.mixed) {
      const ab2_mixed_options o = m_options.mixedOptions();
      ab2_mixed* m = nullptr;
      ctx.check(ab2_mixed_create(ctx.handle(), A.handle(), &o, &m), "ab2_mixed_create");
      ab2_mixed_status st{};
      const int rc = ab2_mixed_solve(m, b.handle(), x.handle(), &st);
      ab2_mixed_destroy(m);
      if (rc != AB2_OK && rc != AB2_ERR_NOT_CONVERGED && rc != AB2_ERR_BREAKDOWN) ctx.check(rc, "ab2_mixed_solve");
      m_status.succeeded = st.succeeded != 0;
      m_status.residual = st.true_residual;
      m_status.iteration_count = st.inner_iterations;
      m_status.error = st.error;
      setup_ms = st.setup_ms;
      solve_ms = st.solve_ms;
    } else {
      const ab2_solver_options o = m_options.solverOptions();
      ab2_solver* s = nullptr;
      ctx.check(ab2_solver_create(ctx.handle(), A.handle(), &o, &s), "ab2_solver_create");
      ab2_status st{};
      const int rc = ab2_solver_solve(s, b.handle(), x.handle(), &st);
      ab2_solver_destroy(s);
      if (rc != AB2_OK && rc != AB2_ERR_NOT_CONVERGED && rc != AB2_ERR_BREAKDOWN) ctx.check(rc, "ab2_solver_solve");
      m_status.succeeded = st.succeeded != 0;
      m_status.residual = st.residual;
      m_status.iteration_count = st.iterations;
      m_status.error = st.error;
      setup_ms = st.setup_ms;
      solve_ms = st.solve_ms;
    }
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    m_stat.record(m_status.iteration_count, setup_ms * 1e-3, solve_ms * 1e-3, wall);
    return m_status.succeeded;
  }

  SolverStat const& getSolverStat() const override { return m_stat; }
  SolverStat& getSolverStat() override { return m_stat; }
  bool hasParallelSupport() const override { return false; }
  const SolverStatus& getStatus() const override { return m_status; }

  const Options& options() const { return m_options; }

 private:
  // SolverStat's counters, updated after each solve as SolverStater does
  // (solve count, iterations, last and total prepare / solve times; the
  // "cpu" times are the host wall clock of the whole call).
  class Stat : public SolverStat {
   public:
    void record(Integer iterations, Real prepare_s, Real solve_s, Real wall_s) {
      ++m_solve_count;
      m_last_iteration_count = iterations;
      m_iteration_count += iterations;
      m_last_prepare_time = prepare_s;
      m_prepare_time += prepare_s;
      m_last_solve_time = solve_s;
      m_solve_time += solve_s;
      m_last_prepare_cpu_time = 0;
      m_last_solve_cpu_time = wall_s;
      m_solve_cpu_time += wall_s;
    }
  };

  Options m_options;
  SolverStatus m_status;
  Stat m_stat;
};

// The factories AlgebraTraits<BackEnd::tag::b200> hands to the facades.  Each
// algebra or default solver gets a context on Options().device; a solver made
// from options uses options.device.
inline IInternalLinearAlgebra<Matrix, Vector>* InternalLinearAlgebraFactory(int device = 0) {
  return new InternalLinearAlgebra(Context(device));
}
inline IInternalLinearSolver<Matrix, Vector>* InternalLinearSolverFactory(const Options& options) {
  return new InternalLinearSolver(options);
}
inline IInternalLinearSolver<Matrix, Vector>* InternalLinearSolverFactory() {
  return new InternalLinearSolver(Options());
}

// simplecsr -> b200: the device matrix from a SimpleCSRMatrix's arrays --
// row offsets (n + 1) and ascending columns of its CSRStructInfo, and the
// value array -- copied to the GPU (CSR + sliced ELL + the 7-point bands when
// the profile has them; AB2_FMT_F32 on request for the mixed solver).
inline Matrix fromSimpleCSR(const Context& ctx, Arccore::ConstArrayView<int> row_offset,
                            Arccore::ConstArrayView<int> cols, Arccore::ConstArrayView<Real> values,
                            int formats = AB2_FMT_CSR | AB2_FMT_ELL | AB2_FMT_STENCIL) {
  const int n = row_offset.size() - 1;
  if (n < 0 || cols.size() != row_offset[n] || values.size() != row_offset[n])
    throw Error(AB2_ERR_BAD_ARG, "fromSimpleCSR: row offsets, columns and values disagree");
  return Matrix(ctx, n, row_offset.data(), cols.data(), values.data(), formats);
}

// simplecsr -> b200 for a vector, and b200 -> simplecsr: host values in and out.
inline Vector fromSimpleCSR(const Context& ctx, Arccore::ConstArrayView<Real> values) {
  Vector v(ctx, values.size());
  if (values.size()) v.upload(values.data());
  return v;
}
inline void toSimpleCSR(const Vector& v, Arccore::ArrayView<Real> values) {
  if (values.size() != v.size()) throw Error(AB2_ERR_BAD_ARG, "toSimpleCSR: size mismatch");
  if (values.size()) v.download(values.data());
}

}  // namespace B200

namespace BackEnd {
namespace tag {
struct b200 {};
}  // namespace tag
}  // namespace BackEnd

template <>
struct AlgebraTraits<BackEnd::tag::b200> {
  using matrix_type = B200::Matrix;
  using vector_type = B200::Vector;
  using options_type = B200::Options;
  using algebra_type = IInternalLinearAlgebra<matrix_type, vector_type>;
  using solver_type = IInternalLinearSolver<matrix_type, vector_type>;

  static auto algebra_factory() { return B200::InternalLinearAlgebraFactory(); }
  static auto solver_factory(const options_type& options) { return B200::InternalLinearSolverFactory(options); }
  static auto solver_factory() { return B200::InternalLinearSolverFactory(); }
  static BackEndId name() { return "b200"; }
};

}  // namespace Alien
