// ref_driver.cpp -- runs Alien's OWN header-only Krylov templates on the CPU.
//
// TEST INFRASTRUCTURE ONLY (oracle).  Built by oracle/Makefile into
// oracle/_ref/libalien_ref.so, straight from the reference sources where they
// lie (ALIEN_REF_SRC, default the read-only reference checkout's src/core):
//   alien/expression/krylov/{Iteration,CG,BiCGStab,DiagPreconditioner,
//                            ILU0Preconditioner,ChebyshevPreconditioner,
//                            FILU0Preconditioner,NeumannPolyPreconditioner}.h
//   alien/handlers/scalar/CSRModifierViewT.h
// Nothing of those files is copied here.  What this file supplies is the
// minimum the templates need from the rest of Alien, which cannot be built in
// this image (Arccore, MPI and Boost are absent):
//   * a CPU algebra (ShimAlgebra) that satisfies the AlgebraT concept used by
//     the templates and restates SimpleCSRInternalLinearAlgebra
//     (kernels/simple_csr/algebra/SimpleCSRInternalLinearAlgebra.h:55-173)
//     through oracle/simplecsr_kernels.h;
//   * a sequential CSR matrix/profile type exposing the members that
//     ILU0Preconditioner.h:51-61 and CSRModifierViewT.h:105-145 touch;
//   * ITraceMng, MatrixDistribution and LUSendRecvTraits stand-ins (the
//     parallel branches that use the latter are never taken: isParallel()
//     is false on one process);
//   * a second matrix type that is not host-only (DevMatrix) with an algebra
//     carrying addLMult/addUMult (ShimDevAlgebra, SimpleCSRMatrixMultT.h:193-233),
//     so that FILU0Preconditioner.h takes its device-algebra branch -- the
//     branch a GPU back end runs.
// The exported C entry points mirror oracle/ab2_oracle.cpp's, so tests can
// check the restatement against the reference templates result for result.

#include <cmath>
#include <cstring>
#include <iostream>
#include <memory>
#include <random>
#include <string>
#include <type_traits>
#include <vector>

#include "../simplecsr_kernels.h"

namespace Alien {

// Discards everything: ChebyshevPreconditioner's Saad branch (_algo1) writes
// to the trace manager unconditionally.
class ITraceMng {
 public:
  std::ostream& info() {
    static std::ostream sink(nullptr);
    return sink;
  }
};

struct MatrixDistribution {};

template <typename Tag>
class LUSendRecvTraits;

namespace shim {

struct Tag {};

struct Profile {
  typedef int IndexType;
  int n = 0;
  std::vector<int> rp, ci, dc;
  std::size_t getNRows() const { return (std::size_t)n; }
  std::size_t getNnz() const { return ci.size(); }
  const int* kcol() const { return rp.data(); }
  const int* cols() const { return ci.data(); }
  const int* dcol() const { return dc.data(); }
};

// The members of DistStructInfo (kernels/simple_csr/DistStructInfo.h) the
// parallel branches of LUFactorisationAlgo read: the rank's columns in the
// distributed numbering (local ids, then ghost ids), the number of local
// entries of each row, and dcol(profile) -- computeUpperDiagOffset
// (DistStructInfo.h:77-92): per row, the first local position whose column is
// not below the row.
struct DistInfo {
  std::vector<int> m_local_row_size;
  std::vector<int> m_cols;
  int m_first_upper_ghost_index = 0;
  int m_send_info = 0;  // FILU0's parallel branch names these; never taken here
  int m_recv_info = 0;
  mutable std::vector<int> m_upper_diag_offset;
  const int* dcol(const Profile& p) const {
    if (m_upper_diag_offset.empty()) {
      m_upper_diag_offset.resize((std::size_t)p.n);
      for (int i = 0; i < p.n; ++i) {
        int idx = p.rp[(std::size_t)i];
        for (int k = p.rp[(std::size_t)i]; k < p.rp[(std::size_t)i] + m_local_row_size[(std::size_t)i]; ++k) {
          if (m_cols[(std::size_t)k] < i) ++idx;
          else break;
        }
        m_upper_diag_offset[(std::size_t)i] = idx;
      }
    }
    return m_upper_diag_offset.data();
  }
};

struct Matrix {
  typedef double ValueType;
  typedef Profile ProfileType;
  typedef Tag TagType;
  typedef DistInfo DistStructInfo;
  static const bool on_host_only = true;

  std::shared_ptr<Profile> profile;
  std::vector<double> values;
  DistInfo dist_info;
  MatrixDistribution dist;

  bool parallel = false;  // one rank of a row-block distribution (dist_info filled)
  int ghosts = 0;
  bool isParallel() const { return parallel; }
  int getSendPolicy() const { return 0; }
  int getRecvPolicy() const { return 0; }
  void* getParallelMng() const { return nullptr; }
  std::size_t getAllocSize() const { return (std::size_t)(profile->n + ghosts); }
  MatrixDistribution const& distribution() const { return dist; }
  Matrix* cloneTo(void*) const { return new Matrix(*this); }
  Profile const& getProfile() const { return *profile; }
  DistInfo const& getDistStructInfo() const { return dist_info; }
  double* data() { return values.data(); }
  const double* data() const { return values.data(); }
  void notifyChanges() {}
  void endUpdate() {}
  ab2_oracle::Csr csr() const { return ab2_oracle::Csr{profile->n, profile->rp.data(), profile->ci.data(), values.data()}; }
};

// The same matrix seen by the templates as living on a device: FILU0's
// solveL/solveU then go through the algebra (copy, addLMult/addUMult,
// pointwiseMult) instead of their host loops.
struct DevMatrix : Matrix {
  static const bool on_host_only = false;
  DevMatrix() = default;
  explicit DevMatrix(Matrix const& m) : Matrix(m) {}
  DevMatrix* cloneTo(void*) const { return new DevMatrix(*this); }
};

struct Vector {
  std::vector<double> v;
  void resize(std::size_t n) { v.resize(n); }
  double* data() { return v.data(); }
  const double* data() const { return v.data(); }
  int size() const { return (int)v.size(); }
};

struct LUOp {
  LUOp(Matrix&, MatrixDistribution const&, std::vector<int>&) {}
  void recvLowerNeighbLUData(double*) {}
  void sendUpperNeighbLUData(double*) {}
};

// Ghost exchange of FILU0's parallel sweeps (never constructed: one process).
struct VecOp {
  template <typename... A>
  explicit VecOp(A&&...) {}
  void lowerRecv() {}
  void upperSend() {}
  void upperRecv() {}
  void lowerSend() {}
};

}  // namespace shim

template <>
class LUSendRecvTraits<shim::Tag> {
 public:
  typedef shim::LUOp matrix_op_type;
  typedef shim::VecOp vector_op_type;
};

// The AlgebraT concept as the Krylov templates call it.
class ShimAlgebra {
 public:
  typedef shim::Matrix Matrix;
  typedef shim::Vector Vector;
  typedef int ResourceType;

  struct NullValueException {
    std::string which;
    explicit NullValueException(std::string const& w) : which(w) {}
  };

  template <typename T>
  class Future {
   public:
    explicit Future(T& v) : m_value(v) {}
    T& operator()() { return m_value; }
    T get() { return m_value; }

   private:
    T& m_value;
  };
  typedef Future<double> FutureType;

  // r.r values seen by the stop test (Iteration only uses the future form of dot).
  std::vector<double> history;
  bool skip_first = true;

  static ResourceType resource(Matrix const& A) { return A.profile->n; }
  void allocate(ResourceType n, Vector& v) { v.v.assign((std::size_t)n, 0.0); }
  template <typename T0, typename... T>
  void allocate(ResourceType n, T0& v0, T&... rest) {
    allocate(n, v0);
    allocate(n, rest...);
  }
  void free(Vector& v) { v.v.clear(); }
  template <typename T0, typename... T>
  void free(T0& v0, T&... rest) {
    free(v0);
    free(rest...);
  }

  void mult(Matrix const& A, Vector const& x, Vector& y) const { ab2_oracle::spmv(A.csr(), x.data(), y.data()); }
  void copy(Vector const& x, Vector& y) const { ab2_oracle::copy(x.size(), x.data(), y.data()); }
  void axpy(double a, Vector const& x, Vector& y) const { ab2_oracle::axpy(x.size(), a, x.data(), y.data()); }
  void scal(double a, Vector& x) const { ab2_oracle::scal(x.size(), a, x.data()); }
  double dot(Vector const& x, Vector const& y) const { return ab2_oracle::dot(x.size(), x.data(), y.data()); }
  void dot(Vector const& x, Vector const& y, FutureType& f) {
    f() = ab2_oracle::dot(x.size(), x.data(), y.data());
    if (&x == &y) {
      if (skip_first) skip_first = false;
      else history.push_back(f());
    }
  }
  double norm2(Vector const& x) const { return std::sqrt(dot(x, x)); }
  void pointwiseMult(Vector const& x, Vector const& y, Vector& w) const {
    ab2_oracle::pmult(x.size(), x.data(), y.data(), w.data());
  }
  void assign(Vector& x, double a) const {
    for (auto& e : x.v) e = a;
  }
  template <typename LambdaT>
  void assign(Vector& x, LambdaT const& f) const {
    for (std::size_t i = 0; i < x.v.size(); ++i) x.v[i] = f(i);
  }
  void computeInvDiag(Matrix const& A, Vector& inv) const {
    std::vector<int> d = ab2_oracle::diag_offsets(A.csr());
    for (int i = 0; i < A.profile->n; ++i) inv.v[i] = 1. / A.values[d[i]];
  }
  template <typename PrecondT>
  void exec(PrecondT& precond, Vector const& x, Vector& y) {
    precond.solve(*this, x, y);
  }
};

// ShimAlgebra over DevMatrix, plus the strict-triangle products of
// SimpleCSRMatrixMultT::_seqAddLMult/_seqAddUMult (:193-233): per row
// tmpy += alpha * a_k * x[c_k] in CSR order.
class ShimDevAlgebra : public ShimAlgebra {
 public:
  typedef shim::DevMatrix Matrix;
  void addLMult(double alpha, Matrix const& A, Vector const& x, Vector& y) const { tri(alpha, A, x, y, true); }
  void addUMult(double alpha, Matrix const& A, Vector const& x, Vector& y) const { tri(alpha, A, x, y, false); }
  template <typename PrecondT>
  void exec(PrecondT& precond, Vector const& x, Vector& y) {
    precond.solve(*this, x, y);
  }

 private:
  static void tri(double alpha, Matrix const& A, Vector const& x, Vector& y, bool lower) {
    const shim::Profile& p = *A.profile;
    for (int i = 0; i < p.n; ++i) {
      double t = y.v[i];
      const int kb = lower ? p.rp[i] : p.dc[i] + 1, ke = lower ? p.dc[i] : p.rp[i + 1];
      for (int k = kb; k < ke; ++k) t += alpha * A.values[k] * x.v[p.ci[k]];
      y.v[i] = t;
    }
  }
};

}  // namespace Alien

#include <alien/expression/krylov/Iteration.h>
#include <alien/expression/krylov/CG.h>
#include <alien/expression/krylov/BiCGStab.h>
#include <alien/expression/krylov/DiagPreconditioner.h>
#include <alien/expression/krylov/ChebyshevPreconditioner.h>
#include <alien/expression/krylov/ILU0Preconditioner.h>
#include <alien/expression/krylov/FILU0Preconditioner.h>
#include <alien/expression/krylov/NeumannPolyPreconditioner.h>

extern "C" {

// Same layout as orc_options / orc_result in ab2_oracle.cpp (dot_mode,
// tree_blocks and cheb_lanczos have no meaning here: the templates sum dots
// sequentially and only know the power-method bounds).
typedef struct {
  int solver;
  int precond;
  double tol;
  int max_iter;
  double poly_factor;
  int poly_order;
  int poly_factor_max_iter;
  int dot_mode;
  int tree_blocks;
  int cheb_saad;
  int cheb_lanczos;
  int filu_factor_iter;
  int filu_solver_iter;
} ref_options;

typedef struct {
  int iterations;
  int converged;
  int error;
  int breakdown;
  double nrm2_b;
  double last_rr;
  double cheb_alpha;
  double cheb_beta;
  int history_len;
} ref_result;

}  // extern "C"

namespace {

using Alien::ShimAlgebra;

Alien::ITraceMng g_trace;
thread_local bool g_saad = false;

Alien::shim::Matrix make_matrix(int n, const int* rp, const int* ci, const double* v) {
  Alien::shim::Matrix A;
  A.profile = std::make_shared<Alien::shim::Profile>();
  A.profile->n = n;
  A.profile->rp.assign(rp, rp + n + 1);
  A.profile->ci.assign(ci, ci + rp[n]);
  A.profile->dc = ab2_oracle::diag_offsets(ab2_oracle::Csr{n, rp, ci, nullptr});
  A.values.assign(v, v + rp[n]);
  return A;
}

int breakdown_code(std::string const& w) {
  if (w == "alpha") return 1;
  if (w == "beta") return 2;
  if (w == "rho") return 3;
  return 9;
}

template <typename Alg, typename SolverT, typename PrecondT>
int run(Alg& alg, SolverT& solver, PrecondT& pc, Alien::Iteration<Alg>& it, typename Alg::Matrix const& A,
        Alien::shim::Vector const& b, Alien::shim::Vector& x, ref_result* res) {
  try {
    solver.solve(pc, it, A, b, x);
  } catch (ShimAlgebra::NullValueException const& e) {
    res->error = -3;
    res->breakdown = breakdown_code(e.which);
  }
  return res->error;
}

template <typename Alg>
int solve_with(int n, const int* rp, const int* ci, const double* v, const double* b, double* x,
               const ref_options* o, ref_result* res, double* hist, int hist_cap) {
  std::memset(res, 0, sizeof(*res));
  Alg alg;
  typename Alg::Matrix A(make_matrix(n, rp, ci, v));
  Alien::shim::Vector vb, vx;
  vb.v.assign(b, b + n);
  vx.v.assign(x, x + n);
  Alien::Iteration<Alg> it(alg, vb, o->tol, o->max_iter, nullptr);

  auto finish = [&]() {
    for (int i = 0; i < n; ++i) x[i] = vx.v[i];
    res->iterations = it();
    res->converged = it.getStatus() ? 1 : 0;
    res->nrm2_b = ab2_oracle::dot(n, b, b);
    res->history_len = (int)alg.history.size();
    res->last_rr = alg.history.empty() ? 0.0 : alg.history.back();
    for (int i = 0; i < (int)alg.history.size() && i < hist_cap && hist; ++i) hist[i] = alg.history[i];
  };

  auto with_solver = [&](auto& pc) {
    if (o->solver == 0) {
      Alien::CG<Alg> s(alg, nullptr);
      run(alg, s, pc, it, A, vb, vx, res);
    } else {
      Alien::BiCGStab<Alg> s(alg, nullptr);
      run(alg, s, pc, it, A, vb, vx, res);
    }
  };

  constexpr bool dev = std::is_same<Alg, Alien::ShimDevAlgebra>::value;
  if (dev != (o->precond == 4)) return -6;
  if constexpr (dev) {
    Alien::FILU0Preconditioner<Alg> pc(alg, A, nullptr);
    pc.setParameter("nb-factor-iter", o->filu_factor_iter);
    pc.setParameter("nb-solver-iter", o->filu_solver_iter);
    pc.init();
    with_solver(pc);
    finish();
    return res->error;
  } else {
  switch (o->precond) {
    case 1: {
      Alien::DiagPreconditioner<Alg> pc(alg, A);
      pc.init();
      with_solver(pc);
      break;
    }
    case 2: {
      Alien::ILU0Preconditioner<Alg> pc(alg, A, nullptr);
      pc.init();
      with_solver(pc);
      break;
    }
    case 3: {
      if (o->cheb_saad) {
        Alien::ChebyshevPreconditioner<Alg, true> pc(alg, A, o->poly_factor, o->poly_order, o->poly_factor_max_iter,
                                                     &g_trace);
        pc.init();
        with_solver(pc);
      } else {
        Alien::ChebyshevPreconditioner<Alg> pc(alg, A, o->poly_factor, o->poly_order, o->poly_factor_max_iter,
                                               nullptr);
        pc.init();
        with_solver(pc);
      }
      break;
    }
    case 5: {
      Alien::NeumannPolyPreconditioner<Alg> pc(alg, A, o->poly_factor, o->poly_order, o->poly_factor_max_iter,
                                               nullptr);
      pc.init();
      with_solver(pc);
      break;
    }
    default: return -6;
  }
  finish();
  return res->error;
  }
}

}  // namespace

extern "C" {

// FILU0 runs on the device-algebra shim (its GPU branch); everything else on
// the host SimpleCSR shim.
int ref_solve(int n, const int* rp, const int* ci, const double* v, const double* b, double* x,
              const ref_options* o, ref_result* res, double* hist, int hist_cap) {
  if (o->precond == 4) return solve_with<Alien::ShimDevAlgebra>(n, rp, ci, v, b, x, o, res, hist, hist_cap);
  return solve_with<ShimAlgebra>(n, rp, ci, v, b, x, o, res, hist, hist_cap);
}

// ILU(0) factor computed by the reference's LUFactorisationAlgo.
int ref_ilu0_factor(int n, const int* rp, const int* ci, const double* v, double* lu) {
  ShimAlgebra alg;
  Alien::shim::Matrix A = make_matrix(n, rp, ci, v);
  Alien::LUFactorisationAlgo<Alien::shim::Matrix, Alien::shim::Vector> algo;
  algo.init(alg, A);
  const Alien::shim::Matrix& LU = algo.getLUMatrix();
  std::memcpy(lu, LU.values.data(), sizeof(double) * (size_t)rp[n]);
  return 0;
}

// One application of the reference's ILU0Preconditioner: x = (LU)^-1 y.
int ref_ilu0_apply(int n, const int* rp, const int* ci, const double* v, const double* y, double* x) {
  ShimAlgebra alg;
  Alien::shim::Matrix A = make_matrix(n, rp, ci, v);
  Alien::ILU0Preconditioner<ShimAlgebra> pc(alg, A, nullptr);
  pc.init();
  Alien::shim::Vector vy, vx;
  vy.v.assign(y, y + n);
  vx.v.assign((std::size_t)n, 0.0);
  alg.exec(pc, vy, vx);
  std::memcpy(x, vx.v.data(), sizeof(double) * (size_t)n);
  return 0;
}

// One rank's block-Jacobi ILU(0): the reference's LUFactorisationAlgo with
// isParallel() true (ILU0Preconditioner.h:93-119 factorisation, :181-231
// sweeps) on the rank's rows in the distributed layout (rp, ci with local ids
// then ghost ids n.., lrs = local entries per row).  lu receives the factor
// (rp[n] values, distributed order), x = (LU)^-1 y.
int ref_bj_ilu0_apply(int n, int ghosts, const int* rp, const int* ci, const double* v, const int* lrs, const double* y,
                      double* x, double* lu) {
  ShimAlgebra alg;
  Alien::shim::Matrix A;
  A.profile = std::make_shared<Alien::shim::Profile>();
  A.profile->n = n;
  A.profile->rp.assign(rp, rp + n + 1);
  A.profile->ci.assign(ci, ci + rp[n]);  // the profile's own columns are not read on this branch
  A.values.assign(v, v + rp[n]);
  A.parallel = true;
  A.ghosts = ghosts;
  A.dist_info.m_local_row_size.assign(lrs, lrs + n);
  A.dist_info.m_cols.assign(ci, ci + rp[n]);
  Alien::LUFactorisationAlgo<Alien::shim::Matrix, Alien::shim::Vector> algo;
  algo.init(alg, A);
  const Alien::shim::Matrix& LU = algo.getLUMatrix();
  if (lu) std::memcpy(lu, LU.values.data(), sizeof(double) * (size_t)rp[n]);
  Alien::shim::Vector vy, vx;
  vy.v.assign(y, y + n);
  vx.v.assign((std::size_t)n, 0.0);
  algo.solve(alg, vy, vx);
  std::memcpy(x, vx.v.data(), sizeof(double) * (size_t)n);
  return 0;
}

// One application of the reference's ChebyshevPreconditioner (non-Saad).
int ref_cheb_apply(int n, const int* rp, const int* ci, const double* v, double factor, int order, int max_iter,
                   const double* xin, double* yout) {
  ShimAlgebra alg;
  Alien::shim::Matrix A = make_matrix(n, rp, ci, v);
  Alien::shim::Vector vx, vy;
  vx.v.assign(xin, xin + n);
  vy.v.assign((std::size_t)n, 0.0);
  if (g_saad) {
    Alien::ChebyshevPreconditioner<ShimAlgebra, true> pc(alg, A, factor, order, max_iter, &g_trace);
    pc.init();
    alg.exec(pc, vx, vy);
  } else {
    Alien::ChebyshevPreconditioner<ShimAlgebra> pc(alg, A, factor, order, max_iter, nullptr);
    pc.init();
    alg.exec(pc, vx, vy);
  }
  std::memcpy(yout, vy.v.data(), sizeof(double) * (size_t)n);
  return 0;
}

// One application of the reference's FILU0Preconditioner on the
// device-algebra shim; lu (optional) receives its factor in CSR order.
int ref_filu0_apply(int n, const int* rp, const int* ci, const double* v, int factor_iter, int solver_iter,
                    const double* y, double* x, double* lu) {
  Alien::ShimDevAlgebra alg;
  Alien::shim::DevMatrix A(make_matrix(n, rp, ci, v));
  Alien::FILU0Preconditioner<Alien::ShimDevAlgebra> pc(alg, A, nullptr);
  pc.setParameter("nb-factor-iter", factor_iter);
  pc.setParameter("nb-solver-iter", solver_iter);
  pc.init();
  Alien::shim::Vector vy, vx;
  vy.v.assign(y, y + n);
  vx.v.assign((std::size_t)n, 0.0);
  alg.exec(pc, vy, vx);
  std::memcpy(x, vx.v.data(), sizeof(double) * (size_t)n);
  if (lu) {
    // the factor, by repeating the reference's own factorisation on a clone
    Alien::FLUFactorisationAlgo<Alien::shim::DevMatrix, Alien::shim::Vector> algo;
    algo.setParameter("nb-factor-iter", factor_iter);
    algo.init(alg, A);
    std::memcpy(lu, algo.getLUMatrix().values.data(), sizeof(double) * (size_t)rp[n]);
  }
  return 0;
}

// One application of the reference's NeumannPolyPreconditioner; factor must
// be nonzero (factor = 0 draws from std::random_device).
int ref_neumann_apply(int n, const int* rp, const int* ci, const double* v, double factor, int order, int max_iter,
                      const double* x, double* y, double* omega) {
  if (factor == 0.0) return -6;
  ShimAlgebra alg;
  Alien::shim::Matrix A = make_matrix(n, rp, ci, v);
  Alien::NeumannPolyPreconditioner<ShimAlgebra> pc(alg, A, factor, order, max_iter, nullptr);
  pc.init();
  Alien::shim::Vector vx, vy;
  vx.v.assign(x, x + n);
  vy.v.assign((std::size_t)n, 0.0);
  alg.exec(pc, vx, vy);
  std::memcpy(y, vy.v.data(), sizeof(double) * (size_t)n);
  if (omega) *omega = factor;
  return 0;
}

// Chebyshev template instance used by ref_cheb_apply (1: saad = true).
int ref_set_cheb_saad(int saad) {
  g_saad = saad != 0;
  return 0;
}

}  // extern "C"
