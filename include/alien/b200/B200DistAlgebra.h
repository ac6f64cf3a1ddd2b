// B200DistAlgebra.h -- Alien's AlgebraT concept on libab2's row-block
// distribution (include/ab2_dist.h), header-only C++17.
//
// The reference runs its Krylov templates (expression/krylov/CG.h,
// BiCGStab.h, Iteration.h, DiagPreconditioner.h, ...) unchanged on every MPI
// rank; what makes them parallel is the algebra: SimpleCSRInternalLinearAlgebra
// over a distributed SimpleCSRMatrix multiplies with a ghost exchange
// (SimpleCSRMatrixMultT::_parallelMult, SimpleCSRMatrixMultT.h:85-128) and
// sums dot products over the ranks (CBLASMPIKernel.h:85-125).
// Alien::B200::DistAlgebra is that algebra on the GPU: one instance per rank,
// each driven by its own host thread (a local group of ranks in one process)
// or process (NCCL), running the same template code:
//
//   auto comms = Alien::B200::Comm::localGroup({ctx0, ctx1});   // or Comm::nccl(...)
//   // on rank r's thread:
//   Alien::B200::DistMatrix A(ctx_r, comms[r], offsets, row_ptr, cols, vals);
//   Alien::B200::DistAlgebra alg(ctx_r, comms[r]);
//   Alien::B200::Vector b, x;  alg.allocate(DistAlgebra::resource(A), b, x);
//   Alien::CG<Alien::B200::DistAlgebra> solver(alg, trace);
//   Alien::B200::DistILU0Preconditioner<> ilu(alg, A);  ilu.init();
//   Alien::Iteration<Alien::B200::DistAlgebra> it(alg, b, tol, max_iter, trace);
//   solver.solve(ilu, it, A, b, x);
//
// Collective members (mult, dot, norm1, norm2, and the DistMatrix
// constructor) must be reached by every rank in the same order, which the
// templates do.  ILU(0) is block Jacobi, as the reference's parallel
// LUFactorisationAlgo (ILU0Preconditioner.h:93-119, 181-231).
#pragma once

#include <ab2_dist.h>
#include <alien/b200/B200Algebra.h>

#include <array>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

namespace Alien {
namespace B200 {

// One rank of a communicator (ab2_comm).
class Comm {
 public:
  Comm() = default;
  static std::vector<Comm> localGroup(std::vector<Context> const& ctxs, double timeout_s = 120.0) {
    std::vector<ab2_context*> hs;
    for (auto const& c : ctxs) hs.push_back(c.handle());
    std::vector<ab2_comm*> out(hs.size(), nullptr);
    const int rc = ab2_comm_local_group(hs.data(), (int)hs.size(), timeout_s, out.data());
    if (rc != AB2_OK) throw Error(rc, "ab2_comm_local_group failed");
    std::vector<Comm> comms;
    for (std::size_t r = 0; r < out.size(); ++r) comms.push_back(Comm(ctxs[r], out[r]));
    return comms;
  }
  static std::array<unsigned char, AB2_COMM_ID_BYTES> ncclUniqueId() {
    std::array<unsigned char, AB2_COMM_ID_BYTES> id{};
    const int rc = ab2_comm_nccl_unique_id(id.data());
    if (rc != AB2_OK) throw Error(rc, "ab2_comm_nccl_unique_id failed");
    return id;
  }
  static Comm nccl(const Context& ctx, const unsigned char* id, int rank, int size) {
    ab2_comm* h = nullptr;
    ctx.check(ab2_comm_nccl_create(ctx.handle(), id, rank, size, &h), "ab2_comm_nccl_create");
    return Comm(ctx, h);
  }
  int rank() const {
    int r = 0;
    ab2_comm_rank(m_h.get(), &r);
    return r;
  }
  int size() const {
    int s = 0;
    ab2_comm_size(m_h.get(), &s);
    return s;
  }
  ab2_comm* handle() const { return m_h.get(); }
  const Context& context() const { return m_ctx; }

 private:
  Comm(const Context& ctx, ab2_comm* h) : m_ctx(ctx), m_h(h, [](ab2_comm* c) { ab2_comm_destroy(c); }) {}
  Context m_ctx;
  std::shared_ptr<ab2_comm> m_h;
};

// This rank's rows of a row-block distributed CSR matrix, columns in global
// numbering (ascending in each row).  Constructing it is collective.
class DistMatrix {
 public:
  typedef double ValueType;

  DistMatrix() = default;
  DistMatrix(const Context& ctx, const Comm& comm, const int* offsets, const int* row_ptr, const int* cols,
             const double* vals, int formats = AB2_FMT_CSR | AB2_FMT_ELL)
      : m_ctx(ctx), m_comm(comm) {
    ab2_dist_matrix* h = nullptr;
    ctx.check(ab2_dist_matrix_create(ctx.handle(), comm.handle(), offsets, row_ptr, cols, vals, formats, &h),
              "ab2_dist_matrix_create");
    m_h = std::shared_ptr<ab2_dist_matrix>(h, [](ab2_dist_matrix* m) { ab2_dist_matrix_destroy(m); });
    ab2_dist_info info{};
    ab2_dist_matrix_get_info(h, &info);
    m_n = info.local_rows;
  }
  int rows() const { return m_n; }
  ab2_dist_matrix* handle() const { return m_h.get(); }
  const ab2_matrix* local() const {
    const ab2_matrix* l = nullptr;
    ab2_dist_matrix_local(m_h.get(), &l);
    return l;
  }
  const Context& context() const { return m_ctx; }
  const Comm& comm() const { return m_comm; }

 private:
  Context m_ctx;
  Comm m_comm;
  std::shared_ptr<ab2_dist_matrix> m_h;
  int m_n = 0;
};

class DistAlgebra {
 public:
  typedef DistMatrix Matrix;
  typedef B200::Vector Vector;
  typedef double ValueType;

  struct ResourceType {
    const DistMatrix* A;
  };

  struct NullValueException {
    std::string which;
    explicit NullValueException(std::string const& w) : which(w) {}
  };

  // SimpleCSRInternalLinearAlgebra's Future: a value holder, computed at once
  // (the distributed dot returns to the host anyway).
  template <typename T>
  class Future {
   public:
    explicit Future(T& value) : m_value(value) {}
    T& operator()() { return m_value; }
    T get() { return m_value; }

   private:
    T& m_value;
  };
  typedef Future<double> FutureType;

  DistAlgebra(const Context& ctx, const Comm& comm) : m_ctx(ctx), m_comm(comm) {}
  const Context& context() const { return m_ctx; }

  static ResourceType resource(Matrix const& A) { return ResourceType{&A}; }

  // Vectors of the rank's rows with room for the ghosts, so that any of
  // them can be multiplied (the reference resizes x before the exchange).
  void allocate(ResourceType const& r, Vector& v) const {
    ab2_vector* h = nullptr;
    chk(ab2_dist_vector_create(m_ctx.handle(), r.A->handle(), &h), "ab2_dist_vector_create");
    v.adopt(m_ctx, h, r.A->rows());
  }
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

  // ------------------------------------------------------------ BLAS-1 on the local rows
  void copy(Vector const& x, Vector& y) const { chk(ab2_copy(h(), x.handle(), y.handle()), "ab2_copy"); }
  void axpy(double a, Vector const& x, Vector& y) const { chk(ab2_axpy(h(), a, x.handle(), y.handle()), "ab2_axpy"); }
  void aypx(double a, Vector& y, Vector const& x) const { chk(ab2_aypx(h(), a, y.handle(), x.handle()), "ab2_aypx"); }
  void scal(double a, Vector& x) const { chk(ab2_scal(h(), a, x.handle()), "ab2_scal"); }
  void pointwiseMult(Vector const& x, Vector const& y, Vector& w) const {
    chk(ab2_pointwise_mult(h(), x.handle(), y.handle(), w.handle()), "ab2_pointwise_mult");
  }
  void assign(Vector& x, double a) const { chk(ab2_assign(h(), x.handle(), a), "ab2_assign"); }
  // x_i = f(i) over the rank's rows, in index order (each rank's generator
  // runs from its own start, as on every MPI rank of the reference).
  template <typename LambdaT>
  void assign(Vector& x, LambdaT const& f) const {
    std::vector<double> v((std::size_t)x.size());
    for (std::size_t i = 0; i < v.size(); ++i) v[i] = f(i);
    x.upload(v.data());
  }
  void reciprocal(Vector& x) const { chk(ab2_reciprocal(h(), x.handle()), "ab2_reciprocal"); }

  // ------------------------------------------------------------ reductions over the ranks
  double dot(Vector const& x, Vector const& y) const {
    double r = 0.0;
    chk(ab2_dist_dot(h(), m_comm.handle(), x.handle(), y.handle(), &r), "ab2_dist_dot");
    return r;
  }
  void dot(Vector const& x, Vector const& y, FutureType& f) const { f() = dot(x, y); }
  double norm1(Vector const& x) const {
    double r = 0.0;
    chk(ab2_dist_norm1(h(), m_comm.handle(), x.handle(), &r), "ab2_dist_norm1");
    return r;
  }
  double norm2(Vector const& x) const {
    double r = 0.0;
    chk(ab2_dist_norm2(h(), m_comm.handle(), x.handle(), &r), "ab2_dist_norm2");
    return r;
  }

  // ------------------------------------------------------------ matrix
  void mult(Matrix const& A, Vector const& x, Vector& y) const {
    chk(ab2_dist_mult(h(), A.handle(), x.handle(), y.handle()), "ab2_dist_mult");
  }
  void computeInvDiag(Matrix const& A, Vector& d) const {
    chk(ab2_compute_inv_diag(h(), A.local(), d.handle()), "ab2_compute_inv_diag");
  }
  void multInvDiag(Matrix const& A, Vector& y) const {
    chk(ab2_mult_inv_diag(h(), A.local(), y.handle()), "ab2_mult_inv_diag");
  }
  void diagonal(Matrix const& A, Vector& d) const { chk(ab2_diagonal(h(), A.local(), d.handle()), "ab2_diagonal"); }

  template <typename PrecondT>
  void exec(PrecondT& precond, Vector const& x, Vector& y) {
    precond.solve(*this, x, y);
  }

 private:
  ab2_context* h() const { return m_ctx.handle(); }
  void chk(int rc, const char* what) const { m_ctx.check(rc, what); }
  Context m_ctx;
  Comm m_comm;
};

// Block-Jacobi ILU(0) on the rank's rows with the interface of
// ILU0Preconditioner.h:273-323; the factorisation is the reference's parallel
// branch (ILU0Preconditioner.h:93-119), the sweeps its parallel solveL/solveU.
template <typename AlgebraT = DistAlgebra>
class DistILU0Preconditioner {
 public:
  typedef AlgebraT AlgebraType;
  typedef typename AlgebraType::Matrix MatrixType;
  typedef typename AlgebraType::Vector VectorType;
  typedef typename MatrixType::ValueType ValueType;

  template <typename TraceT = void>
  DistILU0Preconditioner(AlgebraType& algebra, MatrixType const& matrix, TraceT* = nullptr,
                         int schedule = AB2_ILU_AUTO)
      : m_algebra(algebra), m_matrix(matrix), m_schedule(schedule) {}

  void init() {
    ab2_precond_options o{};
    o.kind = AB2_PC_ILU0;
    o.ilu_schedule = m_schedule;
    ab2_precond* p = nullptr;
    const Context& ctx = m_algebra.context();
    ctx.check(ab2_dist_precond_create(ctx.handle(), m_matrix.handle(), &o, &p), "ab2_dist_precond_create");
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

}  // namespace B200
}  // namespace Alien
