// krylov.cuh -- the device-resident Krylov engine shared by the FP64 solver
// (krylov.cu) and the FP32 inner solves of the mixed-precision solver (mixed.cu).
#pragma once

#include <cuda_runtime.h>

#include "ab2_internal.cuh"

struct ab2_precond;

namespace ab2 {

// Device-resident solver state (one per engine).
template <class T>
struct SolveStateT {
  T nrm2_b, crit;
  T rr;      // last value the stop test compared
  T rho, rho1, den, alpha, beta, omega;
  T rr_r;    // BiCGStab: r.r of the current r (the beta==0 branch of the first step tests r)
  T* x;
  const T* b;
  T* hist;
  int hist_cap, hist_len;
  int iter, max_iter;
  int first, done, converged, error, breakdown;
  int exit_fixup;  // BiCGStab exits on ||s||: x += alpha phat still to do
  int x_pending;   // CG with the deferred x update: x += alpha p still owed
  int bodies;      // loop bodies executed (for launch accounting)
};

using SolveState = SolveStateT<double>;

// One CG or BiCGStab engine over value type T (double or float): work
// vectors, state, stop-test history and the loop graph, reused by every solve.
template <class T>
struct Krylov {
  ab2_context* ctx = nullptr;
  const ab2_matrix* A = nullptr;
  const ab2_precond* pc = nullptr;  // applied in T
  int solver = AB2_SOLVER_CG;
  int variant = AB2_SPMV_AUTO;
  int use_graph = 1;
  T* w[8] = {};  // CG: r z p q (+ p' for the two-kernel body) ; BiCGStab: r r0 p phat v s shat t
  SolveStateT<T>* d_st = nullptr;
  SolveStateT<T>* h_st = nullptr;  // pinned copy, valid after solve()
  T* d_hist = nullptr;
  int hist_cap = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphConditionalHandle handle = 0;
  int body_launches = 0;
  bool fused_diag = false;  // CG with Diag or no preconditioner: the two-kernel body
  // Operator override (set before init): the symmetric unit-diagonal 7-point
  // operator kept as three upper bands on A's grid (the mixed solver's
  // symmetrically scaled Jacobi form), used in place of A's own values.
  const T* unit_bands = nullptr;
  // Stop-test weight (CG with no preconditioner only): the stop test and b.b
  // sum (v_i w_i) v_i -- with w = the diagonal, the norm of the residual
  // before the symmetric scaling.
  const T* stop_weight = nullptr;

  // Allocates the work vectors (max_iter sizes the history) and builds the graph.
  void init(ab2_context* c, const ab2_matrix* a, const ab2_precond* p, int solver_kind, int spmv_variant, int graph_loop,
            int max_iter);
  // Solves A x = b from the x given, to r.r < tol^2 b.b or max_iter
  // iterations (max_iter <= the init value).  Synchronises; h_st holds the
  // final state and ctx->launches counts every kernel.
  void solve(const T* b, T* x, T tol, int max_iter);
  void release();

 private:
  int enqueue_body(cudaGraphConditionalHandle h, int graph_loop);
  template <class F>
  void with_op(F&& f) const;  // f(view of the operator): unit_bands or A in `variant`
  void build_graph();
  const T* diag_inv() const;  // 1/a_ii of a Diag preconditioner in T, else null
};

}  // namespace ab2
