// mixed.cu -- mixed-precision solver: FP32 Krylov inside FP64 iterative
// refinement.  No counterpart in the reference (its solvers run in the
// matrix's value type only); the building blocks are the reference's own CG /
// BiCGStab and preconditioners, instantiated in float (krylov.cu, precond.cu).
//
// One refinement step:
//   r   = b - A x                  FP64 values, FP64 accumulation; r.r in the same pass
//   stop if ||r|| / ||b|| < tol    the true residual, in FP64
//   r32 = float(r / ||r||)         scaled so the inner problem has a unit right-hand side
//   A32 d = r32                    FP32 CG/BiCGStab + FP32 preconditioner, from d = 0,
//                                  to ||r32 - A32 d|| < inner_tol (recursive residual)
//   x  += ||r|| * double(d)        FP64 update
// The FP32 matrix is the FP64 matrix rounded (AB2_FMT_F32); the FP32
// preconditioner is the FP64 set-up rounded (the ILU(0) factor is computed in
// FP64, bit-identical to the reference's, then rounded).
//
// Stops without success when max_outer steps are used or a step fails to
// reduce the true residual (the FP32 inner solve can no longer help).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ab2_internal.cuh"
#include "krylov.cuh"
#include "precond.cuh"
#include "reduce.cuh"
#include "spmv_view.cuh"

namespace ab2 {
namespace {

// r = b - A x and r.r (FP64).
template <class View>
__global__ void __launch_bounds__(kThreads) k_refine_residual(int n, View A, const double* __restrict__ x,
                                                              const double* __restrict__ b, double* __restrict__ r,
                                                              RedSlot red) {
  double acc[1] = {0.0};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const double rv = b[row] - A.row(row, x);
    r[row] = rv;
    acc[0] = fma(rv, rv, acc[0]);
  }
  grid_reduce<1>(acc, red.partials, red.counter, red.result);
}

// r32 = float(r / ||r||), ||r||^2 read from the device.
__global__ void k_refine_scale(int n, const double* __restrict__ r, const double* __restrict__ rr,
                               float* __restrict__ r32) {
  const double s = 1.0 / sqrt(*rr);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) r32[i] = (float)(r[i] * s);
}

// x += ||r|| d.
__global__ void k_refine_update(int n, const float* __restrict__ d, const double* __restrict__ rr,
                                double* __restrict__ x) {
  const double s = sqrt(*rr);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = fma(s, (double)d[i], x[i]);
}

}  // namespace
}  // namespace ab2

using namespace ab2;

struct ab2_mixed {
  ab2_context* ctx = nullptr;
  const ab2_matrix* A = nullptr;
  ab2_mixed_options opts{};
  ab2_precond* pc = nullptr;
  Krylov<float> eng;
  double* d_r = nullptr;   // FP64 residual
  float* d_r32 = nullptr;  // scaled FP32 right-hand side of the inner solve
  float* d_d32 = nullptr;  // FP32 correction
  double* d_rr = nullptr;  // ||r||^2 of the current step (device)
  std::vector<double> history;
  double setup_ms = 0, solve_ms = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

extern "C" {

void ab2_mixed_options_default(ab2_mixed_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->solver = AB2_SOLVER_CG;
  o->precond = AB2_PC_DIAG;
  o->tol = 1e-8;
  o->max_outer = 20;
  o->inner_tol = 1e-4;
  o->inner_max_iter = 1000;
  o->poly_factor = 0.0;
  o->poly_order = 3;
  o->poly_factor_max_iter = 20;
  o->spmv_variant = AB2_SPMV_AUTO;
  o->use_graph = 1;
  o->filu_solver_iter = 3;
}

int ab2_mixed_create(ab2_context* ctx, const ab2_matrix* A, const ab2_mixed_options* o, ab2_mixed** out) {
  if (!ctx || !A || !o || !out) return AB2_ERR_BAD_ARG;
  if (o->solver != AB2_SOLVER_CG && o->solver != AB2_SOLVER_BICGSTAB) return AB2_ERR_BAD_ARG;
  if (o->max_outer < 0 || o->inner_max_iter < 0 || !(o->tol >= 0) || !(o->inner_tol > 0 && o->inner_tol < 1))
    return AB2_ERR_BAD_ARG;
  *out = nullptr;
  if (!A->d_v32) {
    ctx->last_error = "mixed-precision solver needs the matrix's FP32 values (create it with AB2_FMT_F32)";
    return AB2_ERR_BAD_ARG;
  }
  ab2_mixed* M = new (std::nothrow) ab2_mixed();
  if (!M) return AB2_ERR_OOM;
  M->ctx = ctx_retain(ctx);
  int rc = guard(ctx, [&] {
    M->A = A;
    M->opts = *o;
    AB2_CUDA(cudaEventCreate(&M->ev0));
    AB2_CUDA(cudaEventCreate(&M->ev1));
    AB2_CUDA(cudaEventRecord(M->ev0, ctx->stream));
    ab2_precond_options po;
    po.kind = o->precond;
    po.poly_factor = o->poly_factor;
    po.poly_order = o->poly_order;
    po.poly_factor_max_iter = o->poly_factor_max_iter;
    po.ilu_schedule = o->ilu_schedule;
    po.cheb_saad = o->cheb_saad;
    po.cheb_lanczos = o->cheb_lanczos;
    po.filu_factor_iter = o->filu_factor_iter;
    po.filu_solver_iter = o->filu_solver_iter;
    po.filu_tol = o->filu_tol;
    int prc = ab2_precond_create(ctx, A, &po, &M->pc);
    if (prc != AB2_OK) throw Error{prc, ctx->last_error};
    M->pc->variant = o->spmv_variant;
    pc_enable_f32(ctx, M->pc);
    M->eng.init(ctx, A, M->pc, o->solver, o->spmv_variant, o->use_graph, o->inner_max_iter);
    const size_t n = (size_t)A->n;
    M->d_r = dev_alloc<double>(ctx, n);
    M->d_r32 = dev_alloc<float>(ctx, n);
    M->d_d32 = dev_alloc<float>(ctx, n);
    M->d_rr = dev_alloc<double>(ctx, 1);
    AB2_CUDA(cudaEventRecord(M->ev1, ctx->stream));
    AB2_CUDA(cudaEventSynchronize(M->ev1));
    float ms = 0;
    AB2_CUDA(cudaEventElapsedTime(&ms, M->ev0, M->ev1));
    M->setup_ms = ms;
  });
  if (rc != AB2_OK) {
    ab2_mixed_destroy(M);
    return rc;
  }
  *out = M;
  return AB2_OK;
}

int ab2_mixed_solve(ab2_mixed* M, const ab2_vector* b, ab2_vector* x, ab2_mixed_status* status) {
  if (!M || !b || !x || !status || b->n != M->A->n || x->n != M->A->n) return AB2_ERR_BAD_ARG;
  ab2_context* ctx = M->ctx;
  PhaseScope phase_scope(ctx, "MIXED-SOLVE");
  std::memset(status, 0, sizeof(*status));
  M->history.clear();
  return guard(ctx, [&] {
    const ab2_mixed_options& o = M->opts;
    const ab2_matrix* A = M->A;
    const int n = A->n;
    const int g = red_grid(ctx, n);
    const int ge = grid_for(n);
    AB2_CUDA(cudaEventRecord(M->ev0, ctx->stream));
    op_dot(ctx, n, b->d, b->d, M->d_rr, 0);
    const double bb = read_scalar(ctx, M->d_rr);
    int outer = 0, inner = 0, error = AB2_OK;
    bool ok = false;
    double res = 0.0;
    if (bb == 0.0) {
      ok = true;  // null right-hand side: nothing to do (Iteration::nullRhs)
    } else {
      const double nb = std::sqrt(bb);
      double prev = INFINITY;
      for (;;) {
        RedSlot red = red_slot(ctx, 5);
        with_view<double>(A, o.spmv_variant, [&](auto view) {
          k_refine_residual<<<g, kThreads, 0, ctx->stream>>>(n, view, x->d, b->d, M->d_r, red);
        });
        check_launch(ctx, "refine_residual");
        AB2_CUDA(cudaMemcpyAsync(M->d_rr, red.result, sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        const double rr = read_scalar(ctx, M->d_rr);
        res = std::sqrt(rr) / nb;
        M->history.push_back(res);
        if (res < o.tol) {
          ok = true;
          break;
        }
        if (outer >= o.max_outer || !(res < prev) || rr == 0.0) {
          error = AB2_ERR_NOT_CONVERGED;
          break;
        }
        prev = res;
        k_refine_scale<<<ge, kThreads, 0, ctx->stream>>>(n, M->d_r, M->d_rr, M->d_r32);
        check_launch(ctx, "refine_scale");
        AB2_CUDA(cudaMemsetAsync(M->d_d32, 0, sizeof(float) * (size_t)n, ctx->stream));
        M->eng.solve(M->d_r32, M->d_d32, (float)o.inner_tol, o.inner_max_iter);
        const SolveStateT<float>& st = *M->eng.h_st;
        inner += st.iter;
        if (pc_error(ctx, M->pc)) {
          pc_reset(ctx, M->pc);
          error = AB2_ERR_TIMEOUT;
          break;
        }
        if (st.error && st.iter == 0) {  // the inner solve could not start: nothing to add
          error = st.error;
          break;
        }
        k_refine_update<<<ge, kThreads, 0, ctx->stream>>>(n, M->d_d32, M->d_rr, x->d);
        check_launch(ctx, "refine_update");
        ++outer;
      }
    }
    AB2_CUDA(cudaEventRecord(M->ev1, ctx->stream));
    AB2_CUDA(cudaEventSynchronize(M->ev1));
    float ms = 0;
    AB2_CUDA(cudaEventElapsedTime(&ms, M->ev0, M->ev1));
    M->solve_ms = ms;
    status->succeeded = ok ? 1 : 0;
    status->outer_iterations = outer;
    status->inner_iterations = inner;
    status->error = ok ? AB2_OK : error;
    status->true_residual = res;
    status->setup_ms = M->setup_ms;
    status->solve_ms = M->solve_ms;
  });
}

int ab2_mixed_history(const ab2_mixed* M, double* res, int cap, int* len) {
  if (!M || !len || (cap > 0 && !res)) return AB2_ERR_BAD_ARG;
  *len = (int)M->history.size();
  const int m = std::min(cap, *len);
  for (int i = 0; i < m; ++i) res[i] = M->history[(size_t)i];
  return AB2_OK;
}

int ab2_mixed_destroy(ab2_mixed* M) {
  if (!M) return AB2_ERR_BAD_ARG;
  if (M->ctx) ctx_quiesce(M->ctx);
  M->eng.release();
  if (M->pc) ab2_precond_destroy(M->pc);
  if (M->ctx) {
    dev_free(M->ctx, M->d_r);
    dev_free(M->ctx, M->d_r32);
    dev_free(M->ctx, M->d_d32);
    dev_free(M->ctx, M->d_rr);
  }
  if (M->ev0) cudaEventDestroy(M->ev0);
  if (M->ev1) cudaEventDestroy(M->ev1);
  if (M->ctx) ctx_release(M->ctx);
  delete M;
  return AB2_OK;
}

}  // extern "C"
