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
// CG + Diag has a second, scaled form (AB2_MIXED_JACOBI_SCALED): Jacobi-PCG
// on A is plain CG on S A S with S = diag(1/sqrt(a_ii)), so the inner solve
// runs on that unit-diagonal operator -- three FP32 bands on A's 7-point
// grid, s_r = 1/sqrt(a_rr) and each upper value (a_rc s_r) s_c rounded once,
// the lower values read from the neighbours' upper bands -- with no
// preconditioner vector and no z: r32 = float((r / ||r||) s) on the way in,
// x += ||r|| (s d) on the way out.  The inner stop test keeps measuring the
// unscaled residual: it sums (r_i float(a_ii)) r_i, which is ||r||^2 before the
// scaling (with the scaled residual's own norm the inner solves would stop
// elsewhere: on the 192^3 heterogeneous system that took twice the
// iterations).  Per inner iteration it moves 3 bands and 11 vectors of 4
// bytes (56 bytes per row) against 4 bands and 12 vectors (64 bytes) for the
// plain FP32 form on the same bands.
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

// r32 = float(r / ||r||), ||r||^2 read from the device; with sc (the scaled
// Jacobi form) r32 = float((r / ||r||) sc).
__global__ void k_refine_scale(int n, const double* __restrict__ r, const double* __restrict__ rr,
                               const double* __restrict__ sc, float* __restrict__ r32) {
  const double s = 1.0 / sqrt(*rr);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    r32[i] = sc ? (float)((r[i] * s) * sc[i]) : (float)(r[i] * s);
}

// x += ||r|| d; with sc, x += ||r|| (sc d).
__global__ void k_refine_update(int n, const float* __restrict__ d, const double* __restrict__ rr,
                                const double* __restrict__ sc, double* __restrict__ x) {
  const double s = sqrt(*rr);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = fma(s, sc ? (double)d[i] * sc[i] : (double)d[i], x[i]);
}

// The scaled Jacobi operator from A's symmetric bands (D, Ux, Uy, Uz):
// sc_r = 1/sqrt(a_rr); hat_b[r] = float((u_b[r] sc_r) sc_{r+s_b}) for the three
// upper neighbours inside the grid, 0 outside; w32 = float(a_rr), the inner
// stop test's weight.  bad |= 1 where a_rr is not positive and finite (the
// form does not apply).
__global__ void k_scaled_bands(int n, int nx, int ny, int nz, const double* __restrict__ bands,
                               double* __restrict__ sc, float* __restrict__ hat, float* __restrict__ w32, int* bad) {
  const size_t N = (size_t)n;
  const long long sz = (long long)nx * ny;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int i = r % nx, j = (r / nx) % ny, k = (int)(r / sz);
    const double d = bands[r];
    if (!(d > 0.0) || !isfinite(d)) atomicOr(bad, 1);
    const double sr = 1.0 / sqrt(d);
    sc[r] = sr;
    w32[r] = (float)d;
    const bool in[3] = {i < nx - 1, j < ny - 1, k < nz - 1};
    const long long off[3] = {1, nx, sz};
    for (int b = 0; b < 3; ++b) {
      float h = 0.0f;
      if (in[b]) {
        const double sn = 1.0 / sqrt(bands[r + off[b]]);
        h = (float)((bands[(size_t)(b + 1) * N + r] * sr) * sn);
      }
      hat[(size_t)b * N + r] = h;
    }
  }
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
  // scaled Jacobi form: sc = 1/sqrt(a_ii) (FP64), the operator's three FP32 upper bands
  bool scaled = false;
  double* d_sc = nullptr;
  float* d_hat = nullptr;
  float* d_w32 = nullptr;  // float(a_ii): the inner stop test measures the unscaled residual
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
  o->jacobi_form = AB2_MIXED_JACOBI_AUTO;
}

int ab2_mixed_create(ab2_context* ctx, const ab2_matrix* A, const ab2_mixed_options* o, ab2_mixed** out) {
  if (!ctx || !A || !o || !out) return AB2_ERR_BAD_ARG;
  if (o->solver != AB2_SOLVER_CG && o->solver != AB2_SOLVER_BICGSTAB) return AB2_ERR_BAD_ARG;
  if (o->max_outer < 0 || o->inner_max_iter < 0 || !(o->tol >= 0) || !(o->inner_tol > 0 && o->inner_tol < 1))
    return AB2_ERR_BAD_ARG;
  if (o->jacobi_form < AB2_MIXED_JACOBI_AUTO || o->jacobi_form > AB2_MIXED_JACOBI_SCALED) return AB2_ERR_BAD_ARG;
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
    // The scaled Jacobi form where asked for or (AUTO) where the matrix allows it.
    const bool jacobi = o->solver == AB2_SOLVER_CG && o->precond == AB2_PC_DIAG;
    const bool bands_ok = A->st_bands == 4 && A->d_st_v != nullptr;
    if (jacobi && o->jacobi_form == AB2_MIXED_JACOBI_SCALED && !bands_ok)
      throw Error{AB2_ERR_BAD_ARG, "scaled Jacobi form: needs a bit-symmetric 7-point matrix kept as bands "
                                   "(AB2_FMT_STENCIL)"};
    if (jacobi && bands_ok && o->jacobi_form != AB2_MIXED_JACOBI_PLAIN) {
      const size_t n = (size_t)A->n;
      M->d_sc = dev_alloc<double>(ctx, n);
      M->d_hat = dev_alloc<float>(ctx, 3 * n);
      M->d_w32 = dev_alloc<float>(ctx, n);
      int* d_bad = dev_alloc<int>(ctx, 1);
      AB2_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), ctx->stream));
      k_scaled_bands<<<grid_for(A->n), kThreads, 0, ctx->stream>>>(A->n, A->st_nx, A->st_ny, A->st_nz, A->d_st_v,
                                                                   M->d_sc, M->d_hat, M->d_w32, d_bad);
      check_launch(ctx, "scaled_bands");
      int bad = 0;
      AB2_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
      AB2_CUDA(cudaStreamSynchronize(ctx->stream));
      dev_free(ctx, d_bad);
      if (bad && o->jacobi_form == AB2_MIXED_JACOBI_SCALED)
        throw Error{AB2_ERR_BAD_ARG, "scaled Jacobi form: the diagonal must be positive"};
      M->scaled = !bad;
      if (!M->scaled) {
        dev_free(ctx, M->d_sc);
        dev_free(ctx, M->d_hat);
        dev_free(ctx, M->d_w32);
        M->d_sc = nullptr;
        M->d_hat = nullptr;
        M->d_w32 = nullptr;
      }
    }
    ab2_precond_options po;
    po.kind = M->scaled ? AB2_PC_NONE : o->precond;
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
    if (M->scaled) {
      M->eng.unit_bands = M->d_hat;
      M->eng.stop_weight = M->d_w32;
    }
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
        k_refine_scale<<<ge, kThreads, 0, ctx->stream>>>(n, M->d_r, M->d_rr, M->d_sc, M->d_r32);
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
        k_refine_update<<<ge, kThreads, 0, ctx->stream>>>(n, M->d_d32, M->d_rr, M->d_sc, x->d);
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
    status->jacobi_scaled = M->scaled ? 1 : 0;
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
    dev_free(M->ctx, M->d_sc);
    dev_free(M->ctx, M->d_hat);
    dev_free(M->ctx, M->d_w32);
  }
  if (M->ev0) cudaEventDestroy(M->ev0);
  if (M->ev1) cudaEventDestroy(M->ev1);
  if (M->ctx) ctx_release(M->ctx);
  delete M;
  return AB2_OK;
}

}  // extern "C"
