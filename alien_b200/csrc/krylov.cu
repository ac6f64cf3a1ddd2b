// krylov.cu -- CG and BiCGStab with the whole iteration on the device.
//
// The loop bodies follow the reference templates statement by statement:
//   CG        src/core/alien/expression/krylov/CG.h:59-150
//   BiCGStab  src/core/alien/expression/krylov/BiCGStab.h:152-300
//   stop test src/core/alien/expression/krylov/Iteration.h:44-90 (r.r < tol^2 b.b,
//             recursive residual; iter >= max_iter stops without success)
// with the same vector updates (one fma each, same operand order), the same
// breakdown tests (NullValueException "alpha"/"beta"/"rho" becomes
// AB2_ERR_BREAKDOWN + AB2_BREAKDOWN_*), and the same iteration counting
// (BiCGStab's mid-iteration exit on ||s|| does not count, CG.h's first step
// does).
//
// What changes is where the scalars live.  Every dot product is a
// deterministic single-pass grid reduction whose last block also runs the
// scalar part of the algorithm (alpha, beta, omega, the stop test, breakdowns)
// and writes it to a device-resident state block; the next kernel reads its
// scalars from there.  No value crosses to the host inside the loop.  The loop
// itself is a CUDA graph: a conditional WHILE node whose body holds one
// iteration's kernels; the control kernel clears the condition when the solve
// is over.  (use_graph = 0 runs the same kernels from a host loop instead.)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "ab2_internal.cuh"
#include "precond.cuh"
#include "reduce.cuh"
#include "spmv_view.cuh"

namespace ab2 {

// Device-resident solver state (one per solver object).
struct SolveState {
  double nrm2_b, crit;
  double rr;      // last value the stop test compared
  double rho, rho1, den, alpha, beta, omega;
  double rr_r;    // BiCGStab: r.r of the current r (the beta==0 branch of the first step tests r)
  double* x;
  const double* b;
  double* hist;
  int hist_cap, hist_len;
  int iter, max_iter;
  int first, done, converged, error, breakdown;
  int exit_fixup;  // BiCGStab exits on ||s||: x += alpha phat still to do
  int bodies;      // loop bodies executed (for launch accounting)
};

namespace {

constexpr int kCtlThreads = 256;

__device__ __forceinline__ void record(SolveState* st, double v) {
  if (st->hist_len < st->hist_cap) st->hist[st->hist_len] = v;
  st->hist_len += 1;
}

// Iteration::stop(r) with the dot product already computed.
__device__ __forceinline__ bool stop_test(SolveState* st, double dot_rr) {
  if (st->iter >= st->max_iter) return true;
  st->rr = dot_rr;
  record(st, dot_rr);
  st->converged = dot_rr < st->crit ? 1 : 0;
  return st->converged != 0;
}

__device__ __forceinline__ void set_loop(cudaGraphConditionalHandle h, int use_graph, int go) {
  if (use_graph) cudaGraphSetConditional(h, go ? 1u : 0u);
}

static_assert(kCtlThreads == kThreads, "fused reductions use the standalone reduction tree");
int fused_grid(ab2_context* ctx, int n) { return red_grid(ctx, n); }

__global__ void k_state_init(SolveState* st, double tol, int max_iter, double* x, const double* b, double* hist,
                             int hist_cap) {
  st->crit = tol * tol * st->nrm2_b;
  st->rr = st->crit + 1;
  st->x = x;
  st->b = b;
  st->hist = hist;
  st->hist_cap = hist_cap;
  st->hist_len = 0;
  st->iter = 0;
  st->max_iter = max_iter;
  st->first = 1;
  st->converged = st->nrm2_b == 0 ? 1 : 0;
  st->done = st->converged;
  st->error = 0;
  st->breakdown = 0;
  st->exit_fixup = 0;
  st->bodies = 0;
  st->rho = st->rho1 = st->den = st->alpha = st->beta = st->omega = st->rr_r = 0;
}

// r = b - A x (copy b, mult A x, axpy -1).  With r0 != nullptr (BiCGStab):
// also r0 = r and rho1 = r.r0.
template <class View>
__global__ void __launch_bounds__(kCtlThreads) k_residual(int n, View A, SolveState* st, double* r, double* r0,
                                                          RedSlot red) {
  const double* x = st->x;
  const double* b = st->b;
  double acc[1] = {0.0};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const double ax = A.row(row, x);
    const double rv = fma(-1.0, ax, b[row]);
    r[row] = rv;
    if (r0) {
      r0[row] = rv;
      acc[0] = fma(rv, rv, acc[0]);
    }
  }
  if (grid_reduce<1>(acc, red.partials, red.counter, red.result)) {
    if (r0) st->rho1 = red.result[0];
  }
}

// ------------------------------------------------------------------ CG
// rho1 = r.z ; beta = rho1/rho (CG.h:117-118, the code names it alpha)
__global__ void __launch_bounds__(kCtlThreads) k_cg_rz(int n, const double* __restrict__ r, const double* __restrict__ z,
                                                       SolveState* st, RedSlot red) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[0] = fma(r[i], z[i], acc[0]);
  if (grid_reduce<1>(acc, red.partials, red.counter, red.result)) {
    st->rho1 = red.result[0];
    st->beta = st->first ? 0.0 : st->rho1 / st->rho;
  }
}

// p = z (first step, CG.h:89) or z += beta p ; p = z (CG.h:119-120)
__global__ void k_cg_p(int n, const double* __restrict__ z, double* __restrict__ p, const SolveState* st) {
  const double beta = st->beta;
  const int first = st->first;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = first ? z[i] : fma(beta, p[i], z[i]);
}

// q = A p ; den = q.p
template <class View>
__global__ void __launch_bounds__(kCtlThreads) k_cg_spmv(int n, View A, const double* __restrict__ p,
                                                         double* __restrict__ q, SolveState* st, RedSlot red) {
  double acc[1] = {0.0};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const double qv = A.row(row, p);
    q[row] = qv;
    acc[0] = fma(qv, p[row], acc[0]);
  }
  if (grid_reduce<1>(acc, red.partials, red.counter, red.result)) st->den = red.result[0];
}

// alpha = rho1/den ; x += alpha p ; r -= alpha q ; then the loop's stop test on r.
__global__ void __launch_bounds__(kCtlThreads) k_cg_update(int n, const double* __restrict__ p,
                                                           const double* __restrict__ q, double* __restrict__ r,
                                                           SolveState* st, RedSlot red, cudaGraphConditionalHandle h,
                                                           int use_graph) {
  if (st->done) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_loop(h, use_graph, 0);
    return;
  }
  const double den = st->den;
  const bool ok = den != 0;
  const double alpha = ok ? st->rho1 / den : 0.0;
  double* x = st->x;
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double rv = r[i];
    if (ok) {
      x[i] = fma(alpha, p[i], x[i]);
      rv = fma(-alpha, q[i], rv);
      r[i] = rv;
    }
    acc[0] = fma(rv, rv, acc[0]);
  }
  if (grid_reduce<1>(acc, red.partials, red.counter, red.result)) {
    const double rr = red.result[0];
    st->bodies += 1;
    if (!ok) {
      // CG.h:96-104 / 131-139: converged after all, or breakdown "alpha"
      if (stop_test(st, rr)) st->iter += 1;
      else {
        st->error = AB2_ERR_BREAKDOWN;
        st->breakdown = AB2_BREAKDOWN_ALPHA;
      }
      st->done = 1;
    } else {
      st->alpha = alpha;
      st->rho = st->rho1;
      st->iter += 1;
      st->first = 0;
      if (stop_test(st, rr)) st->done = 1;
    }
    set_loop(h, use_graph, !st->done);
  }
}

// ------------------------------------------------------------------ BiCGStab
// p = r (first) or p = r + beta (p - omega v)  (BiCGStab.h:273-276, three BLAS-1 calls)
__global__ void k_bicg_p(int n, const double* __restrict__ r, const double* __restrict__ v, double* __restrict__ p,
                         const SolveState* st) {
  const int first = st->first;
  const double beta = st->beta, omega = st->omega;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (first) p[i] = r[i];
    else p[i] = __dadd_rn(r[i], __dmul_rn(beta, fma(-omega, v[i], p[i])));
  }
}

// v = A phat ; alpha = rho1 / (v.r0), breakdown "alpha" on zero
template <class View>
__global__ void __launch_bounds__(kCtlThreads) k_bicg_v(int n, View A, const double* __restrict__ phat,
                                                        const double* __restrict__ r0, double* __restrict__ v,
                                                        SolveState* st, RedSlot red) {
  double acc[1] = {0.0};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const double vv = A.row(row, phat);
    v[row] = vv;
    acc[0] = fma(vv, r0[row], acc[0]);
  }
  if (grid_reduce<1>(acc, red.partials, red.counter, red.result)) {
    const double d = red.result[0];
    if (d == 0) {
      st->error = AB2_ERR_BREAKDOWN;
      st->breakdown = AB2_BREAKDOWN_ALPHA;
      st->done = 1;
    } else {
      st->alpha = st->rho1 / d;
    }
  }
}

// s = r - alpha v ; stop test on s (exit with x += alpha phat) ; also r.r for the first step
__global__ void __launch_bounds__(kCtlThreads) k_bicg_s(int n, const double* __restrict__ r, const double* __restrict__ v,
                                                        double* __restrict__ s, SolveState* st, RedSlot red) {
  const bool live = !st->done;
  const double alpha = st->alpha;
  double acc[2] = {0.0, 0.0};
  if (live) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      const double rv = r[i];
      const double sv = fma(-alpha, v[i], rv);
      s[i] = sv;
      acc[0] = fma(sv, sv, acc[0]);
      acc[1] = fma(rv, rv, acc[1]);
    }
  }
  if (grid_reduce<2>(acc, red.partials, red.counter, red.result)) {
    if (live) {
      st->rr_r = red.result[1];
      if (stop_test(st, red.result[0])) {
        if (st->first) st->iter += 1;  // BiCGStab.h:194-199 counts this exit, :259-263 does not
        st->exit_fixup = 1;
        st->done = 1;
      }
    }
  }
}

// t = A shat ; omega = t.s / t.t, beta==0 handling (BiCGStab.h:202-216, 266-282)
template <class View>
__global__ void __launch_bounds__(kCtlThreads) k_bicg_t(int n, View A, const double* __restrict__ shat,
                                                        const double* __restrict__ s, double* __restrict__ t,
                                                        SolveState* st, RedSlot red) {
  const bool live = !st->done;
  double acc[2] = {0.0, 0.0};
  if (live) {
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
      const double tv = A.row(row, shat);
      t[row] = tv;
      acc[0] = fma(tv, s[row], acc[0]);
      acc[1] = fma(tv, tv, acc[1]);
    }
  }
  if (grid_reduce<2>(acc, red.partials, red.counter, red.result)) {
    if (live) {
      const double ts = red.result[0], tt = red.result[1];
      if (tt == 0) {
        // first step: stop(r); later steps: stop(s) -- s.s is the value just tested
        const double v = st->first ? st->rr_r : st->rr;
        if (stop_test(st, v)) {
          if (st->first) st->iter += 1;
          st->exit_fixup = 1;
        } else {
          st->error = AB2_ERR_BREAKDOWN;
          st->breakdown = AB2_BREAKDOWN_BETA;
        }
        st->done = 1;
      } else {
        st->omega = ts / tt;
      }
    }
  }
}

// x += omega shat ; x += alpha phat ; r = s - omega t ; loop stop test on r ;
// rho1 = r.r0 ; beta = (rho1/rho)(alpha/omega) ; breakdown "rho" on rho == 0.
__global__ void __launch_bounds__(kCtlThreads) k_bicg_update(int n, const double* __restrict__ shat,
                                                             const double* __restrict__ phat, const double* __restrict__ s,
                                                             const double* __restrict__ t, const double* __restrict__ r0,
                                                             double* __restrict__ r, SolveState* st, RedSlot red,
                                                             cudaGraphConditionalHandle h, int use_graph) {
  double* x = st->x;
  const int done = st->done;
  const int fix = st->exit_fixup;
  const double alpha = st->alpha, omega = st->omega;
  double acc[2] = {0.0, 0.0};
  if (done) {
    if (fix) {
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = fma(alpha, phat[i], x[i]);
    }
  } else {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      double xv = fma(omega, shat[i], x[i]);
      x[i] = fma(alpha, phat[i], xv);
      const double rv = fma(-omega, t[i], s[i]);
      r[i] = rv;
      acc[0] = fma(rv, rv, acc[0]);
      acc[1] = fma(rv, r0[i], acc[1]);
    }
  }
  if (grid_reduce<2>(acc, red.partials, red.counter, red.result)) {
    st->bodies += 1;
    if (done) {
      st->exit_fixup = 0;
    } else {
      st->rho = st->rho1;
      st->iter += 1;
      st->first = 0;
      if (stop_test(st, red.result[0])) {
        st->done = 1;
      } else {
        st->rho1 = red.result[1];
        st->beta = (st->rho1 / st->rho) * (st->alpha / st->omega);
        if (st->rho == 0) {
          st->error = AB2_ERR_BREAKDOWN;
          st->breakdown = AB2_BREAKDOWN_RHO;
          st->done = 1;
        }
      }
    }
    set_loop(h, use_graph, !st->done);
  }
}

// True residual ||b - A x||^2 into out[0], b.b into out[1].
template <class View>
__global__ void __launch_bounds__(kCtlThreads) k_true_residual(int n, View A, const double* __restrict__ x,
                                                               const double* __restrict__ b, RedSlot red) {
  double acc[2] = {0.0, 0.0};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const double rv = b[row] - A.row(row, x);
    acc[0] = fma(rv, rv, acc[0]);
    acc[1] = fma(b[row], b[row], acc[1]);
  }
  grid_reduce<2>(acc, red.partials, red.counter, red.result);
}

}  // namespace

}  // namespace ab2

using namespace ab2;

struct ab2_solver {
  ab2_context* ctx = nullptr;
  const ab2_matrix* A = nullptr;
  ab2_solver_options opts{};
  ab2_precond* pc = nullptr;
  // CG: r z p q ; BiCGStab: r r0 p phat v s shat t
  double* w[8] = {};
  SolveState* d_st = nullptr;
  SolveState* h_st = nullptr;
  double* d_hist = nullptr;
  int hist_cap = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphConditionalHandle handle = 0;
  int body_launches = 0;
  double setup_ms = 0;
  double solve_ms = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace ab2 {
namespace {

// Enqueues one loop iteration.  Returns the number of kernels it launched.
int enqueue_body(ab2_solver* S, cudaGraphConditionalHandle h, int use_graph) {
  ab2_context* ctx = S->ctx;
  const ab2_matrix* A = S->A;
  const int n = A->n;
  const int g = fused_grid(ctx, n);
  const int ge = grid_for(n);
  const long long before = ctx->launches;
  SolveState* st = S->d_st;
  if (S->opts.solver == AB2_SOLVER_CG) {
    double *r = S->w[0], *z = S->w[1], *p = S->w[2], *q = S->w[3];
    pc_apply(ctx, S->pc, r, z);
    k_cg_rz<<<g, kCtlThreads, 0, ctx->stream>>>(n, r, z, st, red_slot(ctx, 1));
    check_launch(ctx, "cg_rz");
    k_cg_p<<<ge, kThreads, 0, ctx->stream>>>(n, z, p, st);
    check_launch(ctx, "cg_p");
    with_view<double>(A, S->opts.spmv_variant, [&](auto view) {
      k_cg_spmv<<<g, kCtlThreads, 0, ctx->stream>>>(n, view, p, q, st, red_slot(ctx, 2));
    });
    check_launch(ctx, "cg_spmv");
    k_cg_update<<<g, kCtlThreads, 0, ctx->stream>>>(n, p, q, r, st, red_slot(ctx, 3), h, use_graph);
    check_launch(ctx, "cg_update");
  } else {
    double *r = S->w[0], *r0 = S->w[1], *p = S->w[2], *phat = S->w[3], *v = S->w[4], *s = S->w[5], *shat = S->w[6],
           *t = S->w[7];
    k_bicg_p<<<ge, kThreads, 0, ctx->stream>>>(n, r, v, p, st);
    check_launch(ctx, "bicg_p");
    pc_apply(ctx, S->pc, p, phat);
    with_view<double>(A, S->opts.spmv_variant, [&](auto view) {
      k_bicg_v<<<g, kCtlThreads, 0, ctx->stream>>>(n, view, phat, r0, v, st, red_slot(ctx, 1));
    });
    check_launch(ctx, "bicg_v");
    k_bicg_s<<<g, kCtlThreads, 0, ctx->stream>>>(n, r, v, s, st, red_slot(ctx, 2));
    check_launch(ctx, "bicg_s");
    pc_apply(ctx, S->pc, s, shat);
    with_view<double>(A, S->opts.spmv_variant, [&](auto view) {
      k_bicg_t<<<g, kCtlThreads, 0, ctx->stream>>>(n, view, shat, s, t, st, red_slot(ctx, 3));
    });
    check_launch(ctx, "bicg_t");
    k_bicg_update<<<g, kCtlThreads, 0, ctx->stream>>>(n, shat, phat, s, t, r0, r, st, red_slot(ctx, 4), h, use_graph);
    check_launch(ctx, "bicg_update");
  }
  return (int)(ctx->launches - before);
}

void build_graph(ab2_solver* S) {
  ab2_context* ctx = S->ctx;
  AB2_CUDA(cudaGraphCreate(&S->graph, 0));
  AB2_CUDA(cudaGraphConditionalHandleCreate(&S->handle, S->graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = S->handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  AB2_CUDA(cudaGraphAddNode(&node, S->graph, nullptr, 0, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  AB2_CUDA(cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  int launched = 0;
  try {
    launched = enqueue_body(S, S->handle, 1);
  } catch (...) {
    cudaGraph_t dummy;
    cudaStreamEndCapture(ctx->stream, &dummy);
    throw;
  }
  AB2_CUDA(cudaStreamEndCapture(ctx->stream, &body));
  ctx->launches -= launched;  // captured, not launched
  S->body_launches = launched;
  AB2_CUDA(cudaGraphInstantiate(&S->exec, S->graph, 0));
}

}  // namespace
}  // namespace ab2

extern "C" {

void ab2_solver_options_default(ab2_solver_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->solver = AB2_SOLVER_CG;
  o->precond = AB2_PC_DIAG;
  o->tol = 1e-6;
  o->max_iter = 1000;
  o->poly_factor = 0.5;
  o->poly_order = 3;
  o->poly_factor_max_iter = 10;
  o->spmv_variant = AB2_SPMV_AUTO;
  o->use_graph = 1;
}

int ab2_solver_create(ab2_context* ctx, const ab2_matrix* A, const ab2_solver_options* o, ab2_solver** out) {
  if (!ctx || !A || !o || !out) return AB2_ERR_BAD_ARG;
  if (o->solver != AB2_SOLVER_CG && o->solver != AB2_SOLVER_BICGSTAB) return AB2_ERR_BAD_ARG;
  if (o->max_iter < 0 || !(o->tol >= 0)) return AB2_ERR_BAD_ARG;
  *out = nullptr;
  ab2_solver* S = new (std::nothrow) ab2_solver();
  if (!S) return AB2_ERR_OOM;
  S->ctx = ctx_retain(ctx);
  int rc = guard(ctx, [&] {
    S->A = A;
    S->opts = *o;
    AB2_CUDA(cudaEventCreate(&S->ev0));
    AB2_CUDA(cudaEventCreate(&S->ev1));
    AB2_CUDA(cudaEventRecord(S->ev0, ctx->stream));
    ab2_precond_options po;
    po.kind = o->precond;
    po.poly_factor = o->poly_factor;
    po.poly_order = o->poly_order;
    po.poly_factor_max_iter = o->poly_factor_max_iter;
    po.ilu_schedule = o->ilu_schedule;
    po.cheb_saad = o->cheb_saad;
    po.cheb_lanczos = o->cheb_lanczos;
    int prc = ab2_precond_create(ctx, A, &po, &S->pc);
    if (prc != AB2_OK) throw Error{prc, ctx->last_error};
    S->pc->variant = o->spmv_variant;
    const int nw = o->solver == AB2_SOLVER_CG ? 4 : 8;
    for (int i = 0; i < nw; ++i) {
      S->w[i] = dev_alloc<double>(ctx, (size_t)A->n);
      AB2_CUDA(cudaMemsetAsync(S->w[i], 0, sizeof(double) * (size_t)std::max(A->n, 1), ctx->stream));
    }
    S->d_st = dev_alloc<SolveState>(ctx, 1);
    AB2_CUDA(cudaMemsetAsync(S->d_st, 0, sizeof(SolveState), ctx->stream));
    AB2_CUDA(cudaMallocHost((void**)&S->h_st, sizeof(SolveState)));
    S->hist_cap = 2 * o->max_iter + 8;  // BiCGStab tests s and r each iteration
    S->d_hist = dev_alloc<double>(ctx, (size_t)S->hist_cap);
    if (o->use_graph) build_graph(S);
    AB2_CUDA(cudaEventRecord(S->ev1, ctx->stream));
    AB2_CUDA(cudaEventSynchronize(S->ev1));
    float ms = 0;
    AB2_CUDA(cudaEventElapsedTime(&ms, S->ev0, S->ev1));
    S->setup_ms = ms;
  });
  if (rc != AB2_OK) {
    ab2_solver_destroy(S);
    return rc;
  }
  *out = S;
  return AB2_OK;
}

int ab2_solver_solve(ab2_solver* S, const ab2_vector* b, ab2_vector* x, ab2_status* status) {
  if (!S || !b || !x || !status || b->n != S->A->n || x->n != S->A->n) return AB2_ERR_BAD_ARG;
  ab2_context* ctx = S->ctx;
  std::memset(status, 0, sizeof(*status));
  return guard(ctx, [&] {
    const int n = S->A->n;
    const ab2_solver_options& o = S->opts;
    AB2_CUDA(cudaEventRecord(S->ev0, ctx->stream));
    // Iteration ctor: b.b and the criterion (Iteration.h:44-68)
    op_dot(ctx, n, b->d, b->d, &S->d_st->nrm2_b, 0);
    k_state_init<<<1, 1, 0, ctx->stream>>>(S->d_st, o.tol, o.max_iter, x->d, b->d, S->d_hist, S->hist_cap);
    check_launch(ctx, "state_init");
    const int g = fused_grid(ctx, n);
    // r = b - A x (and r0, rho1 for BiCGStab)
    double* r0 = o.solver == AB2_SOLVER_BICGSTAB ? S->w[1] : nullptr;
    with_view<double>(S->A, o.spmv_variant, [&](auto view) {
      k_residual<<<g, kCtlThreads, 0, ctx->stream>>>(n, view, S->d_st, S->w[0], r0, red_slot(ctx, 0));
    });
    check_launch(ctx, "residual");
    // Null right-hand side: the reference returns before any iteration.
    AB2_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(SolveState), cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    if (!S->h_st->done) {
      if (o.use_graph) {
        AB2_CUDA(cudaGraphLaunch(S->exec, ctx->stream));
      } else {
        // Host-driven loop over the same kernels, checking the flag in batches.
        for (;;) {
          const int batch = 8;
          for (int i = 0; i < batch; ++i) enqueue_body(S, 0, 0);
          AB2_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(SolveState), cudaMemcpyDeviceToHost, ctx->stream));
          AB2_CUDA(cudaStreamSynchronize(ctx->stream));
          if (S->h_st->done) break;
        }
      }
    }
    AB2_CUDA(cudaEventRecord(S->ev1, ctx->stream));
    AB2_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(SolveState), cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    float ms = 0;
    AB2_CUDA(cudaEventElapsedTime(&ms, S->ev0, S->ev1));
    S->solve_ms = ms;
    const SolveState& st = *S->h_st;
    if (o.use_graph) ctx->launches += (long long)st.bodies * S->body_launches;
    int pe = pc_error(ctx, S->pc);
    status->succeeded = st.converged;
    status->iterations = st.iter;
    status->error = pe ? AB2_ERR_TIMEOUT : st.error;
    status->breakdown = st.breakdown;
    status->nrm2_b = st.nrm2_b;
    status->residual = st.nrm2_b > 0 ? std::sqrt(st.rr) / std::sqrt(st.nrm2_b) : 0.0;
    status->setup_ms = S->setup_ms;
    status->solve_ms = S->solve_ms;
    if (pe) pc_reset(ctx, S->pc);
    // ||b - A x|| / ||b|| (reported, not part of the timed solve)
    RedSlot red = red_slot(ctx, 5);
    with_view<double>(S->A, o.spmv_variant, [&](auto view) {
      k_true_residual<<<g, kCtlThreads, 0, ctx->stream>>>(n, view, x->d, b->d, red);
    });
    check_launch(ctx, "true_residual");
    AB2_CUDA(cudaMemcpyAsync(ctx->h_pinned, red.result, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    status->true_residual = ctx->h_pinned[1] > 0 ? std::sqrt(ctx->h_pinned[0] / ctx->h_pinned[1]) : 0.0;
  });
}

int ab2_solver_history(const ab2_solver* S, double* hist, int cap, int* len) {
  if (!S || !len || (cap > 0 && !hist)) return AB2_ERR_BAD_ARG;
  const int have = std::min(S->h_st ? S->h_st->hist_len : 0, S->hist_cap);
  *len = S->h_st ? S->h_st->hist_len : 0;
  const int m = std::min(have, cap);
  if (m > 0) {
    if (cudaMemcpy(hist, S->d_hist, sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost) != cudaSuccess)
      return AB2_ERR_CUDA;
  }
  return AB2_OK;
}

int ab2_solver_destroy(ab2_solver* S) {
  if (!S) return AB2_ERR_BAD_ARG;
  if (S->ctx) ctx_quiesce(S->ctx);
  if (S->exec) cudaGraphExecDestroy(S->exec);
  if (S->graph) cudaGraphDestroy(S->graph);
  if (S->pc) ab2_precond_destroy(S->pc);
  for (double* p : S->w) dev_free(S->ctx, p);
  dev_free(S->ctx, S->d_st);
  dev_free(S->ctx, S->d_hist);
  if (S->h_st) cudaFreeHost(S->h_st);
  if (S->ev0) cudaEventDestroy(S->ev0);
  if (S->ev1) cudaEventDestroy(S->ev1);
  if (S->ctx) ctx_release(S->ctx);
  delete S;
  return AB2_OK;
}

}  // extern "C"
