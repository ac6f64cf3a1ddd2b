// dist_solver.cu -- CG (expression/krylov/CG.h:59-150) and BiCGStab
// (BiCGStab.h:152-300) with Iteration.h's stop test on the distributed
// algebra, device-resident.
//
// Every rank runs the same sequence of kernels and collectives.  The scalars
// of the recurrence (r.r, r.z, p.q) are rank-ordered sums, identical on every
// rank, so every rank takes the same decisions.  Iterations are queued in
// batches without host synchronisation: after the stop test has ended the
// solve, the kernels that change x, r and p return at once while the
// collectives of the rest of the batch still run on every rank, then the
// host reads the state.  The operations, their order and their rounding are
// those of the reference template on Alien's parallel algebra:
//   prologue  r = b - A x; z = M r; rho1 = r.z; p = z; q = A p; alpha = p.q
//             (0: stop(r) ? done : breakdown "alpha"); x += (rho1/alpha) p;
//             r -= (rho1/alpha) q; rho = rho1
//   loop      while !stop(r): z = M r; rho1 = r.z; z += (rho1/rho) p; p = z;
//             q = A p; alpha = q.p (as above); x, r updated; rho = rho1
// BiCGStab takes the steps of the single-GPU engine's BiCGStab body
// (krylov.cu), each reduction split into local partials (the same tree as
// op_dot), their rank-ordered sum, and a one-thread kernel for the decision.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "ab2_dist.h"
#include "ab2_internal.cuh"
#include "dist.cuh"
#include "precond.cuh"
#include "reduce.cuh"

namespace ab2 {
namespace {

constexpr int kBatch = 8;  // iterations queued between two reads of the state

struct DistState {
  double rho;
  double criteria;
  double last;   // the stop test's last r.r (s.s)
  double rho1, alpha, beta, omega, rr_r;  // BiCGStab
  int iter;
  int max_iter;
  int done;
  int status;
  int pq_zero;   // CG: p.q was 0: the host finishes the step (stop test or breakdown)
  int first;     // the prologue step (no stop test before it)
  int hist_len;
  int breakdown;   // BiCGStab: AB2_BREAKDOWN_*
  int exit_fixup;  // BiCGStab: stopped on s, x += alpha phat still to do
};

// Iteration::stop with the dot product already summed.
__device__ __forceinline__ bool dstop(DistState* st, double rr, double* hist, int cap) {
  if (st->iter >= st->max_iter) return true;
  st->last = rr;
  if (st->hist_len < cap) hist[st->hist_len] = rr;
  st->hist_len += 1;
  st->status = rr < st->criteria;
  return st->status != 0;
}

// g[0] = r.r, g[1] = r.z, g[2] = p.q (rank-ordered sums)
__global__ void k_dcg_stop(DistState* st, const double* g, double* hist, int cap) {
  if (st->done) return;
  if (dstop(st, g[0], hist, cap)) st->done = 1;
}

// p = first ? z : z + (rho1/rho) p   (axpy(alpha, p, z) then copy(z, p))
__global__ void k_dcg_dir(int n, const double* __restrict__ z, double* __restrict__ p, const DistState* st,
                          const double* g) {
  if (st->done) return;
  const bool first = st->first != 0;
  const double beta = first ? 0.0 : g[1] / st->rho;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = first ? z[i] : fma_rn(beta, p[i], z[i]);
}

// alpha = r.z / p.q; x += alpha p; r -= alpha q; rho = r.z
__global__ void k_dcg_update(int n, const double* __restrict__ p, const double* __restrict__ q, double* __restrict__ x,
                             double* __restrict__ r, DistState* st, const double* g) {
  if (st->done) return;
  const double pq = g[2];
  if (pq == 0.0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->pq_zero = 1;
      st->done = 1;
    }
    return;
  }
  const double alpha = g[1] / pq;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = fma_rn(alpha, p[i], x[i]);
    r[i] = fma_rn(-alpha, q[i], r[i]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->rho = g[1];
    st->iter += 1;
    st->first = 0;
  }
}

// ------------------------------------------------------------------ BiCGStab
// p = r (first) or r + beta (p - omega v): axpy, scal, axpy (BiCGStab.h:273-276)
__global__ void k_dbi_p(int n, const double* __restrict__ r, const double* __restrict__ v, double* __restrict__ p,
                        const DistState* st) {
  if (st->done) return;
  const int first = st->first;
  const double beta = st->beta, omega = st->omega;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = first ? r[i] : add_rn(r[i], mul_rn(beta, fma_rn(-omega, v[i], p[i])));
}

// g[0] = v.r0: alpha = rho1 / v.r0, breakdown "alpha" on zero
__global__ void k_dbi_alpha(DistState* st, const double* g) {
  if (st->done) return;
  if (g[0] == 0.0) {
    st->breakdown = AB2_BREAKDOWN_ALPHA;
    st->done = 1;
  } else {
    st->alpha = st->rho1 / g[0];
  }
}

// s = r - alpha v ; partials s.s and r.r (every thread reaches the reduction)
__global__ void __launch_bounds__(kThreads) k_dbi_s(int n, const double* __restrict__ r, const double* __restrict__ v,
                                                    double* __restrict__ s, const DistState* st, RedSlot red) {
  const bool live = !st->done;
  const double alpha = st->alpha;
  double acc[2] = {0.0, 0.0};
  if (live)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      const double rv = r[i];
      const double sv = fma_rn(-alpha, v[i], rv);
      s[i] = sv;
      acc[0] = fma_rn(sv, sv, acc[0]);
      acc[1] = fma_rn(rv, rv, acc[1]);
    }
  grid_reduce<2>(acc, red.partials, red.counter, red.result);
}

// g[0] = s.s, g[1] = r.r: stop test on s (exit with x += alpha phat; the first
// step counts it, BiCGStab.h:194-199, later steps do not, :259-263)
__global__ void k_dbi_sdecide(DistState* st, const double* g, double* hist, int cap) {
  if (st->done) return;
  st->rr_r = g[1];
  if (dstop(st, g[0], hist, cap)) {
    if (st->first) st->iter += 1;
    st->exit_fixup = 1;
    st->done = 1;
  }
}

// partials t.s and t.t (t complete, ghost sums included)
__global__ void __launch_bounds__(kThreads) k_dbi_tdots(int n, const double* __restrict__ t, const double* __restrict__ s,
                                                        const DistState* st, RedSlot red) {
  const bool live = !st->done;
  double acc[2] = {0.0, 0.0};
  if (live)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      const double tv = t[i];
      acc[0] = fma_rn(tv, s[i], acc[0]);
      acc[1] = fma_rn(tv, tv, acc[1]);
    }
  grid_reduce<2>(acc, red.partials, red.counter, red.result);
}

// g[0] = t.s, g[1] = t.t: omega, or the beta == 0 branch (first step:
// stop(r); later: stop(s), whose value was just tested) (BiCGStab.h:202-216, 266-282)
__global__ void k_dbi_omega(DistState* st, const double* g, double* hist, int cap) {
  if (st->done) return;
  if (g[1] == 0.0) {
    const double v = st->first ? st->rr_r : st->last;
    if (dstop(st, v, hist, cap)) {
      if (st->first) st->iter += 1;
      st->exit_fixup = 1;
    } else {
      st->breakdown = AB2_BREAKDOWN_BETA;
    }
    st->done = 1;
  } else {
    st->omega = g[0] / g[1];
  }
}

// x += omega shat ; x += alpha phat ; r = s - omega t, partials r.r and r.r0
// -- or, after a stop on s, the exit's x += alpha phat alone
__global__ void __launch_bounds__(kThreads) k_dbi_update(int n, const double* __restrict__ shat,
                                                         const double* __restrict__ phat, const double* __restrict__ s,
                                                         const double* __restrict__ t, const double* __restrict__ r0,
                                                         double* __restrict__ r, double* __restrict__ x,
                                                         const DistState* st, RedSlot red) {
  const int done = st->done, fix = st->exit_fixup;
  const double alpha = st->alpha, omega = st->omega;
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (done) {
      if (fix) x[i] = fma_rn(alpha, phat[i], x[i]);
    } else {
      x[i] = fma_rn(alpha, phat[i], fma_rn(omega, shat[i], x[i]));
      const double rv = fma_rn(-omega, t[i], s[i]);
      r[i] = rv;
      acc[0] = fma_rn(rv, rv, acc[0]);
      acc[1] = fma_rn(rv, r0[i], acc[1]);
    }
  }
  grid_reduce<2>(acc, red.partials, red.counter, red.result);
}

// g[0] = r.r, g[1] = r.r0: the loop's stop test, rho1, beta, breakdown "rho"
__global__ void k_dbi_tail(DistState* st, const double* g, double* hist, int cap) {
  if (st->done) {
    st->exit_fixup = 0;
    return;
  }
  st->rho = st->rho1;
  st->iter += 1;
  st->first = 0;
  if (dstop(st, g[0], hist, cap)) {
    st->done = 1;
  } else {
    st->rho1 = g[1];
    st->beta = (st->rho1 / st->rho) * (st->alpha / st->omega);
    if (st->rho == 0.0) {
      st->breakdown = AB2_BREAKDOWN_RHO;
      st->done = 1;
    }
  }
}

}  // namespace
}  // namespace ab2

struct ab2_dist_solver {
  ab2_context* ctx = nullptr;
  ab2_comm* comm = nullptr;
  const ab2_dist_matrix* A = nullptr;
  ab2_solver_options o{};
  ab2_precond* pc = nullptr;
  int n = 0;
  double *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *xe = nullptr, *t = nullptr;
  // BiCGStab: r0, v, s, phat and shat (with ghost room), t
  double *r0 = nullptr, *v = nullptr, *sv = nullptr, *phat = nullptr, *shat = nullptr, *tv = nullptr;
  double* g = nullptr;        // rank-ordered sums
  double* hist = nullptr;
  int hist_cap = 0;
  ab2::DistState* st = nullptr;
  ab2::DistState h_st{};
  double setup_ms = 0.0;
};

namespace ab2 {
namespace {

double dist_dot_host(ab2_context* ctx, ab2_comm* c, int n, const double* x, const double* y) {
  RedSlot s = red_slot(ctx, 0);
  op_dot(ctx, n, x, y, s.result, 0);
  dist_sum(ctx, c, s.result, 1, c->d_sum);
  return read_scalar(ctx, c->d_sum);
}

void dcg_step(ab2_dist_solver* S, bool stop_test) {
  ab2_context* ctx = S->ctx;
  ab2_comm* c = S->comm;
  const int n = S->n;
  RedSlot s = red_slot(ctx, 0);
  if (stop_test) {
    op_dot(ctx, n, S->r, S->r, s.result, 0);
    dist_sum(ctx, c, s.result, 1, S->g + 0);
    k_dcg_stop<<<1, 1, 0, ctx->stream>>>(S->st, S->g, S->hist, S->hist_cap);
    check_launch(ctx, "dcg_stop");
  }
  pc_apply(ctx, S->pc, S->r, S->z);
  op_dot(ctx, n, S->r, S->z, s.result, 0);
  dist_sum(ctx, c, s.result, 1, S->g + 1);
  k_dcg_dir<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, S->z, S->p, S->st, S->g);
  check_launch(ctx, "dcg_dir");
  dist_mult(ctx, S->A, S->p, S->q);
  op_dot(ctx, n, S->p, S->q, s.result, 0);
  dist_sum(ctx, c, s.result, 1, S->g + 2);
  k_dcg_update<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, S->p, S->q, S->xe, S->r, S->st, S->g);
  check_launch(ctx, "dcg_update");
}

void dbi_step(ab2_dist_solver* S) {
  ab2_context* ctx = S->ctx;
  ab2_comm* c = S->comm;
  const int n = S->n;
  const int g = red_grid(ctx, n);
  k_dbi_p<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, S->r, S->v, S->p, S->st);
  check_launch(ctx, "dbi_p");
  pc_apply(ctx, S->pc, S->p, S->phat);
  dist_mult(ctx, S->A, S->phat, S->v);
  RedSlot s0 = red_slot(ctx, 0);
  op_dot(ctx, n, S->v, S->r0, s0.result, 0);
  dist_sum(ctx, c, s0.result, 1, S->g + 0);
  k_dbi_alpha<<<1, 1, 0, ctx->stream>>>(S->st, S->g + 0);
  check_launch(ctx, "dbi_alpha");
  RedSlot s1 = red_slot(ctx, 1);
  k_dbi_s<<<g, kThreads, 0, ctx->stream>>>(n, S->r, S->v, S->sv, S->st, s1);
  check_launch(ctx, "dbi_s");
  dist_sum(ctx, c, s1.result, 2, S->g + 1);
  k_dbi_sdecide<<<1, 1, 0, ctx->stream>>>(S->st, S->g + 1, S->hist, S->hist_cap);
  check_launch(ctx, "dbi_sdecide");
  pc_apply(ctx, S->pc, S->sv, S->shat);
  dist_mult(ctx, S->A, S->shat, S->tv);
  RedSlot s2 = red_slot(ctx, 2);
  k_dbi_tdots<<<g, kThreads, 0, ctx->stream>>>(n, S->tv, S->sv, S->st, s2);
  check_launch(ctx, "dbi_tdots");
  dist_sum(ctx, c, s2.result, 2, S->g + 3);
  k_dbi_omega<<<1, 1, 0, ctx->stream>>>(S->st, S->g + 3, S->hist, S->hist_cap);
  check_launch(ctx, "dbi_omega");
  RedSlot s3 = red_slot(ctx, 3);
  k_dbi_update<<<g, kThreads, 0, ctx->stream>>>(n, S->shat, S->phat, S->sv, S->tv, S->r0, S->r, S->xe, S->st, s3);
  check_launch(ctx, "dbi_update");
  dist_sum(ctx, c, s3.result, 2, S->g + 5);
  k_dbi_tail<<<1, 1, 0, ctx->stream>>>(S->st, S->g + 5, S->hist, S->hist_cap);
  check_launch(ctx, "dbi_tail");
}

void read_state(ab2_dist_solver* S) {
  AB2_CUDA(cudaMemcpyAsync(&S->h_st, S->st, sizeof(DistState), cudaMemcpyDeviceToHost, S->ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(S->ctx->stream));
}

void write_state(ab2_dist_solver* S) {
  AB2_CUDA(cudaMemcpyAsync(S->st, &S->h_st, sizeof(DistState), cudaMemcpyHostToDevice, S->ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(S->ctx->stream));
}

void dist_solve(ab2_dist_solver* S, const double* b, double* x, ab2_status* status) {
  ab2_context* ctx = S->ctx;
  ab2_comm* c = S->comm;
  const int n = S->n;
  cudaEvent_t e0, e1;
  AB2_CUDA(cudaEventCreate(&e0));
  AB2_CUDA(cudaEventCreate(&e1));
  AB2_CUDA(cudaEventRecord(e0, ctx->stream));
  DistState& h = S->h_st;
  h = DistState{};
  h.max_iter = S->o.max_iter;
  h.first = 1;
  // Iteration's constructor: criteria = tol^2 b.b; a zero right-hand side is converged
  const double bb = dist_dot_host(ctx, c, n, b, b);
  h.criteria = S->o.tol * S->o.tol * bb;
  h.status = bb == 0.0;
  op_copy(ctx, n, x, S->xe);
  int err = AB2_OK, breakdown = AB2_BREAKDOWN_NONE;
  if (bb != 0.0 && S->o.solver == AB2_SOLVER_BICGSTAB) {
    // r = b - A x ; r0 = r ; rho1 = r.r0 (BiCGStab.h:170-176)
    op_copy(ctx, n, b, S->r);
    dist_mult(ctx, S->A, S->xe, S->v);
    op_axpy(ctx, n, -1.0, S->v, S->r);
    op_copy(ctx, n, S->r, S->r0);
    h.rho1 = dist_dot_host(ctx, c, n, S->r, S->r0);
    write_state(S);
    do {
      for (int k = 0; k < kBatch; ++k) dbi_step(S);
      read_state(S);
    } while (!h.done);
    if (h.breakdown) {
      err = AB2_ERR_BREAKDOWN;
      breakdown = h.breakdown;
    }
  } else if (bb != 0.0) {
    write_state(S);
    op_copy(ctx, n, b, S->r);
    dist_mult(ctx, S->A, S->xe, S->p);
    op_axpy(ctx, n, -1.0, S->p, S->r);
    bool first = true;
    for (;;) {
      for (int k = 0; k < kBatch; ++k) {
        dcg_step(S, !first);
        first = false;
      }
      read_state(S);
      if (!h.done) continue;
      if (h.pq_zero) {
        // CG.h:96-104,131-139: if (it.stop(r)) { it.next(); return; } else breakdown "alpha"
        const double rr = dist_dot_host(ctx, c, n, S->r, S->r);  // collective on every rank alike
        if (h.iter >= h.max_iter) {
          h.iter += 1;
        } else {
          h.last = rr;
          if (h.hist_len < S->hist_cap)
            AB2_CUDA(cudaMemcpyAsync(S->hist + h.hist_len, &rr, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
          h.hist_len += 1;
          h.status = rr < h.criteria;
          if (h.status) h.iter += 1;
          else {
            err = AB2_ERR_BREAKDOWN;
            breakdown = AB2_BREAKDOWN_ALPHA;
          }
        }
      }
      break;
    }
  }
  AB2_CUDA(cudaEventRecord(e1, ctx->stream));
  AB2_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  AB2_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  op_copy(ctx, n, S->xe, x);
  // true residual ||b - A x|| / ||b||
  dist_mult(ctx, S->A, S->xe, S->q);
  op_copy(ctx, n, b, S->t);
  op_axpy(ctx, n, -1.0, S->q, S->t);
  const double tt = dist_dot_host(ctx, c, n, S->t, S->t);
  status->succeeded = h.status;
  status->iterations = h.iter;
  status->error = err;
  status->breakdown = breakdown;
  status->nrm2_b = bb;
  status->residual = bb > 0 ? std::sqrt(h.last / bb) : 0.0;
  status->true_residual = bb > 0 ? std::sqrt(tt / bb) : std::sqrt(tt);
  status->setup_ms = S->setup_ms;
  status->solve_ms = ms;
}

void dist_solver_free(ab2_dist_solver* S) {
  ab2_context* ctx = S->ctx;
  if (ctx) {
    ctx_quiesce(ctx);
    for (void* p : {(void*)S->r, (void*)S->z, (void*)S->p, (void*)S->q, (void*)S->xe, (void*)S->t, (void*)S->g,
                    (void*)S->hist, (void*)S->st, (void*)S->r0, (void*)S->v, (void*)S->sv, (void*)S->tv,
                    (void*)S->phat, (void*)S->shat})
      dev_free(ctx, p);
  }
  if (S->pc) ab2_precond_destroy(S->pc);
  if (ctx) ctx_release(ctx);
  delete S;
}

}  // namespace
}  // namespace ab2

using namespace ab2;

extern "C" {

int ab2_dist_solver_create(ab2_context* ctx, ab2_comm* comm, const ab2_dist_matrix* A, const ab2_solver_options* o,
                           ab2_dist_solver** out) {
  if (!ctx || !comm || !A || !o || !out || A->comm != comm || comm->ctx != ctx || o->max_iter < 0) return AB2_ERR_BAD_ARG;
  *out = nullptr;
  if (o->solver != AB2_SOLVER_CG && o->solver != AB2_SOLVER_BICGSTAB) return AB2_ERR_BAD_ARG;
  ab2_dist_solver* S = new (std::nothrow) ab2_dist_solver();
  if (!S) return AB2_ERR_OOM;
  S->ctx = ctx_retain(ctx);
  S->comm = comm;
  S->A = A;
  S->o = *o;
  S->n = A->n_loc;
  ab2_precond_options po{};
  po.kind = o->precond;
  po.ilu_schedule = o->ilu_schedule;
  const auto t0 = std::chrono::steady_clock::now();
  int rc = ab2_dist_precond_create(ctx, A, &po, &S->pc);
  if (rc == AB2_OK) {
    rc = guard(ctx, [&] {
      const size_t n = (size_t)S->n, room = (size_t)A->n_loc + (size_t)A->n_ghost;
      S->r = dev_alloc<double>(ctx, n);
      S->z = dev_alloc<double>(ctx, n);
      S->p = dev_alloc<double>(ctx, room);
      S->q = dev_alloc<double>(ctx, n);
      S->xe = dev_alloc<double>(ctx, room);
      S->t = dev_alloc<double>(ctx, n);
      S->g = dev_alloc<double>(ctx, 8);
      if (o->solver == AB2_SOLVER_BICGSTAB) {
        S->r0 = dev_alloc<double>(ctx, n);
        S->v = dev_alloc<double>(ctx, n);
        S->sv = dev_alloc<double>(ctx, n);
        S->tv = dev_alloc<double>(ctx, n);
        S->phat = dev_alloc<double>(ctx, room);
        S->shat = dev_alloc<double>(ctx, room);
        AB2_CUDA(cudaMemsetAsync(S->v, 0, sizeof(double) * n, ctx->stream));
      }
      S->hist_cap = 2 * o->max_iter + 4;
      S->hist = dev_alloc<double>(ctx, (size_t)S->hist_cap);
      S->st = dev_alloc<DistState>(ctx, 1);
      AB2_CUDA(cudaMemsetAsync(S->p, 0, sizeof(double) * room, ctx->stream));
      AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    });
  }
  S->setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (rc != AB2_OK) {
    dist_solver_free(S);
    return rc;
  }
  *out = S;
  return AB2_OK;
}

int ab2_dist_solver_solve(ab2_dist_solver* S, const ab2_vector* b, ab2_vector* x, ab2_status* status) {
  if (!S || !b || !x || !status || b->n != S->n || x->n != S->n) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(S->ctx, S->o.solver == AB2_SOLVER_CG ? "DIST-SOLVER-CG" : "DIST-SOLVER-BICGSTAB");
  *status = ab2_status{};
  return guard(S->ctx, [&] { dist_solve(S, b->d, x->d, status); });
}

int ab2_dist_solver_history(const ab2_dist_solver* S, double* hist, int cap, int* len) {
  if (!S || !len || cap < 0 || (cap > 0 && !hist)) return AB2_ERR_BAD_ARG;
  *len = S->h_st.hist_len;
  const int m = std::min({cap, S->h_st.hist_len, S->hist_cap});
  return guard(S->ctx, [&] {
    if (m > 0) {
      AB2_CUDA(cudaMemcpyAsync(hist, S->hist, sizeof(double) * m, cudaMemcpyDeviceToHost, S->ctx->stream));
      AB2_CUDA(cudaStreamSynchronize(S->ctx->stream));
    }
  });
}

int ab2_dist_solver_destroy(ab2_dist_solver* S) {
  if (!S) return AB2_ERR_BAD_ARG;
  dist_solver_free(S);
  return AB2_OK;
}

}  // extern "C"
