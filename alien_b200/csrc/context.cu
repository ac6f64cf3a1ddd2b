// context.cu -- contexts, vectors, device scalars and the BLAS-1 part of the
// algebra (SimpleCSRInternalLinearAlgebra.cc:74-257 / CBLASMPIKernel.h:37-125
// on the CPU side, SYCLKernelInternal.h:110-1087 on the SYCL side).
//
// BLAS-1 rounding follows the reference's operations one for one:
//   axpy  y = fma(a, x, y)     scal  x = a*x      pointwiseMult  w = x*y
//   aypx  y = fma(a, y, x)     dot   deterministic tree (reduce.cuh)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "ab2_internal.cuh"
#include "reduce.cuh"

namespace ab2 {

namespace {

__global__ void k_fill(int n, double a, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = a;
}
__global__ void k_copy(int n, const double* __restrict__ x, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[i];
}
__global__ void k_axpy(int n, double a, const double* __restrict__ x, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = fma(a, x[i], y[i]);
}
__global__ void k_aypx(int n, double a, double* __restrict__ y, const double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = fma(a, y[i], x[i]);
}
__global__ void k_scal(int n, double a, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = a * x[i];
}
// x, y and w may alias (the reference calls pointwiseMult(d, y, y)).
__global__ void k_pmult(int n, const double* x, const double* y, double* w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) w[i] = x[i] * y[i];
}
__global__ void k_reciprocal(int n, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = 1.0 / x[i];
}

__global__ void k_dot(int n, const double* __restrict__ x, const double* __restrict__ y, double* partials,
                      unsigned int* counter, double* out) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[0] = fma(x[i], y[i], acc[0]);
  grid_reduce<1>(acc, partials, counter, out);
}
__global__ void k_asum(int n, const double* __restrict__ x, double* partials, unsigned int* counter, double* out) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[0] += fabs(x[i]);
  grid_reduce<1>(acc, partials, counter, out);
}
__global__ void k_amax(int n, const double* __restrict__ x, double* partials, unsigned int* counter, double* out) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[0] = fmax(acc[0], fabs(x[i]));
  grid_reduce<1, Combine::Max>(acc, partials, counter, out);
}

}  // namespace

// Grid of every reduction over n values, standalone or fused: one block per
// 256 values, at most 8 blocks per SM.  A function of n and the device only,
// so the summation tree -- and the rounding -- is the same on every run.
int red_grid(const ab2_context* ctx, int n) {
  return grid_for(n, kThreads, std::min(kMaxRedBlocks, ctx->num_sms * (2048 / kThreads)));
}

// ---------------------------------------------------------------- phase timers
struct PhaseTimer {
  struct Rec {
    int phase;
    cudaEvent_t a, b;
    bool ended;
  };
  std::vector<std::string> names;
  std::vector<long long> calls;
  std::vector<double> ms;
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  bool print_at_exit = false;

  cudaEvent_t event() {
    cudaEvent_t e = nullptr;
    if (!pool.empty()) {
      e = pool.back();
      pool.pop_back();
    } else if (cudaEventCreate(&e) != cudaSuccess) {
      e = nullptr;
    }
    return e;
  }
  int phase(const char* name) {
    for (size_t i = 0; i < names.size(); ++i)
      if (names[i] == name) return (int)i;
    names.push_back(name);
    calls.push_back(0);
    ms.push_back(0.0);
    return (int)names.size() - 1;
  }
  // Folds every finished record into the totals (waits for their events).
  void resolve() {
    std::vector<Rec> keep;
    for (Rec& r : recs) {
      if (!r.ended) {
        keep.push_back(r);
        continue;
      }
      float t = 0.f;
      if (r.phase >= 0 && cudaEventSynchronize(r.b) == cudaSuccess &&
          cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) {
        ms[(size_t)r.phase] += t;
        calls[(size_t)r.phase] += 1;
      }
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    recs.swap(keep);
  }
  ~PhaseTimer() {
    for (Rec& r : recs) {
      if (r.a) cudaEventDestroy(r.a);
      if (r.b) cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
  }
};

void phase_begin(ab2_context* ctx, const char* name, int* token) {
  PhaseTimer* t = ctx->timer;
  cudaEvent_t a = t->event(), b = t->event();
  if (!a || !b || cudaEventRecord(a, ctx->stream) != cudaSuccess) {
    if (a) t->pool.push_back(a);
    if (b) t->pool.push_back(b);
    return;
  }
  t->recs.push_back(PhaseTimer::Rec{t->phase(name), a, b, false});
  *token = (int)t->recs.size() - 1;
}

void phase_end(ab2_context* ctx, int token) {
  PhaseTimer* t = ctx->timer;
  if (!t || token >= (int)t->recs.size()) return;
  PhaseTimer::Rec& r = t->recs[(size_t)token];
  if (cudaEventRecord(r.b, ctx->stream) != cudaSuccess) r.phase = -1;  // dropped when resolved
  r.ended = true;
  // Bounded memory: fold finished records once many are pending (only when
  // no scope is open, so the tokens of open scopes stay valid).
  if (t->recs.size() >= 4096 && token == (int)t->recs.size() - 1) {
    bool all_ended = true;
    for (const PhaseTimer::Rec& x : t->recs) all_ended = all_ended && x.ended;
    if (all_ended) t->resolve();
  }
}

void ctx_release(ab2_context* ctx) {
  if (ctx->refs.fetch_sub(1) != 1) return;
  ctx_quiesce(ctx);
  if (ctx->timer) {
    if (ctx->timer->print_at_exit) {
      // StdTimer::printInfo's format (utils/StdTimer.h): phase:seconds
      ctx->timer->resolve();
      std::fprintf(stderr, "================================\nPERF INFO : B200-ALGEBRA (device %d)\n", ctx->device);
      for (size_t i = 0; i < ctx->timer->names.size(); ++i)
        std::fprintf(stderr, "%s:%.6f (%lld calls)\n", ctx->timer->names[i].c_str(), ctx->timer->ms[i] * 1e-3,
                     ctx->timer->calls[i]);
      std::fprintf(stderr, "================================\n");
    }
    delete ctx->timer;
    ctx->timer = nullptr;
  }
  dev_free(ctx, ctx->d_partials);
  dev_free(ctx, ctx->d_counters);
  dev_free(ctx, ctx->d_results);
  if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

RedSlot red_slot(ab2_context* ctx, int slot) {
  return RedSlot{ctx->d_partials + (size_t)slot * kMaxRedComps * kMaxRedBlocks, ctx->d_counters + slot,
                 ctx->d_results + (size_t)slot * kMaxRedComps};
}

namespace {
template <class S, class D>
__global__ void k_convert(long long m, const S* __restrict__ a, D* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
    b[i] = (D)a[i];
}
}  // namespace

void op_to_f32(ab2_context* ctx, long long m, const double* a, float* b) {
  k_convert<<<grid_for(m), kThreads, 0, ctx->stream>>>(m, a, b);
  check_launch(ctx, "to_f32");
}

void op_to_f64(ab2_context* ctx, long long m, const float* a, double* b) {
  k_convert<<<grid_for(m), kThreads, 0, ctx->stream>>>(m, a, b);
  check_launch(ctx, "to_f64");
}

void op_fill(ab2_context* ctx, int n, double a, double* x) {
  k_fill<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, a, x);
  check_launch(ctx, "fill");
}
void op_copy(ab2_context* ctx, int n, const double* x, double* y) {
  if (x == y) return;
  k_copy<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, x, y);
  check_launch(ctx, "copy");
}
void op_axpy(ab2_context* ctx, int n, double a, const double* x, double* y) {
  k_axpy<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, a, x, y);
  check_launch(ctx, "axpy");
}
void op_aypx(ab2_context* ctx, int n, double a, double* y, const double* x) {
  k_aypx<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, a, y, x);
  check_launch(ctx, "aypx");
}
void op_scal(ab2_context* ctx, int n, double a, double* x) {
  k_scal<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, a, x);
  check_launch(ctx, "scal");
}
void op_pmult(ab2_context* ctx, int n, const double* x, const double* y, double* w) {
  k_pmult<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, x, y, w);
  check_launch(ctx, "pointwise_mult");
}
void op_reciprocal(ab2_context* ctx, int n, double* x) {
  k_reciprocal<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, x);
  check_launch(ctx, "reciprocal");
}
void op_dot(ab2_context* ctx, int n, const double* x, const double* y, double* out, int slot) {
  RedSlot s = red_slot(ctx, slot);
  k_dot<<<red_grid(ctx, n), kThreads, 0, ctx->stream>>>(n, x, y, s.partials, s.counter, out);
  check_launch(ctx, "dot");
}
void op_norm1(ab2_context* ctx, int n, const double* x, double* out, int slot) {
  RedSlot s = red_slot(ctx, slot);
  k_asum<<<red_grid(ctx, n), kThreads, 0, ctx->stream>>>(n, x, s.partials, s.counter, out);
  check_launch(ctx, "norm1");
}
void op_norm0(ab2_context* ctx, int n, const double* x, double* out, int slot) {
  RedSlot s = red_slot(ctx, slot);
  k_amax<<<red_grid(ctx, n), kThreads, 0, ctx->stream>>>(n, x, s.partials, s.counter, out);
  check_launch(ctx, "norm0");
}
double read_scalar(ab2_context* ctx, const double* d) {
  AB2_CUDA(cudaMemcpyAsync(ctx->h_pinned, d, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  return ctx->h_pinned[0];
}

}  // namespace ab2

using namespace ab2;

namespace {

int check_vec(const ab2_vector* v, int n) {
  if (!v || v->n != n) return AB2_ERR_BAD_ARG;
  return AB2_OK;
}

}  // namespace

extern "C" {

int ab2_context_create(int device, ab2_context** out) {
  if (!out) return AB2_ERR_BAD_ARG;
  *out = nullptr;
  ab2_context* ctx = new (std::nothrow) ab2_context();
  if (!ctx) return AB2_ERR_OOM;
  int rc = guard(ctx, [&] {
    int count = 0;
    AB2_CUDA(cudaGetDeviceCount(&count));
    require(device >= 0 && device < count, "device index out of range");
    ctx->device = device;
    AB2_CUDA(cudaSetDevice(device));
    AB2_CUDA(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
    AB2_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    // Keep freed blocks in the device's default pool (dev_alloc draws from
    // it): solvers and preconditioners created per solve then reuse memory
    // instead of mapping and unmapping hundreds of MB each time.
    cudaMemPool_t pool;
    AB2_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;
    AB2_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    ctx->d_partials = dev_alloc<double>(ctx, (size_t)kRedSlots * kMaxRedComps * kMaxRedBlocks);
    ctx->d_counters = dev_alloc<unsigned int>(ctx, kRedSlots);
    ctx->d_results = dev_alloc<double>(ctx, (size_t)kRedSlots * kMaxRedComps);
    AB2_CUDA(cudaMemset(ctx->d_counters, 0, sizeof(unsigned int) * kRedSlots));
    AB2_CUDA(cudaMallocHost((void**)&ctx->h_pinned, 64 * sizeof(double)));
    // AB2_PERF_TIMER=1: phase timers on, printed when the context goes (as
    // the reference's ALIEN_USE_PERF_TIMER build prints its timers).
    const char* pt = std::getenv("AB2_PERF_TIMER");
    if (pt && pt[0] && pt[0] != '0') {
      ctx->timer = new PhaseTimer();
      ctx->timer->print_at_exit = true;
    }
  });
  if (rc != AB2_OK) {
    fprintf(stderr, "ab2_context_create: %s\n", ctx->last_error.c_str());
    ab2_context_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return AB2_OK;
}

int ab2_context_destroy(ab2_context* ctx) {
  if (!ctx) return AB2_ERR_BAD_ARG;
  ctx_release(ctx);
  return AB2_OK;
}

const char* ab2_last_error_message(const ab2_context* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int ab2_context_stream(const ab2_context* ctx, void** stream) {
  if (!ctx || !stream) return AB2_ERR_BAD_ARG;
  *stream = (void*)ctx->stream;
  return AB2_OK;
}

int ab2_synchronize(ab2_context* ctx) {
  if (!ctx) return AB2_ERR_BAD_ARG;
  return guard(ctx, [&] { AB2_CUDA(cudaStreamSynchronize(ctx->stream)); });
}

int ab2_context_get_info(const ab2_context* ctx, ab2_context_info* info) {
  if (!ctx || !info) return AB2_ERR_BAD_ARG;
  info->device = ctx->device;
  info->num_sms = ctx->num_sms;
  info->reduction_threads = kThreads;
  info->reduction_max_blocks = std::min(kMaxRedBlocks, ctx->num_sms * (2048 / kThreads));
  return AB2_OK;
}

int ab2_context_launch_count(const ab2_context* ctx, long long* count) {
  if (!ctx || !count) return AB2_ERR_BAD_ARG;
  *count = ctx->launches;
  return AB2_OK;
}

// ---------------------------------------------------------------- vectors
int ab2_vector_create(ab2_context* ctx, int n, ab2_vector** out) {
  if (!ctx || !out || n < 0) return AB2_ERR_BAD_ARG;
  *out = nullptr;
  ab2_vector* v = new (std::nothrow) ab2_vector();
  if (!v) return AB2_ERR_OOM;
  v->ctx = ctx_retain(ctx);
  int rc = guard(ctx, [&] {
    v->n = n;
    v->cap = n;
    v->d = dev_alloc<double>(v->ctx, (size_t)n);
    AB2_CUDA(cudaMemsetAsync(v->d, 0, sizeof(double) * (size_t)std::max(n, 1), ctx->stream));
  });
  if (rc != AB2_OK) {
    ab2_vector_destroy(v);
    return rc;
  }
  *out = v;
  return AB2_OK;
}

int ab2_vector_destroy(ab2_vector* v) {
  if (!v) return AB2_ERR_BAD_ARG;
  ctx_quiesce(v->ctx);
  dev_free(v->ctx, v->d);
  ctx_release(v->ctx);
  delete v;
  return AB2_OK;
}

int ab2_vector_size(const ab2_vector* v, int* n) {
  if (!v || !n) return AB2_ERR_BAD_ARG;
  *n = v->n;
  return AB2_OK;
}

int ab2_vector_upload(ab2_context* ctx, ab2_vector* v, const double* host) {
  if (!ctx || !v || (!host && v->n)) return AB2_ERR_BAD_ARG;
  return guard(ctx, [&] {
    AB2_CUDA(cudaMemcpyAsync(v->d, host, sizeof(double) * (size_t)v->n, cudaMemcpyHostToDevice, ctx->stream));
  });
}

int ab2_vector_download(ab2_context* ctx, const ab2_vector* v, double* host) {
  if (!ctx || !v || (!host && v->n)) return AB2_ERR_BAD_ARG;
  return guard(ctx, [&] {
    AB2_CUDA(cudaMemcpyAsync(host, v->d, sizeof(double) * (size_t)v->n, cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int ab2_vector_device_ptr(const ab2_vector* v, void** dptr) {
  if (!v || !dptr) return AB2_ERR_BAD_ARG;
  *dptr = (void*)v->d;
  return AB2_OK;
}

// ---------------------------------------------------------------- BLAS-1
int ab2_axpy(ab2_context* ctx, double a, const ab2_vector* x, ab2_vector* y) {
  if (!ctx || !x || check_vec(y, x->n)) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-AXPY");
  return guard(ctx, [&] { op_axpy(ctx, x->n, a, x->d, y->d); });
}
int ab2_aypx(ab2_context* ctx, double a, ab2_vector* y, const ab2_vector* x) {
  if (!ctx || !x || check_vec(y, x->n)) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-AYPX");
  return guard(ctx, [&] { op_aypx(ctx, x->n, a, y->d, x->d); });
}
int ab2_copy(ab2_context* ctx, const ab2_vector* x, ab2_vector* y) {
  if (!ctx || !x || check_vec(y, x->n)) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-COPY");
  return guard(ctx, [&] { op_copy(ctx, x->n, x->d, y->d); });
}
int ab2_scal(ab2_context* ctx, double a, ab2_vector* x) {
  if (!ctx || !x) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-SCAL");
  return guard(ctx, [&] { op_scal(ctx, x->n, a, x->d); });
}
int ab2_pointwise_mult(ab2_context* ctx, const ab2_vector* x, const ab2_vector* y, ab2_vector* w) {
  if (!ctx || !x || check_vec(y, x->n) || check_vec(w, x->n)) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-PMULT");
  return guard(ctx, [&] { op_pmult(ctx, x->n, x->d, y->d, w->d); });
}
int ab2_assign(ab2_context* ctx, ab2_vector* x, double a) {
  if (!ctx || !x) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-ASSIGN");
  return guard(ctx, [&] { op_fill(ctx, x->n, a, x->d); });
}
int ab2_reciprocal(ab2_context* ctx, ab2_vector* x) {
  if (!ctx || !x) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-RECIPROCAL");
  return guard(ctx, [&] { op_reciprocal(ctx, x->n, x->d); });
}
int ab2_dot(ab2_context* ctx, const ab2_vector* x, const ab2_vector* y, double* result) {
  if (!ctx || !x || !result || check_vec(y, x->n)) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-DOT");
  return guard(ctx, [&] {
    RedSlot s = red_slot(ctx, 0);
    op_dot(ctx, x->n, x->d, y->d, s.result, 0);
    *result = read_scalar(ctx, s.result);
  });
}
int ab2_norm2(ab2_context* ctx, const ab2_vector* x, double* result) {
  if (!ctx || !x || !result) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-NORM2");
  return guard(ctx, [&] {
    RedSlot s = red_slot(ctx, 0);
    op_dot(ctx, x->n, x->d, x->d, s.result, 0);
    *result = std::sqrt(read_scalar(ctx, s.result));
  });
}
int ab2_norm1(ab2_context* ctx, const ab2_vector* x, double* result) {
  if (!ctx || !x || !result) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-NORM1");
  return guard(ctx, [&] {
    RedSlot s = red_slot(ctx, 0);
    op_norm1(ctx, x->n, x->d, s.result, 0);
    *result = read_scalar(ctx, s.result);
  });
}
int ab2_norm0(ab2_context* ctx, const ab2_vector* x, double* result) {
  if (!ctx || !x || !result) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-NORM0");
  return guard(ctx, [&] {
    RedSlot s = red_slot(ctx, 0);
    op_norm0(ctx, x->n, x->d, s.result, 0);
    *result = read_scalar(ctx, s.result);
  });
}

// ---------------------------------------------------------------- device scalars
int ab2_scalar_create(ab2_context* ctx, ab2_scalar** out) {
  if (!ctx || !out) return AB2_ERR_BAD_ARG;
  *out = nullptr;
  ab2_scalar* s = new (std::nothrow) ab2_scalar();
  if (!s) return AB2_ERR_OOM;
  s->ctx = ctx_retain(ctx);
  int rc = guard(ctx, [&] {
    s->d = dev_alloc<double>(s->ctx, 1);
    AB2_CUDA(cudaMemsetAsync(s->d, 0, sizeof(double), ctx->stream));
  });
  if (rc != AB2_OK) {
    ab2_scalar_destroy(s);
    return rc;
  }
  *out = s;
  return AB2_OK;
}
int ab2_scalar_destroy(ab2_scalar* s) {
  if (!s) return AB2_ERR_BAD_ARG;
  ctx_quiesce(s->ctx);
  dev_free(s->ctx, s->d);
  ctx_release(s->ctx);
  delete s;
  return AB2_OK;
}
int ab2_dot_async(ab2_context* ctx, const ab2_vector* x, const ab2_vector* y, ab2_scalar* result) {
  if (!ctx || !x || !result || check_vec(y, x->n)) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-DOT-F");
  return guard(ctx, [&] { op_dot(ctx, x->n, x->d, y->d, result->d, 0); });
}
int ab2_scalar_get(ab2_context* ctx, const ab2_scalar* s, double* value) {
  if (!ctx || !s || !value) return AB2_ERR_BAD_ARG;
  return guard(ctx, [&] { *value = read_scalar(ctx, s->d); });
}

// ---------------------------------------------------------------- phase timers
int ab2_context_set_phase_timing(ab2_context* ctx, int on) {
  if (!ctx) return AB2_ERR_BAD_ARG;
  return guard(ctx, [&] {
    const bool print = ctx->timer && ctx->timer->print_at_exit;
    if (ctx->timer) {
      AB2_CUDA(cudaStreamSynchronize(ctx->stream));
      delete ctx->timer;
      ctx->timer = nullptr;
    }
    if (on) {
      ctx->timer = new PhaseTimer();
      ctx->timer->print_at_exit = print;
    }
  });
}

int ab2_context_phase_times(ab2_context* ctx, ab2_phase_time* out, int cap, int* count) {
  if (!ctx || !count || cap < 0 || (cap > 0 && !out)) return AB2_ERR_BAD_ARG;
  *count = 0;
  if (!ctx->timer) return AB2_OK;
  return guard(ctx, [&] {
    PhaseTimer* t = ctx->timer;
    t->resolve();
    *count = (int)t->names.size();
    for (int i = 0; i < std::min(cap, *count); ++i) {
      std::memset(out[i].name, 0, sizeof(out[i].name));
      std::strncpy(out[i].name, t->names[(size_t)i].c_str(), sizeof(out[i].name) - 1);
      out[i].calls = t->calls[(size_t)i];
      out[i].ms = t->ms[(size_t)i];
    }
  });
}

}  // extern "C"

// ---------------------------------------------------------------- allocation-free dot
//
// Some callers cannot allocate device memory at the moment they need a dot
// product: a host that has handed all free HBM to another allocator (a caching
// pool that reserved it up front, so cudaMalloc would fail or fragment it), or
// a latency-critical loop that must not pay for cudaMalloc/cudaFree, which can
// block the calling thread and synchronise the whole device.  For them,
// ab2_dot_noalloc runs the same reduction kernel as ab2_dot with its block
// partials and arrival counter in the file-scope array below instead of a
// context's buffers.  The array exists once per GPU that loads libab2 and stays
// there until the process exits.
//
// The grid of this variant is ceil(n / kNoAllocChunk) blocks, so it writes at
// most kNoAllocSlots block partials for n up to kNoAllocSlots * kNoAllocChunk
// = 16,777,216 elements; larger n is rejected.  Inside the grid k_dot is the
// usual grid-stride loop: each thread sums the elements spaced one grid apart
// (up to 16 of them), then the block and finally the last block sum in fixed
// trees.  (ab2_dot's grid follows the context's reduction rule instead, so the
// two entry points may sum in different trees and agree to rounding, not bits.)
//
// All calls in the process share the array and it keeps the last call's
// contents; the counter, which must start at zero, is cleared on the caller's
// stream before every launch.  Calls that overlap on the GPU (issued on
// different streams, or from different host threads, without ordering between
// them) race on the shared array and give wrong results.
namespace {

constexpr int kNoAllocChunk = 4096;   // elements per block (256 threads x 16)
constexpr int kNoAllocSlots = 4096;   // block partials the scratch array holds
constexpr int kNoAllocMaxDevices = 64;

// [0, kNoAllocSlots): block partials; [kNoAllocSlots]: arrival counter (as
// unsigned int bits); the rest pads the array to a multiple of 256 bytes.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocSlots + 32];

struct NoAllocDevice {
  bool ready = false;
  double* scratch = nullptr;
};
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::atomic<int> g_noalloc_lock{0};

// Set-up, once per device and with that device current: the host-side name of
// g_noalloc_scratch is only a stand-in, so the device address is looked up
// with cudaGetSymbolAddress and cached.
int noalloc_scratch(int device, double** out) {
  while (g_noalloc_lock.exchange(1)) {
  }
  int rc = AB2_OK;
  NoAllocDevice& d = g_noalloc_dev[device];
  if (!d.ready) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) {
      rc = AB2_ERR_CUDA;
    } else {
      d.scratch = (double*)p;
      d.ready = true;
    }
  }
  *out = d.scratch;
  g_noalloc_lock.store(0);
  return rc;
}

}  // namespace

extern "C" int ab2_dot_noalloc(const double* x, const double* y, int n, double* result, void* stream) {
  if ((!x || !y) && n > 0) return AB2_ERR_BAD_ARG;
  if (!result || n < 0) return AB2_ERR_BAD_ARG;
  if ((long long)n > (long long)kNoAllocSlots * kNoAllocChunk) {
    fprintf(stderr, "ab2_dot_noalloc: n = %d exceeds the maximum of %d elements (%d block partials of %d)\n", n,
            kNoAllocSlots * kNoAllocChunk, kNoAllocSlots, kNoAllocChunk);
    return AB2_ERR_BAD_ARG;
  }
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kNoAllocMaxDevices) return AB2_ERR_CUDA;
  double* scratch = nullptr;
  int rc = noalloc_scratch(device, &scratch);
  if (rc != AB2_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + kNoAllocSlots);
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned int), s) != cudaSuccess) return AB2_ERR_CUDA;
  const int grid = std::max(1, (n + kNoAllocChunk - 1) / kNoAllocChunk);
  ab2::k_dot<<<grid, ab2::kThreads, 0, s>>>(n, x, y, scratch, counter, result);
  return cudaGetLastError() == cudaSuccess ? AB2_OK : AB2_ERR_CUDA;
}
