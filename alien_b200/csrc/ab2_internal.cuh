// ab2_internal.cuh -- internal types and helpers of libab2 (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "ab2.h"

namespace ab2 {

constexpr int kThreads = 256;          // default block size of streaming kernels
constexpr int kMaxRedBlocks = 2048;    // cap on blocks of one deterministic reduction
constexpr int kMaxRedComps = 4;        // values reduced together by one fused kernel
constexpr int kRedSlots = 8;           // independent reduction slots per context
constexpr int kEllSlice = 32;          // rows per sliced-ELL slice
constexpr int kStageCap = 2048;        // nnz staged in shared memory per CSR row block

// Thrown inside libab2 only; every ABI function catches and maps it to a code.
struct Error {
  int code;
  std::string msg;
};

struct PhaseTimer;  // context.cu

}  // namespace ab2

struct ab2_context {
  // Every object created on a context holds a reference, so objects may be
  // destroyed after ab2_context_destroy (as garbage-collected bindings do);
  // the context's memory goes when the last reference does.
  std::atomic<int> refs{1};
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  std::string last_error;
  long long launches = 0;
  // Deterministic reductions: block partials, arrival counters, results.
  double* d_partials = nullptr;       // kRedSlots * kMaxRedComps * kMaxRedBlocks
  unsigned int* d_counters = nullptr; // kRedSlots
  double* d_results = nullptr;        // kRedSlots * kMaxRedComps
  double* h_pinned = nullptr;         // 64 doubles of pinned staging
  // Host-side fault injection (ab2_context_inject_alloc_failure): the
  // fail_alloc_at-th device allocation from the call on fails as OOM.
  long long alloc_count = 0;
  long long fail_alloc_at = 0;
  // Phase timers (ab2_context_set_phase_timing, or AB2_PERF_TIMER=1): null when off.
  ab2::PhaseTimer* timer = nullptr;
};

struct ab2_vector {
  ab2_context* ctx = nullptr;
  int n = 0;
  double* d = nullptr;
  int cap = 0;  // doubles allocated (> n for distributed vectors: room for ghost values)
};

struct ab2_scalar {
  ab2_context* ctx = nullptr;
  double* d = nullptr;
};

struct ab2_matrix {
  ab2_context* ctx = nullptr;
  int n = 0;
  long long nnz = 0;
  int formats = 0;
  long long device_bytes = 0;
  // CSR (always present: ILU0, invdiag and L/U products use it)
  int* d_rp = nullptr;
  int* d_ci = nullptr;
  double* d_v = nullptr;
  int* d_dcol = nullptr;      // first position with col >= row (the diagonal)
  float* d_v32 = nullptr;     // FP32 copy when AB2_FMT_F32
  // row blocks for the shared-memory staged CSR kernel
  int n_row_blocks = 0;
  int* d_row_blocks = nullptr;
  // sliced ELL (BEllPack, 32-row slices, slot-major inside a slice)
  long long ell_stored = 0;
  int* d_ell_off = nullptr;   // n_slices + 1 prefix of slice widths
  int* d_ell_ci = nullptr;    // -1 marks padding
  double* d_ell_v = nullptr;
  float* d_ell_v32 = nullptr;
  // 7-point bands (AB2_FMT_STENCIL, kept when the profile is a 3-D 7-point
  // stencil numbered i + nx (j + ny k)): no column indices, the grid fixes
  // them.  Band-major, n values per band, 0 where a neighbour is outside the
  // grid.  7 bands (Lz, Ly, Lx, D, Ux, Uy, Uz), or 4 (D, Ux, Uy, Uz) when every
  // off-diagonal pair is bit-for-bit symmetric: the lower values are then read
  // from the neighbouring rows' upper bands.
  int st_nx = 0, st_ny = 0, st_nz = 0;
  int st_bands = 0;            // 0 (absent), 4 or 7
  double* d_st_v = nullptr;
  float* d_st_v32 = nullptr;   // FP32 copy when AB2_FMT_F32
  // host mirror of the profile for symbolic set-ups (ILU0 wavefronts, batch
  // checks), downloaded on first use by host_profile()
  mutable std::vector<int> h_rp, h_ci;
  mutable bool h_profile = false;
};

namespace ab2 {

// c + a*b and c - a*b with the product and the sum rounded separately: the
// rounding of Alien's `y += a*x` loops as its stock build compiles them
// (SpMV, addL/UMult, ILU0).  BLAS-1 updates use fma() instead, as CBLAS does.
__device__ __forceinline__ double mul_add_rn(double a, double b, double c) { return __dadd_rn(c, __dmul_rn(a, b)); }
__device__ __forceinline__ float mul_add_rn(float a, float b, float c) { return __fadd_rn(c, __fmul_rn(a, b)); }
__device__ __forceinline__ double mul_sub_rn(double a, double b, double c) { return __dsub_rn(c, __dmul_rn(a, b)); }
__device__ __forceinline__ float mul_sub_rn(float a, float b, float c) { return __fsub_rn(c, __fmul_rn(a, b)); }
// Single roundings for kernels templated on the value type.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    if (e == cudaErrorMemoryAllocation) throw Error{AB2_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(e)};
    throw Error{AB2_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
  }
}

#define AB2_CUDA(call) ::ab2::check_cuda((call), #call)

inline void check_launch(ab2_context* ctx, const char* what) {
  ctx->launches += 1;
  check_cuda(cudaGetLastError(), what);
}

inline void require(bool cond, const char* msg) {
  if (!cond) throw Error{AB2_ERR_BAD_ARG, msg};
}

// Device memory comes from the device's stream-ordered pool (cudaMallocAsync
// on the context's stream; the context raises the pool's release threshold so
// freed blocks stay cached for the next solver instead of going back to the
// driver).  dev_alloc waits for the stream, so the block is valid for any use
// -- including synchronous copies on other streams -- when it returns;
// dev_free is ordered after all work already queued on the stream.
template <class T>
T* dev_alloc(ab2_context* ctx, size_t count, long long* accounted = nullptr) {
  T* p = nullptr;
  if (count == 0) count = 1;
  if (ctx->fail_alloc_at > 0 && ++ctx->alloc_count == ctx->fail_alloc_at) {
    ctx->fail_alloc_at = 0;
    throw Error{AB2_ERR_OOM, "device allocation failed (injected)"};
  }
  check_cuda(cudaMallocAsync((void**)&p, count * sizeof(T), ctx->stream), "cudaMallocAsync");
  check_cuda(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
  if (accounted) *accounted += (long long)(count * sizeof(T));
  return p;
}

inline void dev_free(ab2_context* ctx, void* p) {
  if (p) cudaFreeAsync(p, ctx->stream);
}

// Context references (see ab2_context::refs).
inline ab2_context* ctx_retain(ab2_context* ctx) {
  ctx->refs.fetch_add(1);
  return ctx;
}
void ctx_release(ab2_context* ctx);  // frees the context with its last reference

// Makes ctx's device current and waits for its stream: every destroy starts here.
inline void ctx_quiesce(ab2_context* ctx) {
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
}

// Unsigned division by a divisor fixed at set-up, as a multiply-high and a
// shift (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, the round-up multiplier): with l = ceil(log2 d)
// and m = floor(2^32 (2^l - d) / d) + 1, n / d = (umulhi(n, m) + n) >> l for
// every n < 2^31 (the sum then stays below 2^32).
struct FastDiv {
  unsigned d = 1, m = 1, l = 0;
  FastDiv() = default;
  explicit FastDiv(unsigned div) : d(div) {
    while ((1ull << l) < (unsigned long long)div) ++l;
    m = (unsigned)(((1ull << 32) * ((1ull << l) - div)) / div + 1);
  }
  __host__ __device__ __forceinline__ unsigned div(unsigned n) const {
#ifdef __CUDA_ARCH__
    return (__umulhi(n, m) + n) >> l;
#else
    return (unsigned)((((unsigned long long)n * m) >> 32) + n) >> l;
#endif
  }
};

inline int grid_for(long long n, int threads = kThreads, int cap = 148 * 32) {
  long long g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

// Phase timers: device time of each ABI operation by phase name (the
// reference's StdTimer sentries, e.g. "CSR-SPMV"), from CUDA events recorded
// on the context's stream around the call and resolved when read.
void phase_begin(ab2_context* ctx, const char* name, int* token);
void phase_end(ab2_context* ctx, int token);
struct PhaseScope {
  ab2_context* ctx;
  int tok = -1;
  PhaseScope(ab2_context* c, const char* name) : ctx(c) {
    if (c && c->timer) phase_begin(c, name, &tok);
  }
  ~PhaseScope() {
    if (tok >= 0) phase_end(ctx, tok);
  }
  PhaseScope(const PhaseScope&) = delete;
  PhaseScope& operator=(const PhaseScope&) = delete;
};

// Runs f, mapping exceptions to ABI codes and recording the message on ctx.
template <class F>
int guard(ab2_context* ctx, F&& f) {
  try {
    f();
    return AB2_OK;
  } catch (const Error& e) {
    if (ctx) ctx->last_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    if (ctx) ctx->last_error = "host allocation failed";
    return AB2_ERR_OOM;
  } catch (const std::exception& e) {
    if (ctx) ctx->last_error = e.what();
    return AB2_ERR_CUDA;
  } catch (...) {
    if (ctx) ctx->last_error = "unknown failure";
    return AB2_ERR_CUDA;
  }
}

// ----------------------------------------------------------------- internal ops
// Plain device-pointer versions of the algebra, shared by the ABI entry points,
// the preconditioners and the solvers.  All enqueue on ctx->stream.
struct RedSlot {
  double* partials;
  unsigned int* counter;
  double* result;  // kMaxRedComps doubles on the device
};
RedSlot red_slot(ab2_context* ctx, int slot);
// Blocks of every grid reduction over n values (256 threads each).
int red_grid(const ab2_context* ctx, int n);

void op_fill(ab2_context* ctx, int n, double a, double* x);
void op_copy(ab2_context* ctx, int n, const double* x, double* y);
void op_axpy(ab2_context* ctx, int n, double a, const double* x, double* y);
void op_aypx(ab2_context* ctx, int n, double a, double* y, const double* x);
void op_scal(ab2_context* ctx, int n, double a, double* x);
void op_pmult(ab2_context* ctx, int n, const double* x, const double* y, double* w);
void op_reciprocal(ab2_context* ctx, int n, double* x);
// out[0] = x.y (device pointer, written by the last block)
void op_dot(ab2_context* ctx, int n, const double* x, const double* y, double* out, int slot = 0);
void op_norm0(ab2_context* ctx, int n, const double* x, double* out, int slot = 0);
void op_norm1(ab2_context* ctx, int n, const double* x, double* out, int slot = 0);
double read_scalar(ab2_context* ctx, const double* d);
// Precision conversions (round to nearest; widening is exact).
void op_to_f32(ab2_context* ctx, long long m, const double* a, float* b);
void op_to_f64(ab2_context* ctx, long long m, const float* a, double* b);

// SpMV family (spmv.cu)
void op_spmv(ab2_context* ctx, const ab2_matrix* A, const double* x, double* y, int variant);
void op_add_lu_mult(ab2_context* ctx, const ab2_matrix* A, double alpha, const double* x, double* y, bool lower);
void op_inv_diag(ab2_context* ctx, const ab2_matrix* A, double* inv);
void op_diagonal(ab2_context* ctx, const ab2_matrix* A, double* d);
void op_mult_inv_diag(ab2_context* ctx, const ab2_matrix* A, double* y);
int resolve_variant(const ab2_matrix* A, int variant);
// The 3-D 7-point geometry of A's profile (rows i + nx (j + ny k) holding
// exactly their in-grid neighbours in ascending columns): true and nx, ny, nz
// when it has one (nx, ny, nz >= 2).  Device-side check; synchronises.
bool stencil_geometry(ab2_context* ctx, const ab2_matrix* A, int* nx, int* ny, int* nz);
// Fills A->h_rp / A->h_ci from the device once (synchronises the stream).
void host_profile(const ab2_matrix* A);
// A sliced-ELL copy of A's values in FP32 with S-row slices (S = 16, 32 or
// 64), kept by the caller (the batched solver's autotuner); free_ell frees it.
struct EllLayout {
  int S = 0;
  int* off = nullptr;  // n_slices + 1
  int* ci = nullptr;   // -1 marks padding
  float* v = nullptr;
  long long stored = 0;
};
EllLayout build_ell_f32(ab2_context* ctx, const ab2_matrix* A, int S);
void free_ell(ab2_context* ctx, EllLayout& e);

}  // namespace ab2
