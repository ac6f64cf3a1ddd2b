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
//
// The engine (Krylov<T>) is templated on the value type: T = double is the
// drop-in solver; T = float is the inner solver of the mixed-precision
// refinement (mixed.cu), with FP32 values, FP32 accumulation in every dot and
// FP32 scalars.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <unordered_map>

#include "ab2_internal.cuh"
#include "krylov.cuh"
#include "precond.cuh"
#include "reduce.cuh"
#include "spmv_view.cuh"

namespace ab2 {

namespace {

constexpr int kCtlThreads = 256;

template <class T>
__device__ __forceinline__ void record(SolveStateT<T>* st, T v) {
  if (st->hist_len < st->hist_cap) st->hist[st->hist_len] = v;
  st->hist_len += 1;
}

// Iteration::stop(r) with the dot product already computed.
template <class T>
__device__ __forceinline__ bool stop_test(SolveStateT<T>* st, T dot_rr) {
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

// A reduction slot's buffers seen as T (FP32 partials fit the FP64 slots).
template <class T>
struct Red {
  T* partials;
  unsigned int* counter;
  T* result;
};
template <class T>
Red<T> red_of(ab2_context* ctx, int slot) {
  RedSlot s = red_slot(ctx, slot);
  return Red<T>{reinterpret_cast<T*>(s.partials), s.counter, reinterpret_cast<T*>(s.result)};
}

// b.b into st->nrm2_b: the same tree as op_dot.  With a weight w (the mixed
// solver's scaled Jacobi form): sum (b_i w_i) b_i.
template <class T>
__global__ void __launch_bounds__(kCtlThreads) k_bb(int n, const T* __restrict__ b, const T* __restrict__ w,
                                                    SolveStateT<T>* st, Red<T> red) {
  T acc[1] = {T(0)};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc[0] = fma_rn(w ? mul_rn(b[i], w[i]) : b[i], b[i], acc[0]);
  if (grid_reduce<1>(acc, red.partials, red.counter, red.result)) st->nrm2_b = red.result[0];
}

template <class T>
__global__ void k_state_init(SolveStateT<T>* st, T tol, int max_iter, T* x, const T* b, T* hist, int hist_cap) {
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
  st->x_pending = 0;
  st->bodies = 0;
  st->rho = st->rho1 = st->den = st->alpha = st->beta = st->omega = st->rr_r = 0;
}

// r = b - A x (copy b, mult A x, axpy -1).  With r0 != nullptr (BiCGStab):
// also r0 = r and rho1 = r.r0.
template <class View, class T>
__global__ void __launch_bounds__(kCtlThreads) k_residual(int n, View A, SolveStateT<T>* st, T* r, T* r0, Red<T> red) {
  const T* x = st->x;
  const T* b = st->b;
  T acc[1] = {T(0)};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const T ax = A.row(row, x);
    const T rv = fma_rn(T(-1), ax, b[row]);
    r[row] = rv;
    if (r0) {
      r0[row] = rv;
      acc[0] = fma_rn(rv, rv, acc[0]);
    }
  }
  if (grid_reduce<1>(acc, red.partials, red.counter, red.result)) {
    if (r0) st->rho1 = red.result[0];
  }
}

// ------------------------------------------------------------------ CG
// rho1 = r.z ; beta = rho1/rho (CG.h:117-118, the code names it alpha)
template <class T>
__global__ void __launch_bounds__(kCtlThreads) k_cg_rz(int n, const T* __restrict__ r, const T* __restrict__ z,
                                                       SolveStateT<T>* st, Red<T> red) {
  T acc[1] = {T(0)};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[0] = fma_rn(r[i], z[i], acc[0]);
  if (grid_reduce<1>(acc, red.partials, red.counter, red.result)) {
    st->rho1 = red.result[0];
    st->beta = st->first ? T(0) : st->rho1 / st->rho;
  }
}

// p = z (first step, CG.h:89) or z += beta p ; p = z (CG.h:119-120).
// Element-wise, so the thread that computes an element does not matter: 16
// bytes (4 floats, 2 doubles) per thread and access, then the tail.
template <class T>
__global__ void k_cg_p(int n, const T* __restrict__ z, T* __restrict__ p, const SolveStateT<T>* st) {
  const T beta = st->beta;
  const int first = st->first;
  using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  constexpr int W = 16 / (int)sizeof(T);
  const int nv = n / W;
  const V* __restrict__ zv = reinterpret_cast<const V*>(z);
  V* __restrict__ pv = reinterpret_cast<V*>(p);
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int i = t0; i < nv; i += stride) {
    V a = zv[i];
    if (!first) {
      const V b = pv[i];
      T* pa = reinterpret_cast<T*>(&a);
      const T* pb = reinterpret_cast<const T*>(&b);
#pragma unroll
      for (int u = 0; u < W; ++u) pa[u] = fma_rn(beta, pb[u], pa[u]);
    }
    pv[i] = a;
  }
  for (int i = nv * W + t0; i < n; i += stride) p[i] = first ? z[i] : fma_rn(beta, p[i], z[i]);
}

// k_cg_p with the owed x update of the previous iteration in the same pass
// (x += alpha p_old with the p about to be replaced: the same values and the
// same rounding as updating x in k_cgj_update, one read of p less).  Nothing
// once the solve is done (the host-driven loop queues bodies past the end).
template <class T>
__global__ void k_cg_px(int n, const T* __restrict__ z, T* __restrict__ p, const SolveStateT<T>* st) {
  if (st->done) return;
  const T beta = st->beta, alpha = st->alpha;
  const int first = st->first, owed = st->x_pending;
  T* __restrict__ x = st->x;
  using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  constexpr int W = 16 / (int)sizeof(T);
  const int nv = n / W;
  const V* __restrict__ zv = reinterpret_cast<const V*>(z);
  V* __restrict__ pv = reinterpret_cast<V*>(p);
  V* __restrict__ xv = reinterpret_cast<V*>(x);
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int i = t0; i < nv; i += stride) {
    V a = zv[i];
    if (!first) {
      const V b = pv[i];
      T* pa = reinterpret_cast<T*>(&a);
      const T* pb = reinterpret_cast<const T*>(&b);
      if (owed) {
        V c = xv[i];
        T* pc = reinterpret_cast<T*>(&c);
#pragma unroll
        for (int u = 0; u < W; ++u) pc[u] = fma_rn(alpha, pb[u], pc[u]);
        xv[i] = c;
      }
#pragma unroll
      for (int u = 0; u < W; ++u) pa[u] = fma_rn(beta, pb[u], pa[u]);
    }
    pv[i] = a;
  }
  for (int i = nv * W + t0; i < n; i += stride) {
    if (!first && owed) x[i] = fma_rn(alpha, p[i], x[i]);
    p[i] = first ? z[i] : fma_rn(beta, p[i], z[i]);
  }
}

// After the loop: the last iteration's owed x += alpha p.
template <class T>
__global__ void k_cg_xfix(int n, const T* __restrict__ p, const SolveStateT<T>* st) {
  if (!st->x_pending) return;
  const T alpha = st->alpha;
  T* __restrict__ x = st->x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = fma_rn(alpha, p[i], x[i]);
}

// q = A p ; den = q.p.  VB logical blocks of the reduction grid per block
// (grid_reduce_v): a thread walks its VB logical threads' rows side by side,
// so at any time the GPU works on one contiguous stretch of rows.
template <class View, class T, int VB = 1>
__global__ void __launch_bounds__(kCtlThreads) k_cg_spmv(int n, View A, const T* __restrict__ p, T* __restrict__ q,
                                                         SolveStateT<T>* st, Red<T> red) {
  T acc[VB][1] = {};
  const int lstride = gridDim.x * blockDim.x;  // between a thread's logical threads
  for (int base = blockIdx.x * blockDim.x + threadIdx.x; base < n; base += VB * lstride) {
#pragma unroll
    for (int v = 0; v < VB; ++v) {
      const int row = base + v * lstride;
      if (row < n) {
        const T qv = A.row(row, p);
        q[row] = qv;
        acc[v][0] = fma_rn(qv, p[row], acc[v][0]);
      }
    }
  }
  if (grid_reduce_v<1, VB>(acc, red.partials, red.counter, red.result)) st->den = red.result[0];
}

// k_cg_spmv for FP32 7-point bands in their symmetric form (StencilView<float,
// true, UNIT>), four consecutive rows of one grid line a thread: 16-byte loads
// of p, the bands and q, the row coordinates divided out once per four rows,
// and two sweeps' loads in flight before either is used (one row a thread,
// FP32 moves half the bytes of FP64 per load and the kernel waited on memory
// latency at 0.56 of HBM bandwidth).  Needs nx % 4 == 0 (so the four rows
// share j and k, and p +- nx, +- nx ny stay 16-byte aligned).  Each row sums
// the terms of StencilView::row_f in the same order, so q is bit-identical;
// the rows of logical thread g of the G-block reduction grid are k_cg_spmv's
// (g, g + 256 G, ...), thread t carries logical threads 4t .. 4t + 3 (their
// sweeps in order), and grid_reduce_r reduces their p.q partials with
// k_cg_spmv's tree.
struct BandRows4 {  // one sweep of a thread: four rows' operands
  float4 pc, uxc, pym, uym, pyp, uyc, pzm, uzm, pzp, uzc, dg;
  float pl, uxl, pr;
  int r0;
  bool xl, xr, ym, yp, zm, zp;
};

template <bool UNIT>
__device__ __forceinline__ BandRows4 band_rows4_load(const StencilView<float, true, UNIT>& A, const float* __restrict__ p,
                                                     const float* __restrict__ ux, const float* __restrict__ uy,
                                                     const float* __restrict__ uz, int r0) {
  auto ld4 = [](const float* a) { return __ldg(reinterpret_cast<const float4*>(a)); };
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  const int nx = A.nx, ny = A.ny, nz = A.nz, sy = nx, sz = nx * ny;
  BandRows4 o;
  o.r0 = r0;
  const unsigned qq = A.fx.div((unsigned)r0);
  const int i0 = r0 - (int)qq * nx;
  const int k = (int)A.fy.div(qq);
  const int j = (int)qq - k * ny;
  o.xl = i0 > 0;
  o.xr = i0 + 4 < nx;
  o.ym = j > 0;
  o.yp = j < ny - 1;
  o.zm = k > 0;
  o.zp = k < nz - 1;
  o.pc = ld4(p + r0);
  o.uxc = ld4(ux + r0);
  o.pl = o.xl ? __ldg(p + r0 - 1) : 0.f;
  o.uxl = o.xl ? __ldg(ux + r0 - 1) : 0.f;
  o.pr = o.xr ? __ldg(p + r0 + 4) : 0.f;
  o.pym = o.ym ? ld4(p + r0 - sy) : z4;
  o.uym = o.ym ? ld4(uy + r0 - sy) : z4;
  o.pyp = o.yp ? ld4(p + r0 + sy) : z4;
  o.uyc = o.yp ? ld4(uy + r0) : z4;
  o.pzm = o.zm ? ld4(p + r0 - sz) : z4;
  o.uzm = o.zm ? ld4(uz + r0 - sz) : z4;
  o.pzp = o.zp ? ld4(p + r0 + sz) : z4;
  o.uzc = o.zp ? ld4(uz + r0) : z4;
  o.dg = UNIT ? make_float4(1.f, 1.f, 1.f, 1.f) : ld4(A.v + r0);
  return o;
}

// q for the four rows (stored) and their p.q terms added to acc[u][0].
__device__ __forceinline__ void band_rows4_sum(const BandRows4& o, float* __restrict__ q, float (&acc)[4][1]) {
  const float P[6] = {o.pl, o.pc.x, o.pc.y, o.pc.z, o.pc.w, o.pr};  // p at i0 - 1 .. i0 + 4
  const float UX[5] = {o.uxl, o.uxc.x, o.uxc.y, o.uxc.z, o.uxc.w};  // ux at r0 - 1 .. r0 + 3
  const float PYM[4] = {o.pym.x, o.pym.y, o.pym.z, o.pym.w}, UYM[4] = {o.uym.x, o.uym.y, o.uym.z, o.uym.w};
  const float PYP[4] = {o.pyp.x, o.pyp.y, o.pyp.z, o.pyp.w}, UYC[4] = {o.uyc.x, o.uyc.y, o.uyc.z, o.uyc.w};
  const float PZM[4] = {o.pzm.x, o.pzm.y, o.pzm.z, o.pzm.w}, UZM[4] = {o.uzm.x, o.uzm.y, o.uzm.z, o.uzm.w};
  const float PZP[4] = {o.pzp.x, o.pzp.y, o.pzp.z, o.pzp.w}, UZC[4] = {o.uzc.x, o.uzc.y, o.uzc.z, o.uzc.w};
  const float DG[4] = {o.dg.x, o.dg.y, o.dg.z, o.dg.w};
  float qv[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    float a = 0.f;
    if (o.zm) a = mul_add_rn(UZM[u], PZM[u], a);
    if (o.ym) a = mul_add_rn(UYM[u], PYM[u], a);
    if (u > 0 || o.xl) a = mul_add_rn(UX[u], P[u], a);
    a = mul_add_rn(DG[u], P[u + 1], a);
    if (u < 3 || o.xr) a = mul_add_rn(UX[u + 1], P[u + 2], a);
    if (o.yp) a = mul_add_rn(UYC[u], PYP[u], a);
    if (o.zp) a = mul_add_rn(UZC[u], PZP[u], a);
    qv[u] = a;
    acc[u][0] = fma_rn(a, P[u + 1], acc[u][0]);
  }
  *reinterpret_cast<float4*>(q + o.r0) = make_float4(qv[0], qv[1], qv[2], qv[3]);
}

template <bool UNIT>
__global__ void __launch_bounds__(kCtlThreads) k_cg_spmv_x4(int n, StencilView<float, true, UNIT> A,
                                                            const float* __restrict__ p, float* __restrict__ q,
                                                            SolveStateT<float>* st, Red<float> red, int G) {
  const int S = G * kCtlThreads;  // rows per sweep of the logical grid
  const int t4 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  const size_t N = (size_t)n;
  const float* __restrict__ ux = A.v + (UNIT ? 0 : N);
  const float* __restrict__ uy = ux + N;
  const float* __restrict__ uz = uy + N;
  float acc[4][1] = {{0.f}, {0.f}, {0.f}, {0.f}};
  if (t4 < S) {
    for (int r0 = t4; r0 < n; r0 += 2 * S) {
      const bool two = r0 + S < n;
      const BandRows4 a = band_rows4_load(A, p, ux, uy, uz, r0);
      BandRows4 b;
      if (two) b = band_rows4_load(A, p, ux, uy, uz, r0 + S);
      band_rows4_sum(a, q, acc);
      if (two) band_rows4_sum(b, q, acc);
    }
  }
  if (grid_reduce_r<1, 4>(acc, G, red.partials, red.counter, red.result)) st->den = red.result[0];
}

// alpha = rho1/den ; x += alpha p ; r -= alpha q ; then the loop's stop test on r.
// p1 != nullptr: p is double-buffered (k_cgj_spmv formed it), and the buffer
// it wrote is p0 or p1 by the body count's parity.
template <class T>
__global__ void __launch_bounds__(kCtlThreads) k_cg_update(int n, const T* __restrict__ p0, const T* __restrict__ p1,
                                                           const T* __restrict__ q, T* __restrict__ r,
                                                           SolveStateT<T>* st, Red<T> red,
                                                           cudaGraphConditionalHandle h, int use_graph) {
  if (st->done) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_loop(h, use_graph, 0);
    return;
  }
  const T* __restrict__ p = (p1 && !(st->bodies & 1)) ? p1 : p0;
  const T den = st->den;
  const bool ok = den != T(0);
  const T alpha = ok ? st->rho1 / den : T(0);
  T* x = st->x;
  T acc[1] = {T(0)};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T rv = r[i];
    if (ok) {
      x[i] = fma_rn(alpha, p[i], x[i]);
      rv = fma_rn(-alpha, q[i], rv);
      r[i] = rv;
    }
    acc[0] = fma_rn(rv, rv, acc[0]);
  }
  if (grid_reduce<1>(acc, red.partials, red.counter, red.result)) {
    const T rr = red.result[0];
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

// ------------------------------------------------------------------ CG with Diag or no preconditioner
// The same iteration in two kernels instead of five (precond, r.z, p, SpMV,
// update): the update kernel also applies the Jacobi scaling and reduces r.z
// for the next iteration beside r.r, and the SpMV kernel forms p = z + beta p
// on the fly, reading the previous p from the other of two buffers (a row's
// neighbours must still see the old values).  Every element is computed with
// the operations, operands and order of the five-kernel form and every dot in
// the same grid and tree, so the iterates are bit-identical; the loop moves
// 96 n instead of 128 n vector bytes and launches 2 kernels per iteration.
// The p buffers alternate with the body count (bodies & 1).

// Before the loop: z = D^-1 r (inv = nullptr: z = r, and z is not stored:
// the other kernels then read r in its place), rho1 = r.z, beta = 0.
template <class T>
__global__ void __launch_bounds__(kCtlThreads) k_cgj_start(int n, const T* __restrict__ r, const T* __restrict__ inv,
                                                           T* __restrict__ z, SolveStateT<T>* st, Red<T> red) {
  T acc[1] = {T(0)};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T rv = r[i];
    const T zv = inv ? mul_rn(inv[i], rv) : rv;
    if (inv) z[i] = zv;
    acc[0] = fma_rn(rv, zv, acc[0]);
  }
  if (grid_reduce<1>(acc, red.partials, red.counter, red.result)) {
    st->rho1 = red.result[0];
    st->beta = T(0);
  }
}

// p = first ? z : z + beta p_old (into the other buffer) ; q = A p ; den = q.p
// (VB: as k_cg_spmv)
template <class View, class T, int VB = 1>
__global__ void __launch_bounds__(kCtlThreads) k_cgj_spmv(int n, View A, const T* __restrict__ z, T* p0, T* p1,
                                                          T* __restrict__ q, SolveStateT<T>* st, Red<T> red) {
  if (st->done) return;  // every block returns: the reduction below is skipped as a whole
  const int par = st->bodies & 1;
  const T* __restrict__ po = par ? p1 : p0;
  T* __restrict__ pn = par ? p0 : p1;
  const T beta = st->beta;
  const int first = st->first;
  auto pval = [&](int c) { return first ? z[c] : fma_rn(beta, po[c], z[c]); };
  T acc[VB][1] = {};
  const int lstride = gridDim.x * blockDim.x;  // between a thread's logical threads
  for (int base = blockIdx.x * blockDim.x + threadIdx.x; base < n; base += VB * lstride) {
#pragma unroll
    for (int v = 0; v < VB; ++v) {
      const int row = base + v * lstride;
      if (row < n) {
        const T qv = A.row_f(row, pval);
        const T pr = pval(row);
        pn[row] = pr;
        q[row] = qv;
        acc[v][0] = fma_rn(qv, pr, acc[v][0]);
      }
    }
  }
  if (grid_reduce_v<1, VB>(acc, red.partials, red.counter, red.result)) st->den = red.result[0];
}

// The scalar part of a Jacobi-CG update, in the last block: the state after
// r.r = rr and r.z = rz (CG.h:96-139).
template <class T, bool DEFER_X>
__device__ __forceinline__ void cgj_update_scalars(SolveStateT<T>* st, T rr, T rz, bool ok, T alpha,
                                                   cudaGraphConditionalHandle h, int use_graph) {
  st->bodies += 1;
  if constexpr (DEFER_X) st->x_pending = ok ? 1 : 0;
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
    // the next iteration's rho1 = r.z and beta = rho1 / rho (CG.h:117-118)
    st->rho1 = rz;
    st->beta = rz / st->rho;
    if (stop_test(st, rr)) st->done = 1;
  }
  set_loop(h, use_graph, !st->done);
}

// alpha = rho1/den ; x += alpha p ; r -= alpha q ; z = D^-1 r ; r.r (stop test) and r.z (next rho1).
// inv = nullptr: z = r, not stored (z may be null).  w: the stop test sums
// (r_i w_i) r_i instead (the scaled Jacobi form's unscaled residual norm).
// DEFER_X: x is not touched here; x += alpha p is owed (x_pending) and paid
// by the next k_cg_px, which reads p anyway, or by k_cg_xfix after the loop.
template <class T, bool DEFER_X = false>
__global__ void __launch_bounds__(kCtlThreads, 8) k_cgj_update(int n, const T* p0, const T* p1, const T* __restrict__ q,
                                                            T* __restrict__ r, T* __restrict__ z,
                                                            const T* __restrict__ inv, const T* __restrict__ w,
                                                            SolveStateT<T>* st, Red<T> red,
                                                            cudaGraphConditionalHandle h, int use_graph) {
  if (st->done) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_loop(h, use_graph, 0);
    return;
  }
  const T* __restrict__ p = (st->bodies & 1) ? p0 : p1;  // the buffer k_cgj_spmv wrote
  const T den = st->den;
  const bool ok = den != T(0);
  const T alpha = ok ? st->rho1 / den : T(0);
  T* x = st->x;
  (void)x;
  T acc[2] = {T(0), T(0)};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T rv = r[i];
    if (ok) {
      if constexpr (!DEFER_X) x[i] = fma_rn(alpha, p[i], x[i]);
      rv = fma_rn(-alpha, q[i], rv);
      r[i] = rv;
    }
    acc[0] = fma_rn(w ? mul_rn(rv, w[i]) : rv, rv, acc[0]);
    const T zv = inv ? mul_rn(inv[i], rv) : rv;
    if (inv) z[i] = zv;
    acc[1] = fma_rn(rv, zv, acc[1]);
  }
  if (grid_reduce<2>(acc, red.partials, red.counter, red.result))
    cgj_update_scalars<T, DEFER_X>(st, red.result[0], red.result[1], ok, alpha, h, use_graph);
}

// k_cgj_update<float> for n % 4 == 0: four consecutive elements a thread
// (16-byte accesses).  Logical thread g of the G-block reduction grid owns
// elements g, g + 256 G, ... as in k_cgj_update; thread t carries logical
// threads 4t .. 4t + 3, and grid_reduce_r sums their r.r and r.z partials
// with k_cgj_update's tree, so every value and scalar is bit-identical.
template <bool DEFER_X>
__global__ void __launch_bounds__(kCtlThreads) k_cgj_update_x4(int n, const float* p0, const float* p1,
                                                               const float* __restrict__ q, float* __restrict__ r,
                                                               float* __restrict__ z, const float* __restrict__ inv,
                                                               const float* __restrict__ w, SolveStateT<float>* st,
                                                               Red<float> red, cudaGraphConditionalHandle h,
                                                               int use_graph, int G) {
  if (st->done) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_loop(h, use_graph, 0);
    return;
  }
  const float* __restrict__ p = (st->bodies & 1) ? p0 : p1;
  const float den = st->den;
  const bool ok = den != 0.f;
  const float alpha = ok ? st->rho1 / den : 0.f;
  float* x = st->x;
  (void)x;
  (void)p;
  const int S = G * kCtlThreads;
  const int t4 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  float acc[4][2] = {};
  auto ld4 = [](const float* a) { return *reinterpret_cast<const float4*>(a); };
  if (t4 < S) {
    for (int i = t4; i < n; i += 2 * S) {
      const bool two = i + S < n;
      const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
      float4 rv[2] = {z4, z4}, qv[2] = {z4, z4}, wv[2] = {z4, z4}, iv[2] = {z4, z4}, pv[2] = {z4, z4},
             xv[2] = {z4, z4};
#pragma unroll
      for (int h2 = 0; h2 < 2; ++h2) {
        if (h2 == 1 && !two) break;
        const int e = i + h2 * S;
        rv[h2] = ld4(r + e);
        if (ok) {
          qv[h2] = ld4(q + e);
          if constexpr (!DEFER_X) {
            pv[h2] = ld4(p + e);
            xv[h2] = ld4(x + e);
          }
        }
        if (w) wv[h2] = ld4(w + e);
        if (inv) iv[h2] = ld4(inv + e);
      }
#pragma unroll
      for (int h2 = 0; h2 < 2; ++h2) {
        if (h2 == 1 && !two) break;
        const int e = i + h2 * S;
        float R[4] = {rv[h2].x, rv[h2].y, rv[h2].z, rv[h2].w};
        const float Q[4] = {qv[h2].x, qv[h2].y, qv[h2].z, qv[h2].w};
        const float W4[4] = {wv[h2].x, wv[h2].y, wv[h2].z, wv[h2].w};
        const float I4[4] = {iv[h2].x, iv[h2].y, iv[h2].z, iv[h2].w};
        float Z[4];
        if (ok) {
          if constexpr (!DEFER_X) {
            const float P4[4] = {pv[h2].x, pv[h2].y, pv[h2].z, pv[h2].w};
            float X[4] = {xv[h2].x, xv[h2].y, xv[h2].z, xv[h2].w};
#pragma unroll
            for (int u = 0; u < 4; ++u) X[u] = fma_rn(alpha, P4[u], X[u]);
            *reinterpret_cast<float4*>(x + e) = make_float4(X[0], X[1], X[2], X[3]);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) R[u] = fma_rn(-alpha, Q[u], R[u]);
          *reinterpret_cast<float4*>(r + e) = make_float4(R[0], R[1], R[2], R[3]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          acc[u][0] = fma_rn(w ? mul_rn(R[u], W4[u]) : R[u], R[u], acc[u][0]);
          Z[u] = inv ? mul_rn(I4[u], R[u]) : R[u];
          acc[u][1] = fma_rn(R[u], Z[u], acc[u][1]);
        }
        if (inv) *reinterpret_cast<float4*>(z + e) = make_float4(Z[0], Z[1], Z[2], Z[3]);
      }
    }
  }
  if (grid_reduce_r<2, 4>(acc, G, red.partials, red.counter, red.result))
    cgj_update_scalars<float, DEFER_X>(st, red.result[0], red.result[1], ok, alpha, h, use_graph);
}

// ------------------------------------------------------------------ BiCGStab
// p = r (first) or p = r + beta (p - omega v)  (BiCGStab.h:273-276, three BLAS-1 calls)
template <class T>
__global__ void k_bicg_p(int n, const T* __restrict__ r, const T* __restrict__ v, T* __restrict__ p,
                         const SolveStateT<T>* st) {
  const int first = st->first;
  const T beta = st->beta, omega = st->omega;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (first) p[i] = r[i];
    else p[i] = add_rn(r[i], mul_rn(beta, fma_rn(-omega, v[i], p[i])));
  }
}

// v = A phat ; alpha = rho1 / (v.r0), breakdown "alpha" on zero
template <class View, class T>
__global__ void __launch_bounds__(kCtlThreads) k_bicg_v(int n, View A, const T* __restrict__ phat,
                                                        const T* __restrict__ r0, T* __restrict__ v, SolveStateT<T>* st,
                                                        Red<T> red) {
  T acc[1] = {T(0)};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const T vv = A.row(row, phat);
    v[row] = vv;
    acc[0] = fma_rn(vv, r0[row], acc[0]);
  }
  if (grid_reduce<1>(acc, red.partials, red.counter, red.result)) {
    const T d = red.result[0];
    if (d == T(0)) {
      st->error = AB2_ERR_BREAKDOWN;
      st->breakdown = AB2_BREAKDOWN_ALPHA;
      st->done = 1;
    } else {
      st->alpha = st->rho1 / d;
    }
  }
}

// s = r - alpha v ; stop test on s (exit with x += alpha phat) ; also r.r for the first step
template <class T>
__global__ void __launch_bounds__(kCtlThreads) k_bicg_s(int n, const T* __restrict__ r, const T* __restrict__ v,
                                                        T* __restrict__ s, SolveStateT<T>* st, Red<T> red) {
  const bool live = !st->done;
  const T alpha = st->alpha;
  T acc[2] = {T(0), T(0)};
  if (live) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      const T rv = r[i];
      const T sv = fma_rn(-alpha, v[i], rv);
      s[i] = sv;
      acc[0] = fma_rn(sv, sv, acc[0]);
      acc[1] = fma_rn(rv, rv, acc[1]);
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
template <class View, class T>
__global__ void __launch_bounds__(kCtlThreads) k_bicg_t(int n, View A, const T* __restrict__ shat,
                                                        const T* __restrict__ s, T* __restrict__ t, SolveStateT<T>* st,
                                                        Red<T> red) {
  const bool live = !st->done;
  T acc[2] = {T(0), T(0)};
  if (live) {
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
      const T tv = A.row(row, shat);
      t[row] = tv;
      acc[0] = fma_rn(tv, s[row], acc[0]);
      acc[1] = fma_rn(tv, tv, acc[1]);
    }
  }
  if (grid_reduce<2>(acc, red.partials, red.counter, red.result)) {
    if (live) {
      const T ts = red.result[0], tt = red.result[1];
      if (tt == T(0)) {
        // first step: stop(r); later steps: stop(s) -- s.s is the value just tested
        const T v = st->first ? st->rr_r : st->rr;
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
template <class T>
__global__ void __launch_bounds__(kCtlThreads) k_bicg_update(int n, const T* __restrict__ shat, const T* __restrict__ phat,
                                                             const T* __restrict__ s, const T* __restrict__ t,
                                                             const T* __restrict__ r0, T* __restrict__ r,
                                                             SolveStateT<T>* st, Red<T> red, cudaGraphConditionalHandle h,
                                                             int use_graph) {
  T* x = st->x;
  const int done = st->done;
  const int fix = st->exit_fixup;
  const T alpha = st->alpha, omega = st->omega;
  T acc[2] = {T(0), T(0)};
  if (done) {
    if (fix) {
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = fma_rn(alpha, phat[i], x[i]);
    }
  } else {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      T xv = fma_rn(omega, shat[i], x[i]);
      x[i] = fma_rn(alpha, phat[i], xv);
      const T rv = fma_rn(-omega, t[i], s[i]);
      r[i] = rv;
      acc[0] = fma_rn(rv, rv, acc[0]);
      acc[1] = fma_rn(rv, r0[i], acc[1]);
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
        if (st->rho == T(0)) {
          st->error = AB2_ERR_BREAKDOWN;
          st->breakdown = AB2_BREAKDOWN_RHO;
          st->done = 1;
        }
      }
    }
    set_loop(h, use_graph, !st->done);
  }
}

// True residual ||b - A x||^2 into out[0], b.b into out[1] (FP64).
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

namespace {

template <class T>
void pc_apply_t(ab2_context* ctx, const ab2_precond* pc, const T* x, T* y) {
  if constexpr (sizeof(T) == sizeof(double)) pc_apply(ctx, pc, x, y);
  else pc_apply_f32(ctx, pc, x, y);
}


// Logical reduction blocks per launched block for a fused-reduction kernel
// on a reduction grid of g blocks: 2 when the grid does not fit the GPU in
// one wave (and halves evenly), else 1.  Asked of the runtime once per kernel.
int red_blocks_per_sm(const void* kernel) {
  static std::mutex mu;
  static std::unordered_map<const void*, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(kernel);
  if (it != cache.end()) return it->second;
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kCtlThreads, 0) != cudaSuccess) {
    (void)cudaGetLastError();
    b = 0;
  }
  cache[kernel] = b;
  return b;
}

int red_virtual(const ab2_context* ctx, const void* kernel, int g) {
  const int per_sm = red_blocks_per_sm(kernel);
  return (per_sm > 0 && g > per_sm * ctx->num_sms && g % 2 == 0) ? 2 : 1;
}

// q = A p (and p formed) with the p.q reduction, one wave where the
// reduction grid allows it.
template <class View, class T>
void launch_cgj_spmv(ab2_context* ctx, int g, int n, View view, const T* z, T* p0, T* p1, T* q, SolveStateT<T>* st,
                     Red<T> red) {
  if (red_virtual(ctx, (const void*)k_cgj_spmv<View, T, 1>, g) == 2)
    k_cgj_spmv<View, T, 2><<<g / 2, kCtlThreads, 0, ctx->stream>>>(n, view, z, p0, p1, q, st, red);
  else
    k_cgj_spmv<View, T, 1><<<g, kCtlThreads, 0, ctx->stream>>>(n, view, z, p0, p1, q, st, red);
}

template <class View>
struct sym_bands_f32 : std::false_type {};
template <bool UNIT>
struct sym_bands_f32<StencilView<float, true, UNIT>> : std::true_type {
  static constexpr bool unit = UNIT;
};

template <class View, class T>
void launch_cg_spmv(ab2_context* ctx, int g, int n, View view, const T* p, T* q, SolveStateT<T>* st, Red<T> red) {
  if constexpr (sym_bands_f32<View>::value) {
    if (view.nx % 4 == 0) {  // four rows a thread, the same q and the same p.q tree
      k_cg_spmv_x4<sym_bands_f32<View>::unit><<<(g + 3) / 4, kCtlThreads, 0, ctx->stream>>>(n, view, p, q, st, red, g);
      return;
    }
  }
  if (red_virtual(ctx, (const void*)k_cg_spmv<View, T, 1>, g) == 2)
    k_cg_spmv<View, T, 2><<<g / 2, kCtlThreads, 0, ctx->stream>>>(n, view, p, q, st, red);
  else
    k_cg_spmv<View, T, 1><<<g, kCtlThreads, 0, ctx->stream>>>(n, view, p, q, st, red);
}

}  // namespace

template <class T>
template <class F>
void Krylov<T>::with_op(F&& f) const {
  if constexpr (sizeof(T) == sizeof(float)) {
    if (unit_bands) {
      f(stencil_view<T, true, true>(A, unit_bands));
      return;
    }
  }
  with_view<T>(A, variant, f);
}

// Enqueues one loop iteration.  Returns the number of kernels it launched.
template <class T>
int Krylov<T>::enqueue_body(cudaGraphConditionalHandle h, int graph_loop) {
  const int n = A->n;
  const int g = red_grid(ctx, n);
  const int ge = grid_for(n);
  const long long before = ctx->launches;
  SolveStateT<T>* st = d_st;
  if (fused_diag) {
    // without a Jacobi scaling z is r itself: read r, store no z
    const T* inv = diag_inv();
    T *r = w[0], *z = inv ? w[1] : nullptr, *p0 = w[2], *q = w[3], *p1 = w[4];
    if constexpr (sizeof(T) == sizeof(double)) {
      // FP64: p formed on the fly inside the SpMV (two p buffers)
      with_op([&](auto view) {
        launch_cgj_spmv<decltype(view), T>(ctx, g, n, view, z ? z : r, p0, p1, q, st, red_of<T>(ctx, 2));
      });
      check_launch(ctx, "cgj_spmv");
      k_cgj_update<<<g, kCtlThreads, 0, ctx->stream>>>(n, p0, p1, q, r, z, inv, stop_weight, st, red_of<T>(ctx, 3), h,
                                                       graph_loop);
    } else {
      // FP32: p = z + beta p in place by its own streaming kernel, then the
      // plain SpMV; the same values, the same p.q tree, one launch more.  In
      // FP32 the fused SpMV's per-row work (7 neighbours' p formed from z and
      // the old p: 20 loads) left it latency-bound at 2.8 TB/s; split, the
      // mixed 192^3 Jacobi solve took 70.5 ms against 83.8 ms.  In FP64 the
      // split was slower (165.7 against 142.5 ms), so FP64 keeps the fused form.
      (void)p1;
      k_cg_px<<<ge, kThreads, 0, ctx->stream>>>(n, z ? z : r, p0, st);
      check_launch(ctx, "cg_px");
      with_op([&](auto view) {
        launch_cg_spmv<decltype(view), T>(ctx, g, n, view, p0, q, st, red_of<T>(ctx, 2));
      });
      check_launch(ctx, "cg_spmv");
      if (n % 4 == 0)  // four elements a thread, the same values and trees
        k_cgj_update_x4<true><<<(g + 3) / 4, kCtlThreads, 0, ctx->stream>>>(n, p0, p0, q, r, z, inv, stop_weight, st,
                                                                           red_of<T>(ctx, 3), h, graph_loop, g);
      else
        k_cgj_update<T, true><<<g, kCtlThreads, 0, ctx->stream>>>(n, p0, p0, q, r, z, inv, stop_weight, st,
                                                                  red_of<T>(ctx, 3), h, graph_loop);
    }
    check_launch(ctx, "cgj_update");
  } else if (solver == AB2_SOLVER_CG) {
    T *r = w[0], *z = w[1], *p = w[2], *q = w[3];
    pc_apply_t(ctx, pc, r, z);
    k_cg_rz<<<g, kCtlThreads, 0, ctx->stream>>>(n, r, z, st, red_of<T>(ctx, 1));
    check_launch(ctx, "cg_rz");
    if constexpr (sizeof(T) == sizeof(double)) {
      // FP64: p = z + beta p formed inside the SpMV (two p buffers), as the
      // Diag body does; the same values and trees
      T* p1 = w[4];
      with_op([&](auto view) {
        launch_cgj_spmv<decltype(view), T>(ctx, g, n, view, z, p, p1, q, st, red_of<T>(ctx, 2));
      });
      check_launch(ctx, "cgj_spmv");
      k_cg_update<<<g, kCtlThreads, 0, ctx->stream>>>(n, p, p1, q, r, st, red_of<T>(ctx, 3), h, graph_loop);
    } else {
      k_cg_p<<<ge, kThreads, 0, ctx->stream>>>(n, z, p, st);
      check_launch(ctx, "cg_p");
      with_op([&](auto view) {
        launch_cg_spmv<decltype(view), T>(ctx, g, n, view, p, q, st, red_of<T>(ctx, 2));
      });
      check_launch(ctx, "cg_spmv");
      k_cg_update<<<g, kCtlThreads, 0, ctx->stream>>>(n, p, (const T*)nullptr, q, r, st, red_of<T>(ctx, 3), h,
                                                      graph_loop);
    }
    check_launch(ctx, "cg_update");
  } else {
    T *r = w[0], *r0 = w[1], *p = w[2], *phat = w[3], *v = w[4], *s = w[5], *shat = w[6], *t = w[7];
    k_bicg_p<<<ge, kThreads, 0, ctx->stream>>>(n, r, v, p, st);
    check_launch(ctx, "bicg_p");
    pc_apply_t(ctx, pc, p, phat);
    with_op([&](auto view) {
      k_bicg_v<<<g, kCtlThreads, 0, ctx->stream>>>(n, view, phat, r0, v, st, red_of<T>(ctx, 1));
    });
    check_launch(ctx, "bicg_v");
    k_bicg_s<<<g, kCtlThreads, 0, ctx->stream>>>(n, r, v, s, st, red_of<T>(ctx, 2));
    check_launch(ctx, "bicg_s");
    pc_apply_t(ctx, pc, s, shat);
    with_op([&](auto view) {
      k_bicg_t<<<g, kCtlThreads, 0, ctx->stream>>>(n, view, shat, s, t, st, red_of<T>(ctx, 3));
    });
    check_launch(ctx, "bicg_t");
    k_bicg_update<<<g, kCtlThreads, 0, ctx->stream>>>(n, shat, phat, s, t, r0, r, st, red_of<T>(ctx, 4), h,
                                                       graph_loop);
    check_launch(ctx, "bicg_update");
  }
  return (int)(ctx->launches - before);
}

template <class T>
const T* Krylov<T>::diag_inv() const {
  if (pc->kind != AB2_PC_DIAG) return nullptr;
  if constexpr (sizeof(T) == sizeof(double)) return pc->d_inv;
  else return pc->d_inv32;
}

template <class T>
void Krylov<T>::build_graph() {
  AB2_CUDA(cudaGraphCreate(&graph, 0));
  AB2_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  AB2_CUDA(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  AB2_CUDA(cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  int launched = 0;
  try {
    launched = enqueue_body(handle, 1);
  } catch (...) {
    cudaGraph_t dummy;
    cudaStreamEndCapture(ctx->stream, &dummy);
    throw;
  }
  AB2_CUDA(cudaStreamEndCapture(ctx->stream, &body));
  ctx->launches -= launched;  // captured, not launched
  body_launches = launched;
  AB2_CUDA(cudaGraphInstantiate(&exec, graph, 0));
}

template <class T>
void Krylov<T>::init(ab2_context* c, const ab2_matrix* a, const ab2_precond* p, int solver_kind, int spmv_variant,
                     int graph_loop, int max_iter) {
  ctx = c;
  A = a;
  pc = p;
  solver = solver_kind;
  variant = spmv_variant;
  use_graph = graph_loop;
  fused_diag = solver == AB2_SOLVER_CG && pc && (pc->kind == AB2_PC_DIAG || pc->kind == AB2_PC_NONE);
  const int nw = fused_diag ? 5 : solver == AB2_SOLVER_CG ? (sizeof(T) == sizeof(double) ? 5 : 4) : 8;
  for (int i = 0; i < nw; ++i) {
    w[i] = dev_alloc<T>(ctx, (size_t)A->n);
    AB2_CUDA(cudaMemsetAsync(w[i], 0, sizeof(T) * (size_t)std::max(A->n, 1), ctx->stream));
  }
  d_st = dev_alloc<SolveStateT<T>>(ctx, 1);
  AB2_CUDA(cudaMemsetAsync(d_st, 0, sizeof(SolveStateT<T>), ctx->stream));
  AB2_CUDA(cudaMallocHost((void**)&h_st, sizeof(SolveStateT<T>)));
  std::memset(h_st, 0, sizeof(SolveStateT<T>));
  hist_cap = 2 * max_iter + 8;  // BiCGStab tests s and r each iteration
  d_hist = dev_alloc<T>(ctx, (size_t)hist_cap);
  if (use_graph) build_graph();
}

template <class T>
void Krylov<T>::solve(const T* b, T* x, T tol, int max_iter) {
  const int n = A->n;
  const int g = red_grid(ctx, n);
  // Iteration ctor: b.b and the criterion (Iteration.h:44-68)
  k_bb<<<g, kCtlThreads, 0, ctx->stream>>>(n, b, stop_weight, d_st, red_of<T>(ctx, 0));
  check_launch(ctx, "dot");
  k_state_init<<<1, 1, 0, ctx->stream>>>(d_st, tol, max_iter, x, b, d_hist, hist_cap);
  check_launch(ctx, "state_init");
  // r = b - A x (and r0, rho1 for BiCGStab)
  T* r0 = solver == AB2_SOLVER_BICGSTAB ? w[1] : nullptr;
  with_op([&](auto view) {
    k_residual<<<g, kCtlThreads, 0, ctx->stream>>>(n, view, d_st, w[0], r0, red_of<T>(ctx, 0));
  });
  check_launch(ctx, "residual");
  if (fused_diag) {
    const T* inv = diag_inv();
    k_cgj_start<<<g, kCtlThreads, 0, ctx->stream>>>(n, w[0], inv, inv ? w[1] : nullptr, d_st, red_of<T>(ctx, 1));
    check_launch(ctx, "cgj_start");
  }
  // Null right-hand side: the reference returns before any iteration.
  AB2_CUDA(cudaMemcpyAsync(h_st, d_st, sizeof(SolveStateT<T>), cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  if (!h_st->done) {
    if (use_graph) {
      AB2_CUDA(cudaGraphLaunch(exec, ctx->stream));
    } else {
      // Host-driven loop over the same kernels, checking the flag in batches.
      for (;;) {
        const int batch = 8;
        for (int i = 0; i < batch; ++i) enqueue_body(0, 0);
        AB2_CUDA(cudaMemcpyAsync(h_st, d_st, sizeof(SolveStateT<T>), cudaMemcpyDeviceToHost, ctx->stream));
        AB2_CUDA(cudaStreamSynchronize(ctx->stream));
        if (h_st->done) break;
      }
    }
  }
  if constexpr (sizeof(T) == sizeof(float)) {
    if (fused_diag) {  // the FP32 body defers x += alpha p to the next pass: the last one is owed
      k_cg_xfix<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, w[2], d_st);
      check_launch(ctx, "cg_xfix");
    }
  }
  AB2_CUDA(cudaMemcpyAsync(h_st, d_st, sizeof(SolveStateT<T>), cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  if (use_graph) ctx->launches += (long long)h_st->bodies * body_launches;
}

template <class T>
void Krylov<T>::release() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  exec = nullptr;
  graph = nullptr;
  if (ctx) {
    for (T*& p : w) {
      dev_free(ctx, p);
      p = nullptr;
    }
    dev_free(ctx, d_st);
    dev_free(ctx, d_hist);
  }
  d_st = nullptr;
  d_hist = nullptr;
  if (h_st) cudaFreeHost(h_st);
  h_st = nullptr;
}

template struct Krylov<double>;
template struct Krylov<float>;

}  // namespace ab2

using namespace ab2;

struct ab2_solver {
  ab2_context* ctx = nullptr;
  const ab2_matrix* A = nullptr;
  ab2_solver_options opts{};
  ab2_precond* pc = nullptr;
  Krylov<double> eng;
  double setup_ms = 0;
  double solve_ms = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

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
  o->filu_solver_iter = 3;  // the krylov example's filu-solver-niter default
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
    po.filu_factor_iter = o->filu_factor_iter;
    po.filu_solver_iter = o->filu_solver_iter;
    po.filu_tol = o->filu_tol;
    int prc = ab2_precond_create(ctx, A, &po, &S->pc);
    if (prc != AB2_OK) throw Error{prc, ctx->last_error};
    S->pc->variant = o->spmv_variant;
    S->eng.init(ctx, A, S->pc, o->solver, o->spmv_variant, o->use_graph, o->max_iter);
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
  PhaseScope phase_scope(S->ctx, S->opts.solver == AB2_SOLVER_CG ? "SOLVER-CG" : "SOLVER-BICGSTAB");
  ab2_context* ctx = S->ctx;
  std::memset(status, 0, sizeof(*status));
  return guard(ctx, [&] {
    const int n = S->A->n;
    const ab2_solver_options& o = S->opts;
    AB2_CUDA(cudaEventRecord(S->ev0, ctx->stream));
    S->eng.solve(b->d, x->d, o.tol, o.max_iter);
    AB2_CUDA(cudaEventRecord(S->ev1, ctx->stream));
    AB2_CUDA(cudaEventSynchronize(S->ev1));
    float ms = 0;
    AB2_CUDA(cudaEventElapsedTime(&ms, S->ev0, S->ev1));
    S->solve_ms = ms;
    const SolveState& st = *S->eng.h_st;
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
      k_true_residual<<<red_grid(ctx, n), kCtlThreads, 0, ctx->stream>>>(n, view, x->d, b->d, red);
    });
    check_launch(ctx, "true_residual");
    AB2_CUDA(cudaMemcpyAsync(ctx->h_pinned, red.result, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    status->true_residual = ctx->h_pinned[1] > 0 ? std::sqrt(ctx->h_pinned[0] / ctx->h_pinned[1]) : 0.0;
  });
}

int ab2_solver_history(const ab2_solver* S, double* hist, int cap, int* len) {
  if (!S || !len || (cap > 0 && !hist)) return AB2_ERR_BAD_ARG;
  const SolveState* st = S->eng.h_st;
  const int have = std::min(st ? st->hist_len : 0, S->eng.hist_cap);
  *len = st ? st->hist_len : 0;
  const int m = std::min(have, cap);
  if (m > 0) {
    if (cudaMemcpy(hist, S->eng.d_hist, sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost) != cudaSuccess)
      return AB2_ERR_CUDA;
  }
  return AB2_OK;
}

int ab2_solver_destroy(ab2_solver* S) {
  if (!S) return AB2_ERR_BAD_ARG;
  if (S->ctx) ctx_quiesce(S->ctx);
  S->eng.release();
  if (S->pc) ab2_precond_destroy(S->pc);
  if (S->ev0) cudaEventDestroy(S->ev0);
  if (S->ev1) cudaEventDestroy(S->ev1);
  if (S->ctx) ctx_release(S->ctx);
  delete S;
  return AB2_OK;
}

}  // extern "C"
