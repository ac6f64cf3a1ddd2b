// spmv_view.cuh -- per-row SpMV views used by the fused kernels.
//
// A view computes sum_k a_k x[c_k] for one row in column order, rounding as
// the loop of SimpleCSRMatrixMultT.h:184-190 does, so a fused kernel that
// calls it produces exactly the y of the standalone SpMV kernels.
#pragma once

#include "ab2_internal.cuh"

namespace ab2 {

template <class T>
struct CsrView {
  const int* __restrict__ rp;
  const int* __restrict__ ci;
  const T* __restrict__ v;
  __device__ __forceinline__ T row(int r, const T* __restrict__ x) const {
    T acc = 0;
    const int e = rp[r + 1];
    for (int k = rp[r]; k < e; ++k) acc = mul_add_rn(__ldcs(v + k), __ldg(x + __ldcs(ci + k)), acc);
    return acc;
  }
  // The same sum with the operand x[c] given by f(c) (computed on the fly).
  template <class F>
  __device__ __forceinline__ T row_f(int r, F&& f) const {
    T acc = 0;
    const int e = rp[r + 1];
    for (int k = rp[r]; k < e; ++k) acc = mul_add_rn(__ldcs(v + k), f(__ldcs(ci + k)), acc);
    return acc;
  }
};

template <class T>
struct EllView {
  const int* __restrict__ off;
  const int* __restrict__ ci;
  const T* __restrict__ v;
  __device__ __forceinline__ T row(int r, const T* __restrict__ x) const {
    const int s = r >> 5, lane = r & 31;
    const int o = off[s];
    const int w = off[s + 1] - o;
    const size_t base = (size_t)o * kEllSlice + lane;
    const int* cp = ci + base;
    const T* vp = v + base;
    return ell_row_sum(cp, vp, w, x);
  }
  template <class F>
  __device__ __forceinline__ T row_f(int r, F&& f) const {
    const int s = r >> 5, lane = r & 31;
    const int o = off[s];
    const int w = off[s + 1] - o;
    const size_t base = (size_t)o * kEllSlice + lane;
    const int* cp = ci + base;
    const T* vp = v + base;
    T acc = 0;
    for (int j = 0; j < w; j += 8) {
      int c[8];
      T a[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const bool in = j + u < w;
        c[u] = in ? __ldcs(cp + (size_t)(j + u) * kEllSlice) : -1;
        a[u] = in ? __ldcs(vp + (size_t)(j + u) * kEllSlice) : (T)0;
      }
      T xv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) xv[u] = c[u] >= 0 ? f(c[u]) : (T)0;
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (c[u] >= 0) acc = mul_add_rn(a[u], xv[u], acc);
    }
    return acc;
  }

  // Slots in groups of 8, all loads of a group issued before the first use
  // (a 7-point row is one group), predicated on the slice width.
  static __device__ __forceinline__ T ell_row_sum(const int* cp, const T* vp, int w, const T* __restrict__ x) {
    T acc = 0;
    for (int j = 0; j < w; j += 8) {
      int c[8];
      T a[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const bool in = j + u < w;
        c[u] = in ? __ldcs(cp + (size_t)(j + u) * kEllSlice) : -1;
        a[u] = in ? __ldcs(vp + (size_t)(j + u) * kEllSlice) : (T)0;
      }
      T xv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) xv[u] = c[u] >= 0 ? __ldg(x + c[u]) : (T)0;
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (c[u] >= 0) acc = mul_add_rn(a[u], xv[u], acc);
    }
    return acc;
  }
};

// Sliced ELL with S-row slices (the batched solver's autotuned layouts,
// build_ell_f32): the same slot-major layout and column-order sum as EllView.
template <class T, int S>
struct EllViewS {
  const int* __restrict__ off;
  const int* __restrict__ ci;
  const T* __restrict__ v;
  __device__ __forceinline__ T row(int r, const T* __restrict__ x) const {
    const int s = r / S, lane = r % S;
    const int o = off[s];
    const int w = off[s + 1] - o;
    const size_t base = (size_t)o * S + lane;
    const int* cp = ci + base;
    const T* vp = v + base;
    T acc = 0;
    for (int j = 0; j < w; j += 8) {
      int c[8];
      T a[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const bool in = j + u < w;
        c[u] = in ? __ldcs(cp + (size_t)(j + u) * S) : -1;
        a[u] = in ? __ldcs(vp + (size_t)(j + u) * S) : T(0);
      }
      T xv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) xv[u] = c[u] >= 0 ? __ldg(x + c[u]) : T(0);
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (c[u] >= 0) acc = mul_add_rn(a[u], xv[u], acc);
    }
    return acc;
  }
  // The same sum with the operand x[c] given by f(c) (computed on the fly).
  template <class F>
  __device__ __forceinline__ T row_f(int r, F&& f) const {
    const int s = r / S, lane = r % S;
    const int o = off[s];
    const int w = off[s + 1] - o;
    const size_t base = (size_t)o * S + lane;
    const int* cp = ci + base;
    const T* vp = v + base;
    T acc = 0;
    for (int j = 0; j < w; j += 8) {
      int c[8];
      T a[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const bool in = j + u < w;
        c[u] = in ? __ldcs(cp + (size_t)(j + u) * S) : -1;
        a[u] = in ? __ldcs(vp + (size_t)(j + u) * S) : T(0);
      }
      T xv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) xv[u] = c[u] >= 0 ? f(c[u]) : T(0);
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (c[u] >= 0) acc = mul_add_rn(a[u], xv[u], acc);
    }
    return acc;
  }
};

// CSR with LPR consecutive lanes per row (the batched solver's "rows per
// warp" = 32 / LPR): lane g of the group sums the row's entries g, g + LPR,
// ... in order (product and sum rounded apart), then the group adds its
// partials by an xor butterfly (offsets LPR/2 .. 1), so every lane of the
// group holds the same total.  Not the row-sequential order: only the
// batched solver uses it, and its oracle restates this tree.
template <class T, int LPR>
struct CsrGroupView {
  static_assert(LPR == 2 || LPR == 4 || LPR == 8 || LPR == 16 || LPR == 32, "lanes per row: a power of two <= 32");
  const int* __restrict__ rp;
  const int* __restrict__ ci;
  const T* __restrict__ v;
  // Every lane of the warp must call it (the shuffles); g = lane's index in its group.
  __device__ __forceinline__ T row_group(int r, bool valid, int g, const T* __restrict__ x) const {
    T acc = 0;
    if (valid) {
      const int e = rp[r + 1];
      for (int k = rp[r] + g; k < e; k += LPR) acc = mul_add_rn(__ldcs(v + k), __ldg(x + __ldcs(ci + k)), acc);
    }
#pragma unroll
    for (int off = LPR / 2; off > 0; off >>= 1) acc = acc + __shfl_xor_sync(0xffffffffu, acc, off);
    return acc;
  }
};

template <class V>
struct lanes_per_row {
  static constexpr int value = 1;
};
template <class T, int LPR>
struct lanes_per_row<CsrGroupView<T, LPR>> {
  static constexpr int value = LPR;
};

// 7-point bands (ab2_matrix::d_st_v): row r = i + nx (j + ny k) holds its
// in-grid neighbours in ascending column order -nx ny, -nx, -1, 0, +1, +nx,
// +nx ny, so the sum runs over the same terms in the same order as the CSR
// row and rounds identically; neighbours outside the grid are skipped, not
// added as zeros.  The coordinates come from two invariant divisions.  SYM: 4
// bands (D, Ux, Uy, Uz) and the lower values read from the neighbouring
// rows' upper bands (bit-for-bit the same numbers in a symmetric matrix).
// UNIT (with SYM): a unit diagonal that is not stored, 3 bands (Ux, Uy, Uz);
// the diagonal term is 1 * x_r, as a stored 1 would give.
template <class T, bool SYM, bool UNIT = false>
struct StencilView {
  static_assert(SYM || !UNIT, "a unit-diagonal operator is kept in its symmetric form");
  static constexpr int kUx = UNIT ? 0 : 1;  // band index of Ux (then Uy, Uz)
  const T* __restrict__ v;
  int n, nx, ny, nz;
  FastDiv fx, fy;
  template <class F>
  __device__ __forceinline__ T row_f(int r, F&& f) const {
    const unsigned q = fx.div((unsigned)r);
    const int i = r - (int)q * nx;
    const int k = (int)fy.div(q);
    const int j = (int)q - k * ny;
    const int sx = 1, sy = nx, sz = nx * ny;
    const bool in[7] = {k > 0, j > 0, i > 0, true, i < nx - 1, j < ny - 1, k < nz - 1};
    const int off[7] = {-sz, -sy, -sx, 0, sx, sy, sz};
    const size_t N = (size_t)n;
    T a[7];
    if constexpr (SYM) {
      // lower value of row r toward r - s = upper value of row r - s toward r
      // (band rows addressed as base + 32-bit row index)
      const T* __restrict__ ux = v + kUx * N;
      const T* __restrict__ uy = ux + N;
      const T* __restrict__ uz = uy + N;
      a[0] = in[0] ? __ldg(uz + (r - sz)) : T(0);
      a[1] = in[1] ? __ldg(uy + (r - sy)) : T(0);
      a[2] = in[2] ? __ldg(ux + (r - sx)) : T(0);
      a[3] = UNIT ? T(1) : __ldg(v + r);
      a[4] = in[4] ? __ldg(ux + r) : T(0);
      a[5] = in[5] ? __ldg(uy + r) : T(0);
      a[6] = in[6] ? __ldg(uz + r) : T(0);
    } else {
#pragma unroll
      for (int b = 0; b < 7; ++b) a[b] = in[b] ? __ldcs(v + (size_t)b * N + r) : T(0);
    }
    T xv[7];
#pragma unroll
    for (int b = 0; b < 7; ++b) xv[b] = in[b] ? f(r + off[b]) : T(0);
    T acc = 0;
#pragma unroll
    for (int b = 0; b < 7; ++b)
      if (in[b]) acc = mul_add_rn(a[b], xv[b], acc);
    return acc;
  }
  __device__ __forceinline__ T row(int r, const T* __restrict__ x) const {
    return row_f(r, [x](int c) { return __ldg(x + c); });
  }
};

template <class T, bool SYM, bool UNIT = false>
StencilView<T, SYM, UNIT> stencil_view(const ab2_matrix* A, const T* bands) {
  return StencilView<T, SYM, UNIT>{bands, A->n, A->st_nx, A->st_ny, A->st_nz, FastDiv((unsigned)A->st_nx),
                                   FastDiv((unsigned)A->st_ny)};
}

// Calls f(view) with the view the variant selects: the 7-point bands when
// chosen and present in T, ELL when chosen and present, else CSR.
// kStencil = false leaves the band views out (callers whose kernels are never
// given a 7-point matrix, so that they are not instantiated for it).
template <class T, bool kStencil = true, class F>
void with_view(const ab2_matrix* A, int variant, F&& f) {
  const bool f32 = sizeof(T) == 4;
  const int v = resolve_variant(A, variant);
  const T* ev = (const T*)(f32 ? (const void*)A->d_ell_v32 : (const void*)A->d_ell_v);
  const T* cv = (const T*)(f32 ? (const void*)A->d_v32 : (const void*)A->d_v);
  const T* sv = (const T*)(f32 ? (const void*)A->d_st_v32 : (const void*)A->d_st_v);
  if (kStencil && v == AB2_SPMV_STENCIL && sv) {
    if constexpr (kStencil) {
      if (A->st_bands == 4) f(stencil_view<T, true>(A, sv));
      else f(stencil_view<T, false>(A, sv));
    }
  } else if ((v == AB2_SPMV_ELL || v == AB2_SPMV_STENCIL) && ev) {
    f(EllView<T>{A->d_ell_off, A->d_ell_ci, ev});
  } else {
    require(cv != nullptr, "matrix values missing in the requested precision");
    f(CsrView<T>{A->d_rp, A->d_ci, cv});
  }
}

}  // namespace ab2
