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

// Calls f(view) with the view the variant selects (ELL when present, else CSR).
template <class T, class F>
void with_view(const ab2_matrix* A, int variant, F&& f) {
  const bool f32 = sizeof(T) == 4;
  const int v = resolve_variant(A, variant);
  const T* ev = (const T*)(f32 ? (const void*)A->d_ell_v32 : (const void*)A->d_ell_v);
  const T* cv = (const T*)(f32 ? (const void*)A->d_v32 : (const void*)A->d_v);
  if (v == AB2_SPMV_ELL && ev) {
    f(EllView<T>{A->d_ell_off, A->d_ell_ci, ev});
  } else {
    require(cv != nullptr, "matrix values missing in the requested precision");
    f(CsrView<T>{A->d_rp, A->d_ci, cv});
  }
}

}  // namespace ab2
