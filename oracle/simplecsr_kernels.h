// simplecsr_kernels.h -- sequential restatement of Alien's SimpleCSR algebra
// kernels.  TEST INFRASTRUCTURE ONLY (oracle): included by ab2_oracle.cpp and by
// the reference-template driver in oracle/ref/, never by the product.
//
//   spmv        SimpleCSRMatrixMultT.h:172-191 (row-sequential sum; the product and
//               the sum are rounded separately, as the stock build of that loop
//               -- no -march, or ISO -std=c++17 -- compiles it)
//   dcol        CSRStructInfo.h:291-309
//   BLAS-1      CBLASMPIKernel.h:37-125
#pragma once
#include <cmath>
#include <cstring>
#include <vector>
#ifdef ORC_THREADS
#include "host_threads.h"
#endif

namespace ab2_oracle {

// T is double for the reference's algebra; float instantiations restate the
// FP32 inner solves of the mixed-precision solver (same operations in float).
template <class T>
struct CsrT {
  int n;
  const int* rp;
  const int* ci;
  const T* v;
};
using Csr = CsrT<double>;

// dcol[i] = first position k in row i with col >= i (CSRStructInfo.h:291-309).
template <class T>
inline std::vector<int> diag_offsets(const CsrT<T>& A) {
  std::vector<int> d(A.n);
  for (int i = 0; i < A.n; ++i) {
    int k = A.rp[i];
    while (k < A.rp[i + 1] && A.ci[k] < i) ++k;
    d[i] = k;
  }
  return d;
}

// ORC_THREADS (the all-cores CPU baseline build, oracle/Makefile): the row
// loop of the SpMV and the BLAS-1 loops run on the host threads of
// host_threads.h -- each element computed as in the sequential form -- and
// the dot sums per-thread partials (contiguous blocks, each summed
// sequentially) in thread order.  A restatement for timing, not the
// reference: its dot order differs.
#ifdef ORC_THREADS
#define ORC_FOR(n, i, body)                                                        \
  HostPool::get().run((n), [&](int, long long lo_, long long hi_) {                \
    for (long long i = lo_; i < hi_; ++i) body;                                     \
  })
#else
#define ORC_FOR(n, i, body) \
  for (long long i = 0; i < (long long)(n); ++i) body
#endif

template <class T>
inline void spmv(const CsrT<T>& A, const T* x, T* y) {
  ORC_FOR(A.n, i, {
    T acc = 0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) acc = acc + A.v[k] * x[A.ci[k]];
    y[i] = acc;
  });
}

// BLAS-1 as CBLAS kernels compute it on FMA hardware: axpy is one fma per
// element; ddot is summed sequentially here (its order is implementation
// defined; the GPU sums the same products in a fixed tree).
template <class T>
inline T dot(int n, const T* x, const T* y) {
#ifdef ORC_THREADS
  std::vector<T> part((size_t)HostPool::get().size(), T(0));
  HostPool::get().run(n, [&](int t, long long lo, long long hi) {
    T s = 0;
    for (long long i = lo; i < hi; ++i) s = std::fma(x[i], y[i], s);
    part[(size_t)t] = s;
  });
  T s = 0;
  for (const T p : part) s = s + p;
  return s;
#else
  T s = 0;
  for (int i = 0; i < n; ++i) s = std::fma(x[i], y[i], s);
  return s;
#endif
}
template <class T>
inline void axpy(int n, T a, const T* x, T* y) {
  ORC_FOR(n, i, y[i] = std::fma(a, x[i], y[i]));
}
template <class T>
inline void scal(int n, T a, T* x) {
  ORC_FOR(n, i, x[i] = a * x[i]);
}
template <class T>
inline void copy(int n, const T* x, T* y) {
  std::memcpy(y, x, sizeof(T) * (size_t)n);
}
template <class T>
inline void pmult(int n, const T* x, const T* y, T* w) {
  ORC_FOR(n, i, w[i] = x[i] * y[i]);
}

}  // namespace ab2_oracle
