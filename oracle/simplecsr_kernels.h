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

namespace ab2_oracle {

struct Csr {
  int n;
  const int* rp;
  const int* ci;
  const double* v;
};

// dcol[i] = first position k in row i with col >= i (CSRStructInfo.h:291-309).
inline std::vector<int> diag_offsets(const Csr& A) {
  std::vector<int> d(A.n);
  for (int i = 0; i < A.n; ++i) {
    int k = A.rp[i];
    while (k < A.rp[i + 1] && A.ci[k] < i) ++k;
    d[i] = k;
  }
  return d;
}

inline void spmv(const Csr& A, const double* x, double* y) {
  for (int i = 0; i < A.n; ++i) {
    double acc = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) acc = acc + A.v[k] * x[A.ci[k]];
    y[i] = acc;
  }
}

// BLAS-1 as CBLAS kernels compute it on FMA hardware: axpy is one fma per
// element; ddot is summed sequentially here (its order is implementation
// defined; the GPU sums the same products in a fixed tree).
inline double dot(int n, const double* x, const double* y) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = std::fma(x[i], y[i], s);
  return s;
}
inline void axpy(int n, double a, const double* x, double* y) {
  for (int i = 0; i < n; ++i) y[i] = std::fma(a, x[i], y[i]);
}
inline void scal(int n, double a, double* x) {
  for (int i = 0; i < n; ++i) x[i] = a * x[i];
}
inline void copy(int n, const double* x, double* y) { std::memcpy(y, x, sizeof(double) * (size_t)n); }
inline void pmult(int n, const double* x, const double* y, double* w) {
  for (int i = 0; i < n; ++i) w[i] = x[i] * y[i];
}


}  // namespace ab2_oracle
