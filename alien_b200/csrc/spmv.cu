// spmv.cu -- device matrices and the SpMV family.
//
// Reference counterparts:
//   y = A x        SimpleCSRMatrixMultT.h:172-191 (CSR, row-sequential sum)
//                  SYCLBEllPackMatrix.cc:624-688   (BEllPack, one work-item per row)
//   y += a L/U x   SimpleCSRMatrixMultT.h:193-233
//   1/a_ii         SimpleCSRMatrixMultT.h:478-509 (diagonal found through dcol,
//                  CSRStructInfo.h:291-309)
//   conversion     SimpleCSRtoSYCLMatrixConverter.cc:74-104, BEllPack layout
//                  SYCLBEllPackMatrix.cc:70-215
//
// Every variant sums a row's products in column order, rounding each product
// and each partial sum (mul_add_rn) exactly as the reference loop does, so all
// variants give bit-identical y (the grouped-lane variant excepted, see
// ab2.h).  For 3-D 7-point profiles the values may also be kept as bands
// without column indices (AB2_FMT_STENCIL): 7 bands, or 4 when the matrix is
// bit-for-bit symmetric, read by StencilView (spmv_view.cuh).  The
// sliced-ELL layout keeps 32-row slices (not the reference's 1024) and stores
// slot j of the slice's rows contiguously, so the 32 lanes of a warp read 256
// contiguous bytes of values and 128 of column indices per slot.  Padding slots
// carry column -1 and are skipped, so padding never touches x.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>
#include <cstring>

#include "ab2_internal.cuh"
#include "spmv_view.cuh"

namespace ab2 {

namespace {

// ----------------------------------------------------------------- set-up kernels
__global__ void k_validate(int n, const int* __restrict__ rp, const int* __restrict__ ci, int* bad) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const int a = rp[row], b = rp[row + 1];
    if (b < a) {
      atomicOr(bad, 1);
      continue;
    }
    int prev = -1;
    for (int k = a; k < b; ++k) {
      const int c = ci[k];
      if (c < 0 || c >= n) atomicOr(bad, 2);
      if (c <= prev) atomicOr(bad, 4);
      prev = c;
    }
  }
}

__global__ void k_dcol(int n, const int* __restrict__ rp, const int* __restrict__ ci, int* __restrict__ dcol) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    int k = rp[row];
    const int e = rp[row + 1];
    while (k < e && ci[k] < row) ++k;
    dcol[row] = k;
  }
}

// Sliced ELL with S-row slices (S = kEllSlice for the matrix's own copy).
template <class T>
__global__ void k_ell_fill(int n, int S, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ v, const int* __restrict__ off, int* __restrict__ eci,
                           T* __restrict__ ev) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const int s = row / S, lane = row % S;
    const int w = off[s + 1] - off[s];
    const size_t base = (size_t)off[s] * S + lane;
    const int a = rp[row], len = rp[row + 1] - a;
    for (int j = 0; j < w; ++j) {
      const size_t at = base + (size_t)j * S;
      eci[at] = j < len ? ci[a + j] : -1;
      ev[at] = j < len ? (T)v[a + j] : (T)0;
    }
  }
}

// Padding rows past n in the last slice.
__global__ void k_ell_pad_tail(int n, int n_pad, int S, const int* __restrict__ off, int* __restrict__ eci) {
  const int row = n + blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n_pad) return;
  const int s = row / S, lane = row % S;
  const int w = off[s + 1] - off[s];
  for (int j = 0; j < w; ++j) eci[(size_t)off[s] * S + lane + (size_t)j * S] = -1;
}

__global__ void k_to_f32(long long m, const double* __restrict__ a, float* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// ----------------------------------------------------------------- SpMV kernels
template <class T>
__global__ void __launch_bounds__(kThreads) k_spmv_csr_scalar(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                                              const T* __restrict__ v, const T* __restrict__ x,
                                                              T* __restrict__ y) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    T acc = 0;
    const int e = rp[row + 1];
    for (int k = rp[row]; k < e; ++k) acc = mul_add_rn(v[k], __ldg(x + ci[k]), acc);
    y[row] = acc;
  }
}

// One block per row block: the block's values and columns are staged into
// shared memory with coalesced loads, then each thread sums one row from there.
template <class T>
__global__ void __launch_bounds__(kThreads) k_spmv_csr_staged(const int* __restrict__ blocks, const int* __restrict__ rp,
                                                              const int* __restrict__ ci, const T* __restrict__ v,
                                                              const T* __restrict__ x, T* __restrict__ y) {
  __shared__ T s_v[kStageCap];
  __shared__ int s_c[kStageCap];
  const int r0 = blocks[blockIdx.x], r1 = blocks[blockIdx.x + 1];
  const int k0 = rp[r0], k1 = rp[r1];
  const int cnt = k1 - k0;
  if (cnt <= kStageCap) {
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
      s_v[t] = __ldcs(v + k0 + t);
      s_c[t] = __ldcs(ci + k0 + t);
    }
    __syncthreads();
    for (int row = r0 + threadIdx.x; row < r1; row += blockDim.x) {
      const int a = rp[row] - k0, b = rp[row + 1] - k0;
      T acc = 0;
      for (int k = a; k < b; ++k) acc = mul_add_rn(s_v[k], __ldg(x + s_c[k]), acc);
      y[row] = acc;
    }
  } else {
    // A single row longer than the staging buffer: sequential in thread 0 to
    // keep the reference's summation order (rare; not on the stencil path).
    if (threadIdx.x == 0) {
      for (int row = r0; row < r1; ++row) {
        T acc = 0;
        for (int k = rp[row]; k < rp[row + 1]; ++k) acc = mul_add_rn(v[k], __ldg(x + ci[k]), acc);
        y[row] = acc;
      }
    }
  }
}

// A group of LPR lanes per row (LPR = 4, 8, 16 or 32, chosen from the mean
// row length), for matrices whose rows are long: the lanes read the row's
// values and columns as 16- and 8-byte pairs (2 doubles, 2 int32 columns),
// two pairs in flight per lane per pass, and the group sums its lanes'
// partial sums with shuffles.  The row's sum is therefore grouped, not
// sequential: results differ from the reference's row-sequential order in
// the last bits, which is why no solver or AUTO choice uses this kernel
// (ab2_mult_variant only).  Pairs start at even entry offsets, so the value
// and column arrays (whole device allocations) give aligned loads; an odd
// first entry and an odd last entry are read singly.
template <int LPR>
__global__ void __launch_bounds__(kThreads) k_spmv_csr_vector(int n, const int* __restrict__ rp,
                                                              const int* __restrict__ ci, const double* __restrict__ v,
                                                              const double* __restrict__ x, double* __restrict__ y) {
  constexpr int RPW = 32 / LPR;  // rows per warp per pass
  const int lane = threadIdx.x & 31, sub = lane % LPR, grp = lane / LPR;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  // every lane of the warp runs every pass (the shuffles take the full mask);
  // a group past the last row works on an empty row and stores nothing
  for (long long w0 = warp * RPW; w0 < n; w0 += nwarps * RPW) {
    const long long row = w0 + grp;
    int b = 0, e = 0;
    if (row < n) {
      b = rp[row];
      e = rp[row + 1];
    }
    double acc = 0;
    const int a0 = min(e, (b + 1) & ~1);  // first even offset in the row
    const int a1 = max(a0, e & ~1);       // end of the paired body
    if (sub == 0 && b < a0) acc = mul_add_rn(v[b], __ldg(x + ci[b]), acc);
    int k = a0 + 2 * sub;
    for (; k + 2 * LPR < a1; k += 4 * LPR) {
      const double2 v0 = *reinterpret_cast<const double2*>(v + k);
      const int2 c0 = *reinterpret_cast<const int2*>(ci + k);
      const double2 v1 = *reinterpret_cast<const double2*>(v + k + 2 * LPR);
      const int2 c1 = *reinterpret_cast<const int2*>(ci + k + 2 * LPR);
      const double x0 = __ldg(x + c0.x), x1 = __ldg(x + c0.y), x2 = __ldg(x + c1.x), x3 = __ldg(x + c1.y);
      acc = mul_add_rn(v0.x, x0, acc);
      acc = mul_add_rn(v0.y, x1, acc);
      acc = mul_add_rn(v1.x, x2, acc);
      acc = mul_add_rn(v1.y, x3, acc);
    }
    if (k < a1) {
      const double2 v0 = *reinterpret_cast<const double2*>(v + k);
      const int2 c0 = *reinterpret_cast<const int2*>(ci + k);
      acc = mul_add_rn(v0.x, __ldg(x + c0.x), acc);
      acc = mul_add_rn(v0.y, __ldg(x + c0.y), acc);
    }
    if (sub == 0 && a1 < e) acc = mul_add_rn(v[a1], __ldg(x + ci[a1]), acc);
#pragma unroll
    for (int off = LPR / 2; off > 0; off >>= 1) acc = add_rn(acc, __shfl_down_sync(0xffffffffu, acc, off, LPR));
    if (sub == 0 && row < n) y[row] = acc;
  }
}

template <int LPR>
void launch_csr_vector(ab2_context* ctx, const ab2_matrix* A, const double* v, const double* x, double* y) {
  const long long n = A->n, warps = std::min<long long>((n + 32 / LPR - 1) / (32 / LPR), (long long)ctx->num_sms * 64);
  k_spmv_csr_vector<LPR><<<(int)((warps * 32 + kThreads - 1) / kThreads), kThreads, 0, ctx->stream>>>(
      A->n, A->d_rp, A->d_ci, v, x, y);
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_spmv_ell(int n, const int* __restrict__ off, const int* __restrict__ eci,
                                                       const T* __restrict__ ev, const T* __restrict__ x,
                                                       T* __restrict__ y) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const int s = row >> 5, lane = row & 31;
  const int o = off[s];
  const int w = off[s + 1] - o;
  const size_t base = (size_t)o * kEllSlice + lane;
  y[row] = EllView<T>::ell_row_sum(eci + base, ev + base, w, x);
}

// y = A x through a row view (the 7-point bands).
template <class View, class T>
__global__ void __launch_bounds__(kThreads) k_spmv_view(int n, View A, const T* __restrict__ x, T* __restrict__ y) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) y[row] = A.row(row, x);
}

// ----------------------------------------------------------------- 7-point bands
// geo[0] = min over rows with 7 entries (starts at n); then geo[1..2] = the
// first two columns of that row: r - nx ny and r - nx.
__global__ void k_first_full_row7(int n, const int* __restrict__ rp, int* geo) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    if (rp[r + 1] - rp[r] == 7) atomicMin(geo, r);
}

__global__ void k_full_row7_cols(int n, const int* __restrict__ rp, const int* __restrict__ ci, int* geo) {
  const int r = geo[0];
  if (r < n) {
    geo[1] = ci[rp[r]];
    geo[2] = ci[rp[r] + 1];
  }
}

// Rows must hold exactly their in-grid 7-point neighbours, in ascending columns.
__global__ void k_stencil7_check(int n, int nx, int ny, int nz, const int* __restrict__ rp, const int* __restrict__ ci,
                                 int* bad) {
  const long long nxny = (long long)nx * ny;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int i = r % nx, j = (r / nx) % ny, k = (int)(r / nxny);
    int e = rp[r];
    const int end = rp[r + 1];
    bool ok = true;
    auto expect = [&](long long c) {
      ok = ok && e < end && ci[e] == c;
      ++e;
    };
    if (k > 0) expect(r - nxny);
    if (j > 0) expect(r - nx);
    if (i > 0) expect(r - 1);
    expect(r);
    if (i < nx - 1) expect(r + 1);
    if (j < ny - 1) expect(r + nx);
    if (k < nz - 1) expect(r + nxny);
    if (!ok || e != end) atomicOr(bad, 1);
  }
}

// The 7 bands (Lz, Ly, Lx, D, Ux, Uy, Uz; band-major) from a checked 7-point
// CSR profile; 0 where the neighbour is outside the grid.
__global__ void k_stencil7_fill(int n, int nx, int ny, int nz, const int* __restrict__ rp, const double* __restrict__ v,
                                double* __restrict__ bands) {
  const long long nxny = (long long)nx * ny;
  const size_t N = (size_t)n;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int i = r % nx, j = (r / nx) % ny, k = (int)(r / nxny);
    const bool in[7] = {k > 0, j > 0, i > 0, true, i < nx - 1, j < ny - 1, k < nz - 1};
    int e = rp[r];
    for (int b = 0; b < 7; ++b) bands[(size_t)b * N + r] = in[b] ? v[e++] : 0.0;
  }
}

// bad |= 1 unless every off-diagonal pair is equal bit for bit: the upper
// value of row r toward r + s against the lower value of row r + s toward r.
__global__ void k_stencil7_symmetric(int n, int nx, int ny, int nz, const double* __restrict__ bands, int* bad) {
  const long long nxny = (long long)nx * ny;
  const size_t N = (size_t)n;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int i = r % nx, j = (r / nx) % ny, k = (int)(r / nxny);
    bool ok = true;
    auto same = [](double a, double b) { return __double_as_longlong(a) == __double_as_longlong(b); };
    if (i < nx - 1) ok = ok && same(bands[4 * N + r], bands[2 * N + r + 1]);
    if (j < ny - 1) ok = ok && same(bands[5 * N + r], bands[1 * N + r + nx]);
    if (k < nz - 1) ok = ok && same(bands[6 * N + r], bands[0 * N + r + nxny]);
    if (!ok) atomicOr(bad, 1);
  }
}

__global__ void k_add_lu(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                         const int* __restrict__ dcol, double alpha, const double* __restrict__ x, double* __restrict__ y,
                         bool lower) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    double acc = y[row];
    const int a = lower ? rp[row] : dcol[row] + 1;
    const int b = lower ? dcol[row] : rp[row + 1];
    for (int k = a; k < b; ++k) acc = mul_add_rn(__dmul_rn(alpha, v[k]), x[ci[k]], acc);
    y[row] = acc;
  }
}

// The reference divides by values[dcol[row]] whatever column sits there; a row
// with nothing at or right of the diagonal reads 0 here (giving inf).
__global__ void k_inv_diag(int n, const int* __restrict__ rp, const double* __restrict__ v, const int* __restrict__ dcol,
                           double* __restrict__ inv) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const int d = dcol[row];
    inv[row] = 1. / (d < rp[row + 1] ? v[d] : 0.0);
  }
}

__global__ void k_mult_inv_diag(int n, const int* __restrict__ rp, const double* __restrict__ v,
                                const int* __restrict__ dcol, double* __restrict__ y) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const int d = dcol[row];
    y[row] = y[row] / (d < rp[row + 1] ? v[d] : 0.0);
  }
}

__global__ void k_diagonal(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                           const int* __restrict__ dcol, double* __restrict__ d) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const int k = dcol[row];
    d[row] = (k < rp[row + 1] && ci[k] == row) ? v[k] : 0.0;
  }
}

// Row blocks of the staged kernel, built on the device: every 256-row chunk is
// split greedily into blocks of at most kStageCap entries (a longer row gets a
// block of its own).  The staged kernel sums each row in column order whatever
// the blocking, so only the launch shape depends on it.
__device__ int chunk_blocks(int c, int n, const int* __restrict__ rp, int* out) {
  const int end = min(n, (c + 1) * kThreads);
  int r = c * kThreads, m = 0;
  while (r < end) {
    const int start = r;
    long long nz = 0;
    while (r < end) {
      const int len = rp[r + 1] - rp[r];
      if (nz + len > kStageCap) break;
      nz += len;
      ++r;
    }
    if (r == start) ++r;
    if (out) out[m] = r;
    ++m;
  }
  return m;
}

__global__ void k_rowblock_count(int n, int nc, const int* __restrict__ rp, long long* __restrict__ cnt) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
    cnt[c] = chunk_blocks(c, n, rp, nullptr);
}

__global__ void k_rowblock_emit(int n, int nc, const int* __restrict__ rp, const long long* __restrict__ off,
                                int* __restrict__ blocks) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
    chunk_blocks(c, n, rp, blocks + 1 + off[c]);
  if (blockIdx.x == 0 && threadIdx.x == 0) blocks[0] = 0;
}

// Longest row of every 32-row slice.
__global__ void k_slice_width(int n, int ns, int S, const int* __restrict__ rp, long long* __restrict__ w) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
    int m = 0;
    for (int r = s * S; r < min(n, (s + 1) * S); ++r) m = max(m, rp[r + 1] - rp[r]);
    w[s] = m;
  }
}

// out[i] = in[0] + ... + in[i-1] for i <= m (one block of 1024 threads: each
// sums a contiguous segment, the segment sums are scanned in shared memory).
__global__ void __launch_bounds__(1024) k_scan_excl(int m, const long long* __restrict__ in, long long* __restrict__ out) {
  __shared__ long long s[1024];
  const int t = threadIdx.x;
  const int per = (m + 1023) / 1024;
  const int a = min(m, t * per), b = min(m, a + per);
  long long acc = 0;
  for (int i = a; i < b; ++i) acc += in[i];
  s[t] = acc;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    const long long v = t >= d ? s[t - d] : 0;
    __syncthreads();
    s[t] += v;
    __syncthreads();
  }
  long long run = s[t] - acc;
  for (int i = a; i < b; ++i) {
    out[i] = run;
    run += in[i];
  }
  if (t == 1023) out[m] = s[1023];
}

__global__ void k_narrow(int m, const long long* __restrict__ in, int* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) out[i] = (int)in[i];
}

long long read_ll(ab2_context* ctx, const long long* d) {
  long long v = 0;
  AB2_CUDA(cudaMemcpyAsync(&v, d, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  return v;
}

}  // namespace

int resolve_variant(const ab2_matrix* A, int variant) {
  if (variant == AB2_SPMV_AUTO)
    return A->st_bands ? AB2_SPMV_STENCIL : (A->formats & AB2_FMT_ELL) ? AB2_SPMV_ELL : AB2_SPMV_CSR_STAGED;
  return variant;
}

bool stencil_geometry(ab2_context* ctx, const ab2_matrix* A, int* nx_out, int* ny_out, int* nz_out) {
  const int n = A->n;
  if (n == 0) return false;
  // Geometry from the first full row: its columns start r - nx ny, r - nx.
  int* d_geo = dev_alloc<int>(ctx, 4);
  int geo[4] = {n, 0, 0, 0};
  AB2_CUDA(cudaMemcpyAsync(d_geo, geo, sizeof(geo), cudaMemcpyHostToDevice, ctx->stream));
  k_first_full_row7<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, A->d_rp, d_geo);
  check_launch(ctx, "first_full_row");
  k_full_row7_cols<<<1, 1, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, d_geo);
  check_launch(ctx, "full_row_cols");
  AB2_CUDA(cudaMemcpyAsync(geo, d_geo, sizeof(geo), cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  const int r7 = geo[0];
  bool ok = r7 < n;
  long long nx = 0, ny = 0, nz = 0;
  if (ok) {
    const long long nxny = (long long)r7 - geo[1];
    nx = (long long)r7 - geo[2];
    ok = nx >= 2 && nxny > nx && nxny % nx == 0 && n % nxny == 0;
    if (ok) {
      ny = nxny / nx;
      nz = n / nxny;
      ok = ny >= 2 && nz >= 2;
    }
  }
  if (ok) {
    AB2_CUDA(cudaMemsetAsync(d_geo + 3, 0, sizeof(int), ctx->stream));
    k_stencil7_check<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, (int)nx, (int)ny, (int)nz, A->d_rp, A->d_ci,
                                                                d_geo + 3);
    check_launch(ctx, "stencil_check");
    int bad = 0;
    AB2_CUDA(cudaMemcpyAsync(&bad, d_geo + 3, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    ok = bad == 0;
  }
  dev_free(ctx, d_geo);
  if (!ok) return false;
  *nx_out = (int)nx;
  *ny_out = (int)ny;
  *nz_out = (int)nz;
  return true;
}

template <class T>
void spmv_t(ab2_context* ctx, const ab2_matrix* A, const T* v_csr, const T* v_ell, const T* x, T* y, int variant) {
  const int n = A->n;
  if (n == 0) return;
  switch (resolve_variant(A, variant)) {
    case AB2_SPMV_CSR_SCALAR:
      k_spmv_csr_scalar<T><<<grid_for(n, kThreads, 1 << 30), kThreads, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, v_csr, x, y);
      break;
    case AB2_SPMV_CSR_STAGED:
      k_spmv_csr_staged<T><<<A->n_row_blocks, kThreads, 0, ctx->stream>>>(A->d_row_blocks, A->d_rp, A->d_ci, v_csr, x, y);
      break;
    case AB2_SPMV_CSR_VECTOR:
      if constexpr (sizeof(T) == 8) {  // FP64 only: ab2_mult_variant is its one caller
        const long long mean = A->nnz / n;
        if (mean <= 8) launch_csr_vector<4>(ctx, A, v_csr, x, y);
        else if (mean <= 16) launch_csr_vector<8>(ctx, A, v_csr, x, y);
        else if (mean <= 32) launch_csr_vector<16>(ctx, A, v_csr, x, y);
        else launch_csr_vector<32>(ctx, A, v_csr, x, y);
      } else {
        throw Error{AB2_ERR_UNSUPPORTED, "the grouped-lane SpMV runs in FP64 only"};
      }
      break;
    case AB2_SPMV_STENCIL:
      require(A->st_bands != 0, "matrix has no 7-point bands (AB2_FMT_STENCIL on a 7-point profile)");
      with_view<T>(A, AB2_SPMV_STENCIL, [&](auto view) {
        k_spmv_view<<<grid_for(n, kThreads, 1 << 30), kThreads, 0, ctx->stream>>>(n, view, x, y);
      });
      break;
    case AB2_SPMV_ELL:
      require(v_ell != nullptr, "matrix has no sliced-ELL copy in this precision");
      k_spmv_ell<T><<<(n + kThreads - 1) / kThreads, kThreads, 0, ctx->stream>>>(n, A->d_ell_off, A->d_ell_ci, v_ell, x, y);
      break;
    default: throw Error{AB2_ERR_BAD_ARG, "unknown SpMV variant"};
  }
  check_launch(ctx, "spmv");
}

void op_spmv(ab2_context* ctx, const ab2_matrix* A, const double* x, double* y, int variant) {
  spmv_t<double>(ctx, A, A->d_v, A->d_ell_v, x, y, variant);
}

void op_spmv_f32(ab2_context* ctx, const ab2_matrix* A, const float* x, float* y, int variant) {
  require(A->d_v32 != nullptr, "matrix has no FP32 copy (AB2_FMT_F32)");
  spmv_t<float>(ctx, A, A->d_v32, A->d_ell_v32, x, y, variant);
}

void op_add_lu_mult(ab2_context* ctx, const ab2_matrix* A, double alpha, const double* x, double* y, bool lower) {
  k_add_lu<<<grid_for(A->n), kThreads, 0, ctx->stream>>>(A->n, A->d_rp, A->d_ci, A->d_v, A->d_dcol, alpha, x, y, lower);
  check_launch(ctx, "add_lu_mult");
}

void op_inv_diag(ab2_context* ctx, const ab2_matrix* A, double* inv) {
  k_inv_diag<<<grid_for(A->n), kThreads, 0, ctx->stream>>>(A->n, A->d_rp, A->d_v, A->d_dcol, inv);
  check_launch(ctx, "inv_diag");
}

void op_mult_inv_diag(ab2_context* ctx, const ab2_matrix* A, double* y) {
  k_mult_inv_diag<<<grid_for(A->n), kThreads, 0, ctx->stream>>>(A->n, A->d_rp, A->d_v, A->d_dcol, y);
  check_launch(ctx, "mult_inv_diag");
}

void op_diagonal(ab2_context* ctx, const ab2_matrix* A, double* d) {
  k_diagonal<<<grid_for(A->n), kThreads, 0, ctx->stream>>>(A->n, A->d_rp, A->d_ci, A->d_v, A->d_dcol, d);
  check_launch(ctx, "diagonal");
}

// The 7-point bands from the device CSR values: 7 bands, or 4 when the
// values are bit-for-bit symmetric (re-decided on every value update).
static void refresh_stencil(ab2_context* ctx, ab2_matrix* A) {
  const int n = A->n;
  const size_t N = (size_t)n;
  double* b7 = dev_alloc<double>(ctx, 7 * N);
  k_stencil7_fill<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, A->st_nx, A->st_ny, A->st_nz, A->d_rp, A->d_v, b7);
  check_launch(ctx, "stencil_fill");
  int* d_bad = dev_alloc<int>(ctx, 1);
  AB2_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), ctx->stream));
  k_stencil7_symmetric<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, A->st_nx, A->st_ny, A->st_nz, b7, d_bad);
  check_launch(ctx, "stencil_symmetric");
  int bad = 0;
  AB2_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  dev_free(ctx, d_bad);
  const int nb = bad ? 7 : 4;
  if (nb != A->st_bands) {
    if (A->d_st_v) A->device_bytes -= (long long)(A->st_bands * N * sizeof(double));
    if (A->d_st_v32) A->device_bytes -= (long long)(A->st_bands * N * sizeof(float));
    dev_free(ctx, A->d_st_v);
    dev_free(ctx, A->d_st_v32);
    A->d_st_v = nullptr;
    A->d_st_v32 = nullptr;
    A->st_bands = 0;
    A->d_st_v = dev_alloc<double>(ctx, nb * N, &A->device_bytes);
    if (A->formats & AB2_FMT_F32) A->d_st_v32 = dev_alloc<float>(ctx, nb * N, &A->device_bytes);
    A->st_bands = nb;
  }
  // symmetric: D, Ux, Uy, Uz are the last four of the seven bands
  AB2_CUDA(cudaMemcpyAsync(A->d_st_v, b7 + (7 - nb) * N, sizeof(double) * nb * N, cudaMemcpyDeviceToDevice,
                           ctx->stream));
  dev_free(ctx, b7);
  if (A->d_st_v32) {
    k_to_f32<<<grid_for((long long)nb * n), kThreads, 0, ctx->stream>>>((long long)nb * n, A->d_st_v, A->d_st_v32);
    check_launch(ctx, "stencil_to_f32");
  }
}

// Fills the value arrays (CSR, ELL, the 7-point bands and the FP32 copies)
// from the device CSR values.
static void refresh_values(ab2_context* ctx, ab2_matrix* A) {
  const int n = A->n;
  if (A->st_nx > 0) refresh_stencil(ctx, A);
  if (A->formats & AB2_FMT_ELL) {
    k_ell_fill<double><<<grid_for(n), kThreads, 0, ctx->stream>>>(n, kEllSlice, A->d_rp, A->d_ci, A->d_v, A->d_ell_off, A->d_ell_ci,
                                                                  A->d_ell_v);
    check_launch(ctx, "ell_fill");
  }
  if (A->formats & AB2_FMT_F32) {
    k_to_f32<<<grid_for(A->nnz), kThreads, 0, ctx->stream>>>(A->nnz, A->d_v, A->d_v32);
    check_launch(ctx, "to_f32");
    if (A->formats & AB2_FMT_ELL) {
      k_ell_fill<float><<<grid_for(n), kThreads, 0, ctx->stream>>>(n, kEllSlice, A->d_rp, A->d_ci, A->d_v, A->d_ell_off, A->d_ell_ci,
                                                                  A->d_ell_v32);
      check_launch(ctx, "ell_fill_f32");
    }
  }
}

}  // namespace ab2

namespace ab2 {

EllLayout build_ell_f32(ab2_context* ctx, const ab2_matrix* A, int S) {
  require(S == 16 || S == 32 || S == 64, "ELL slice width must be 16, 32 or 64");
  EllLayout e;
  e.S = S;
  const int n = A->n;
  const int ns = (n + S - 1) / S;
  long long* d_w = dev_alloc<long long>(ctx, (size_t)ns + 1);
  long long* d_woff = dev_alloc<long long>(ctx, (size_t)ns + 1);
  if (ns > 0) {
    k_slice_width<<<grid_for(ns), kThreads, 0, ctx->stream>>>(n, ns, S, A->d_rp, d_w);
    check_launch(ctx, "slice_width");
  }
  k_scan_excl<<<1, 1024, 0, ctx->stream>>>(ns, d_w, d_woff);
  check_launch(ctx, "slice_scan");
  const long long acc = read_ll(ctx, d_woff + ns);
  require(acc < (1LL << 31) && acc * S < (1LL << 31) * 8, "matrix too large for the sliced-ELL layout");
  e.stored = acc * S;
  e.off = dev_alloc<int>(ctx, (size_t)ns + 1);
  e.ci = dev_alloc<int>(ctx, (size_t)e.stored);
  e.v = dev_alloc<float>(ctx, (size_t)e.stored);
  k_narrow<<<grid_for(ns + 1), kThreads, 0, ctx->stream>>>(ns + 1, d_woff, e.off);
  check_launch(ctx, "slice_offsets");
  dev_free(ctx, d_w);
  dev_free(ctx, d_woff);
  const int n_pad = ns * S;
  if (n_pad > n) {
    k_ell_pad_tail<<<1, S, 0, ctx->stream>>>(n, n_pad, S, e.off, e.ci);
    check_launch(ctx, "ell_pad_tail");
  }
  k_ell_fill<float><<<grid_for(n), kThreads, 0, ctx->stream>>>(n, S, A->d_rp, A->d_ci, A->d_v, e.off, e.ci, e.v);
  check_launch(ctx, "ell_fill_f32");
  return e;
}

void free_ell(ab2_context* ctx, EllLayout& e) {
  dev_free(ctx, e.off);
  dev_free(ctx, e.ci);
  dev_free(ctx, e.v);
  e = EllLayout{};
}

void host_profile(const ab2_matrix* A) {
  if (A->h_profile) return;
  ab2_context* ctx = A->ctx;
  A->h_rp.resize((size_t)A->n + 1);
  A->h_ci.resize((size_t)A->nnz);
  AB2_CUDA(cudaMemcpyAsync(A->h_rp.data(), A->d_rp, sizeof(int) * ((size_t)A->n + 1), cudaMemcpyDeviceToHost,
                           ctx->stream));
  if (A->nnz)
    AB2_CUDA(cudaMemcpyAsync(A->h_ci.data(), A->d_ci, sizeof(int) * (size_t)A->nnz, cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  A->h_profile = true;
}

}  // namespace ab2

using namespace ab2;

extern "C" {

int ab2_matrix_create_csr(ab2_context* ctx, int n, const int* row_ptr, const int* cols, const double* vals, int formats,
                          ab2_matrix** out) {
  if (!ctx || !out || n < 0 || !row_ptr || (n > 0 && (!cols || !vals))) return AB2_ERR_BAD_ARG;
  *out = nullptr;
  if (row_ptr[0] != 0 || row_ptr[n] < 0) {
    ctx->last_error = "row_ptr must start at 0 and end at nnz >= 0";
    return AB2_ERR_BAD_ARG;
  }
  ab2_matrix* A = new (std::nothrow) ab2_matrix();
  if (!A) return AB2_ERR_OOM;
  A->ctx = ctx_retain(ctx);
  int rc = guard(ctx, [&] {
    A->n = n;
    A->nnz = row_ptr[n];
    A->formats = (formats | AB2_FMT_CSR);
    const size_t nnz = (size_t)A->nnz;
    A->d_rp = dev_alloc<int>(ctx, (size_t)n + 1, &A->device_bytes);
    A->d_ci = dev_alloc<int>(ctx, nnz, &A->device_bytes);
    A->d_v = dev_alloc<double>(ctx, nnz, &A->device_bytes);
    A->d_dcol = dev_alloc<int>(ctx, (size_t)n, &A->device_bytes);
    AB2_CUDA(cudaMemcpyAsync(A->d_rp, row_ptr, sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice, ctx->stream));
    AB2_CUDA(cudaMemcpyAsync(A->d_ci, cols, sizeof(int) * nnz, cudaMemcpyHostToDevice, ctx->stream));
    AB2_CUDA(cudaMemcpyAsync(A->d_v, vals, sizeof(double) * nnz, cudaMemcpyHostToDevice, ctx->stream));
    if (n > 0) {
      // Device-side profile check: every later kernel indexes x by these columns.
      int* d_bad = dev_alloc<int>(ctx, 1);
      AB2_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), ctx->stream));
      k_validate<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, d_bad);
      check_launch(ctx, "validate");
      int bad = 0;
      AB2_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
      AB2_CUDA(cudaStreamSynchronize(ctx->stream));
      dev_free(ctx, d_bad);
      if (bad & 1) throw Error{AB2_ERR_BAD_ARG, "row_ptr is not non-decreasing"};
      if (bad & 2) throw Error{AB2_ERR_BAD_ARG, "column index out of range"};
      if (bad & 4) throw Error{AB2_ERR_BAD_ARG, "columns must be strictly increasing inside each row"};
      k_dcol<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, A->d_rp, A->d_ci, A->d_dcol);
      check_launch(ctx, "dcol");
    }
    // Row blocks of the staged kernel (the profile is valid from here on).
    {
      const int nc = (n + kThreads - 1) / kThreads;
      long long* d_cnt = dev_alloc<long long>(ctx, (size_t)nc + 1);
      long long* d_off = dev_alloc<long long>(ctx, (size_t)nc + 1);
      if (nc > 0) {
        k_rowblock_count<<<grid_for(nc), kThreads, 0, ctx->stream>>>(n, nc, A->d_rp, d_cnt);
        check_launch(ctx, "rowblock_count");
      }
      k_scan_excl<<<1, 1024, 0, ctx->stream>>>(nc, d_cnt, d_off);
      check_launch(ctx, "rowblock_scan");
      const long long nb = read_ll(ctx, d_off + nc);
      A->n_row_blocks = (int)nb;
      A->d_row_blocks = dev_alloc<int>(ctx, (size_t)nb + 1, &A->device_bytes);
      k_rowblock_emit<<<grid_for(std::max(nc, 1)), kThreads, 0, ctx->stream>>>(n, nc, A->d_rp, d_off, A->d_row_blocks);
      check_launch(ctx, "rowblock_emit");
      dev_free(ctx, d_cnt);
      dev_free(ctx, d_off);
    }
    if (A->formats & AB2_FMT_ELL) {
      const int ns = (n + kEllSlice - 1) / kEllSlice;
      long long* d_w = dev_alloc<long long>(ctx, (size_t)ns + 1);
      long long* d_woff = dev_alloc<long long>(ctx, (size_t)ns + 1);
      if (ns > 0) {
        k_slice_width<<<grid_for(ns), kThreads, 0, ctx->stream>>>(n, ns, kEllSlice, A->d_rp, d_w);
        check_launch(ctx, "slice_width");
      }
      k_scan_excl<<<1, 1024, 0, ctx->stream>>>(ns, d_w, d_woff);
      check_launch(ctx, "slice_scan");
      const long long acc = read_ll(ctx, d_woff + ns);
      require(acc < (1LL << 31) && acc * kEllSlice < (1LL << 31) * 8, "matrix too large for the sliced-ELL layout");
      A->ell_stored = acc * kEllSlice;
      A->d_ell_off = dev_alloc<int>(ctx, (size_t)ns + 1, &A->device_bytes);
      A->d_ell_ci = dev_alloc<int>(ctx, (size_t)A->ell_stored, &A->device_bytes);
      A->d_ell_v = dev_alloc<double>(ctx, (size_t)A->ell_stored, &A->device_bytes);
      k_narrow<<<grid_for(ns + 1), kThreads, 0, ctx->stream>>>(ns + 1, d_woff, A->d_ell_off);
      check_launch(ctx, "slice_offsets");
      dev_free(ctx, d_w);
      dev_free(ctx, d_woff);
      const int n_pad = ns * kEllSlice;
      if (n_pad > n) {
        k_ell_pad_tail<<<1, kEllSlice, 0, ctx->stream>>>(n, n_pad, kEllSlice, A->d_ell_off, A->d_ell_ci);
        check_launch(ctx, "ell_pad_tail");
      }
    }
    if (A->formats & AB2_FMT_F32) {
      A->d_v32 = dev_alloc<float>(ctx, nnz, &A->device_bytes);
      if (A->formats & AB2_FMT_ELL) A->d_ell_v32 = dev_alloc<float>(ctx, (size_t)A->ell_stored, &A->device_bytes);
    }
    if (A->formats & AB2_FMT_STENCIL) {
      // kept only for a 7-point profile; the flag reports what is present
      int nx = 0, ny = 0, nz = 0;
      if (stencil_geometry(ctx, A, &nx, &ny, &nz)) {
        A->st_nx = nx;
        A->st_ny = ny;
        A->st_nz = nz;
      } else {
        A->formats &= ~AB2_FMT_STENCIL;
      }
    }
    refresh_values(ctx, A);
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  });
  if (rc != AB2_OK) {
    ab2_matrix_destroy(A);
    return rc;
  }
  *out = A;
  return AB2_OK;
}

int ab2_matrix_update_values(ab2_context* ctx, ab2_matrix* A, const double* vals) {
  if (!ctx || !A || (!vals && A->nnz)) return AB2_ERR_BAD_ARG;
  return guard(ctx, [&] {
    AB2_CUDA(cudaMemcpyAsync(A->d_v, vals, sizeof(double) * (size_t)A->nnz, cudaMemcpyHostToDevice, ctx->stream));
    refresh_values(ctx, A);
  });
}

int ab2_matrix_destroy(ab2_matrix* A) {
  if (!A) return AB2_ERR_BAD_ARG;
  if (A->ctx) ctx_quiesce(A->ctx);
  dev_free(A->ctx, A->d_rp);
  dev_free(A->ctx, A->d_ci);
  dev_free(A->ctx, A->d_v);
  dev_free(A->ctx, A->d_dcol);
  dev_free(A->ctx, A->d_v32);
  dev_free(A->ctx, A->d_row_blocks);
  dev_free(A->ctx, A->d_ell_off);
  dev_free(A->ctx, A->d_ell_ci);
  dev_free(A->ctx, A->d_ell_v);
  dev_free(A->ctx, A->d_ell_v32);
  dev_free(A->ctx, A->d_st_v);
  dev_free(A->ctx, A->d_st_v32);
  if (A->ctx) ctx_release(A->ctx);
  delete A;
  return AB2_OK;
}

int ab2_matrix_get_info(const ab2_matrix* A, ab2_matrix_info* info) {
  if (!A || !info) return AB2_ERR_BAD_ARG;
  info->n = A->n;
  info->nnz = A->nnz;
  info->ell_stored = A->ell_stored;
  info->ell_slice = kEllSlice;
  info->formats = A->formats;
  info->device_bytes = A->device_bytes;
  info->stencil_bands = A->st_bands;
  info->stencil_nx = A->st_nx;
  info->stencil_ny = A->st_ny;
  info->stencil_nz = A->st_nz;
  return AB2_OK;
}

int ab2_mult(ab2_context* ctx, const ab2_matrix* A, const ab2_vector* x, ab2_vector* y) {
  return ab2_mult_variant(ctx, A, x, y, AB2_SPMV_AUTO);
}

int ab2_mult_variant(ab2_context* ctx, const ab2_matrix* A, const ab2_vector* x, ab2_vector* y, int variant) {
  if (!ctx || !A || !x || !y || x->n != A->n || y->n != A->n || x->d == y->d) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-SPMV");
  return guard(ctx, [&] { op_spmv(ctx, A, x->d, y->d, variant); });
}

int ab2_add_lmult(ab2_context* ctx, double alpha, const ab2_matrix* A, const ab2_vector* x, ab2_vector* y) {
  if (!ctx || !A || !x || !y || x->n != A->n || y->n != A->n || x->d == y->d) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-AddLMult");
  return guard(ctx, [&] { op_add_lu_mult(ctx, A, alpha, x->d, y->d, true); });
}

int ab2_add_umult(ab2_context* ctx, double alpha, const ab2_matrix* A, const ab2_vector* x, ab2_vector* y) {
  if (!ctx || !A || !x || !y || x->n != A->n || y->n != A->n || x->d == y->d) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-AddUMult");
  return guard(ctx, [&] { op_add_lu_mult(ctx, A, alpha, x->d, y->d, false); });
}

int ab2_compute_inv_diag(ab2_context* ctx, const ab2_matrix* A, ab2_vector* inv) {
  if (!ctx || !A || !inv || inv->n != A->n) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-INVDIAG");
  return guard(ctx, [&] { op_inv_diag(ctx, A, inv->d); });
}

int ab2_mult_inv_diag(ab2_context* ctx, const ab2_matrix* A, ab2_vector* y) {
  if (!ctx || !A || !y || y->n != A->n) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-MULTINVDIAG");
  return guard(ctx, [&] { op_mult_inv_diag(ctx, A, y->d); });
}

int ab2_diagonal(ab2_context* ctx, const ab2_matrix* A, ab2_vector* d) {
  if (!ctx || !A || !d || d->n != A->n) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "CSR-DIAGONAL");
  return guard(ctx, [&] { op_diagonal(ctx, A, d->d); });
}

}  // extern "C"
