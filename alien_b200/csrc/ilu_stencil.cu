// ilu_stencil.cu -- ILU(0) factorisation and sweeps scheduled for 7-point
// matrices in lexicographic order.
//
// The arithmetic is exactly the general path's (ILU0Preconditioner.h:156-231:
// same per-row operations, same column order, product and difference rounded
// apart, an IEEE division by the pivot), so factor and applications are bit
// for bit those of the wavefront kernels in precond.cu and of the sequential
// reference.  Only the schedule differs.
//
// In a 3-D 7-point matrix numbered i + nx (j + ny k), row (i,j,k) of the
// forward sweep depends on (i,j,k-1), (i,j-1,k) and (i-1,j,k).  A CTA of
// 16 x 16 threads owns a 16 x 16 tile of z-lines, one thread per line, and
// walks the tile's diagonals i+j+k = s: at step s thread (i,j) computes cell
// k = s - i - j.  Its k-1 input is its own previous value (a register), the
// i-1 and j-1 inputs were computed by neighbouring threads at step s-1 (shared
// memory, one __syncthreads per step).  Only the first line of a tile reads a
// value owned by another tile; those come through global memory with the
// sentinel-value wait of sentinel.cuh, loaded ahead with the band values.
// Tiles are claimed from an atomic ticket in the order the dependencies run (a
// tile waits only on tiles with a smaller ticket), so no co-residency is
// needed.  The backward sweep runs the same walk on the mirrored grid; the
// factorisation runs it too: in a 7-point matrix ILU(0) changes only the
// diagonal, and row (i,j,k) needs the final pivots of the same three
// neighbours (value propagated: the pivot).
//
// Measured on B200 at 192^3 this schedule applies the factor in 1.7 ms
// against 3.45 ms for the wavefront schedule and sets up in ~6 ms instead of
// ~220 ms; a warp-per-8x4-tile variant (shuffles instead of shared memory)
// measured 2.9 ms.  Each step of a walk costs about one L2 round trip, so the
// ~574 dependent steps of a sweep, not bandwidth, bound it.
//
// The factor is kept in eight structure-of-arrays bands (L to -k/-j/-i, U to
// +i/+j/+k, pivot, original diagonal) so each thread's loads are plain
// indexed reads, and a copy in CSR order for ab2_precond_ilu0_values.
#include <cuda_runtime.h>

#include <algorithm>

#include "ab2_internal.cuh"
#include "precond.cuh"
#include "sentinel.cuh"

namespace ab2 {

namespace {

constexpr int kTile = 16;

enum { kFactor = 0, kLower = 1, kUpper = 2 };

struct Geom {
  int nx, ny, nz, ntx, nty;
  long long nxny;
};

struct Bands {
  double *Lk, *Lj, *Li, *Ui, *Uj, *Uk, *P, *D;
};

// Rows must hold exactly the in-grid 7-point neighbours, in ascending columns.
__global__ void k_stencil_check(int n, Geom g, const int* __restrict__ rp, const int* __restrict__ ci, int* bad) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int i = r % g.nx, j = (r / g.nx) % g.ny, k = (int)(r / g.nxny);
    int e = rp[r];
    const int end = rp[r + 1];
    bool ok = true;
    auto expect = [&](long long c) {
      ok = ok && e < end && ci[e] == c;
      ++e;
    };
    if (k > 0) expect(r - g.nxny);
    if (j > 0) expect(r - g.nx);
    if (i > 0) expect(r - 1);
    expect(r);
    if (i < g.nx - 1) expect(r + 1);
    if (j < g.ny - 1) expect(r + g.nx);
    if (k < g.nz - 1) expect(r + g.nxny);
    if (!ok || e != end) atomicOr(bad, 1);
  }
}

__global__ void k_stencil_extract(int n, Geom g, const int* __restrict__ rp, const double* __restrict__ v, Bands b) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int i = r % g.nx, j = (r / g.nx) % g.ny, k = (int)(r / g.nxny);
    int e = rp[r];
    b.Lk[r] = k > 0 ? v[e++] : 0.0;
    b.Lj[r] = j > 0 ? v[e++] : 0.0;
    b.Li[r] = i > 0 ? v[e++] : 0.0;
    b.D[r] = v[e++];
    b.Ui[r] = i < g.nx - 1 ? v[e++] : 0.0;
    b.Uj[r] = j < g.ny - 1 ? v[e++] : 0.0;
    b.Uk[r] = k < g.nz - 1 ? v[e++] : 0.0;
  }
}

__global__ void k_stencil_pack(int n, Geom g, const int* __restrict__ rp, Bands b, double* __restrict__ lu) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int i = r % g.nx, j = (r / g.nx) % g.ny, k = (int)(r / g.nxny);
    int e = rp[r];
    if (k > 0) lu[e++] = b.Lk[r];
    if (j > 0) lu[e++] = b.Lj[r];
    if (i > 0) lu[e++] = b.Li[r];
    lu[e++] = b.P[r];
    if (i < g.nx - 1) lu[e++] = b.Ui[r];
    if (j < g.ny - 1) lu[e++] = b.Uj[r];
    if (k < g.nz - 1) lu[e++] = b.Uk[r];
  }
}

// Per-step inputs loaded prefetch_depth<MODE>() steps ahead: band values of
// the step's cell, and the value owned by the neighbouring tile (bi / bj,
// first line of the tile only), possibly still the sentinel when loaded.
struct Pre {
  double a0, a1, a2, a3, u0, u1, u2, bi, bj;
};

template <int MODE>
__host__ __device__ constexpr int prefetch_depth() {
  return MODE == kFactor ? 4 : 8;
}

template <int MODE>
__global__ void __launch_bounds__(kTile* kTile) k_stencil_wave(Geom g, Bands b, const double* in, double* out,
                                                                double* reset, unsigned int* tickets, int* err) {
  constexpr int kPrefetch = prefetch_depth<MODE>();
  __shared__ double s_val[2][kTile][kTile + 1];
  __shared__ int s_tile;
  const int li = threadIdx.x % kTile, lj = threadIdx.x / kTile;
  const int ntiles = g.ntx * g.nty;
  const int nsteps = g.nz + 2 * (kTile - 1);
  constexpr bool up = MODE == kUpper;
  const int di = up ? 1 : -1;  // global offset of the i-neighbour read (j: di*nx)
  double* wave = MODE == kFactor ? b.P : out;  // the array whose values propagate

  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(tickets + MODE, 1u);
    __syncthreads();
    const int tile = s_tile;
    if (tile >= ntiles) break;
    const int ai = (tile % g.ntx) * kTile + li;  // walk coordinates (mirrored for the U sweep)
    const int aj = (tile / g.ntx) * kTile + lj;
    const bool active = ai < g.nx && aj < g.ny;
    const int gi = up ? g.nx - 1 - ai : ai;
    const int gj = up ? g.ny - 1 - aj : aj;
    const long long line = active ? gi + (long long)g.nx * gj : 0;

    auto cell = [&](int s, long long& r) {
      const int ak = s - li - lj;
      if (!active || ak < 0 || ak >= g.nz) return -1;
      r = line + g.nxny * (up ? g.nz - 1 - ak : ak);
      return ak;
    };
    auto load = [&](int s, Pre& p) {
      long long r = 0;
      if (cell(s, r) < 0) return;
      if (lj == 0 && aj > 0) p.bj = ld_relaxed(wave + r + di * (long long)g.nx);
      if (li == 0 && ai > 0) p.bi = ld_relaxed(wave + r + di);
      if (MODE == kFactor) {
        p.a0 = b.D[r];
        p.a1 = b.Lk[r];
        p.a2 = b.Lj[r];
        p.a3 = b.Li[r];
        p.u0 = r >= g.nxny ? b.Uk[r - g.nxny] : 0.0;
        p.u1 = r >= g.nx ? b.Uj[r - g.nx] : 0.0;
        p.u2 = r >= 1 ? b.Ui[r - 1] : 0.0;
      } else if (MODE == kLower) {
        p.a0 = in[r];
        p.a1 = b.Lk[r];
        p.a2 = b.Lj[r];
        p.a3 = b.Li[r];
      } else {
        p.a0 = in[r];
        p.a1 = b.Ui[r];
        p.a2 = b.Uj[r];
        p.a3 = b.Uk[r];
        p.u0 = b.P[r];
      }
    };

    Pre pre[kPrefetch];
#pragma unroll
    for (int u = 0; u < kPrefetch; ++u) {
      pre[u] = Pre{0, 0, 0, 0, 0, 0, 0, 0, 0};
      load(u, pre[u]);
    }
    double own = 0.0;
    for (int s0 = 0; s0 < nsteps; s0 += kPrefetch) {
#pragma unroll
      for (int u = 0; u < kPrefetch; ++u) {
        const int s = s0 + u;
        if (s < nsteps) {
          const Pre c = pre[u];
          load(s + kPrefetch, pre[u]);
          long long r = 0;
          const int ak = cell(s, r);
          double val = 0.0;
          if (ak >= 0) {
            const double* prev = &s_val[(s + 1) & 1][0][0];
            double vi = 0.0, vj = 0.0;
            if (aj > 0) {
              vj = lj > 0 ? prev[(lj - 1) * (kTile + 1) + li]
                          : (is_sentinel(c.bj) ? wait_value(wave + r + di * (long long)g.nx, err) : c.bj);
            }
            if (ai > 0) {
              vi = li > 0 ? prev[lj * (kTile + 1) + li - 1] : (is_sentinel(c.bi) ? wait_value(wave + r + di, err) : c.bi);
            }
            if (MODE == kFactor) {
              // a_ik /= pivot_k, then a_ii -= a_ik a_ki, columns ascending (-k, -j, -i)
              double d = c.a0;
              if (ak > 0) {
                const double l = c.a1 / own;
                d = mul_sub_rn(l, c.u0, d);
                b.Lk[r] = l;
              }
              if (aj > 0) {
                const double l = c.a2 / vj;
                d = mul_sub_rn(l, c.u1, d);
                b.Lj[r] = l;
              }
              if (ai > 0) {
                const double l = c.a3 / vi;
                d = mul_sub_rn(l, c.u2, d);
                b.Li[r] = l;
              }
              val = d;
            } else if (MODE == kLower) {
              double acc = c.a0;  // columns ascending: -k, -j, -i
              if (ak > 0) acc = mul_sub_rn(c.a1, own, acc);
              if (aj > 0) acc = mul_sub_rn(c.a2, vj, acc);
              if (ai > 0) acc = mul_sub_rn(c.a3, vi, acc);
              reset[r] = sentinel_value();  // after in[r] was read: in and reset may alias
              val = acc;
            } else {
              double acc = c.a0;  // columns ascending: +i, +j, +k
              if (ai > 0) acc = mul_sub_rn(c.a1, vi, acc);
              if (aj > 0) acc = mul_sub_rn(c.a2, vj, acc);
              if (ak > 0) acc = mul_sub_rn(c.a3, own, acc);
              reset[r] = sentinel_value();
              val = acc / c.u0;
            }
            st_relaxed(wave + r, not_sentinel(val));
            own = val;
          }
          s_val[s & 1][lj][li] = val;
          __syncthreads();
        }
      }
    }
  }
  // Hand the other sweep its ticket back (it does not run concurrently).
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (MODE == kLower) tickets[kUpper] = 0u;
    if (MODE == kUpper) tickets[kLower] = 0u;
  }
}

Geom geom_of(const Ilu0Data& d) {
  Geom g;
  g.nx = d.st_nx;
  g.ny = d.st_ny;
  g.nz = d.st_nz;
  g.ntx = (g.nx + kTile - 1) / kTile;
  g.nty = (g.ny + kTile - 1) / kTile;
  g.nxny = (long long)g.nx * g.ny;
  return g;
}

Bands bands_of(const Ilu0Data& d, int n) {
  double* p = d.d_bands;
  const size_t m = (size_t)n;
  return Bands{p, p + m, p + 2 * m, p + 3 * m, p + 4 * m, p + 5 * m, p + 6 * m, p + 7 * m};
}

int wave_grid(ab2_context* ctx, const Geom& g) { return std::max(1, std::min(g.ntx * g.nty, ctx->num_sms * 2)); }

}  // namespace

bool ilu_stencil_setup(ab2_context* ctx, const ab2_matrix* A, Ilu0Data& d) {
  const int n = A->n;
  const int* rp = A->h_rp.data();
  const int* ci = A->h_ci.data();
  // Geometry from the first full row: its columns start r - nx ny, r - nx.
  int r7 = -1;
  for (int r = 0; r < n; ++r)
    if (rp[r + 1] - rp[r] == 7) {
      r7 = r;
      break;
    }
  if (r7 < 0) return false;
  const long long nxny = (long long)r7 - ci[rp[r7]];
  const long long nx = (long long)r7 - ci[rp[r7] + 1];
  if (nx < 2 || nxny <= nx || nxny % nx != 0 || n % nxny != 0) return false;
  const long long ny = nxny / nx, nz = n / nxny;
  if (ny < 2 || nz < 2) return false;
  d.st_nx = (int)nx;
  d.st_ny = (int)ny;
  d.st_nz = (int)nz;
  const Geom g = geom_of(d);
  int* d_bad = dev_alloc<int>(1);
  AB2_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), ctx->stream));
  k_stencil_check<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, g, A->d_rp, A->d_ci, d_bad);
  check_launch(ctx, "stencil_check");
  int bad = 0;
  AB2_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  dev_free(d_bad);
  if (bad) return false;

  d.d_bands = dev_alloc<double>((size_t)n * 8);
  d.d_tile_tickets = dev_alloc<unsigned int>(3);
  AB2_CUDA(cudaMemsetAsync(d.d_tile_tickets, 0, 3 * sizeof(unsigned int), ctx->stream));
  const Bands b = bands_of(d, n);
  k_stencil_extract<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, g, A->d_rp, A->d_v, b);
  check_launch(ctx, "stencil_extract");
  k_fill_bits<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, kSentinel, b.P);
  check_launch(ctx, "stencil_fill");
  k_stencil_wave<kFactor><<<wave_grid(ctx, g), kTile * kTile, 0, ctx->stream>>>(g, b, nullptr, nullptr, nullptr,
                                                                                d.d_tile_tickets, d.d_err);
  check_launch(ctx, "stencil_factor");
  k_stencil_pack<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, g, A->d_rp, b, d.d_lu);
  check_launch(ctx, "stencil_pack");
  d.stencil = true;
  d.levels_l = d.levels_u = (int)(nx + ny + nz - 2);
  return true;
}

// y -> d_tmp (forward walk; leaves z at the sentinel) -> z (backward walk;
// puts d_tmp back to the sentinel).
void ilu_stencil_apply(ab2_context* ctx, const ab2_matrix* A, const Ilu0Data& d, const double* y, double* z) {
  const Geom g = geom_of(d);
  const Bands b = bands_of(d, A->n);
  k_stencil_wave<kLower><<<wave_grid(ctx, g), kTile * kTile, 0, ctx->stream>>>(g, b, y, d.d_tmp, z, d.d_tile_tickets,
                                                                               d.d_err);
  check_launch(ctx, "stencil_lsweep");
  k_stencil_wave<kUpper><<<wave_grid(ctx, g), kTile * kTile, 0, ctx->stream>>>(g, b, d.d_tmp, z, d.d_tmp,
                                                                               d.d_tile_tickets, d.d_err);
  check_launch(ctx, "stencil_usweep");
}

// The sweeps' propagation vector (d_tmp) is refilled by pc_reset; nothing else
// of this schedule needs resetting besides the tickets.
void ilu_stencil_reset(ab2_context* ctx, const Ilu0Data& d) {
  (void)ctx;
  (void)d;
}

}  // namespace ab2
