// ilu_stencil.cu -- ILU(0) factorisation and sweeps scheduled for 7-point
// matrices in lexicographic order.
//
// The arithmetic is exactly the general path's (ILU0Preconditioner.h:156-231:
// same per-row operations, same column order, product and difference rounded
// apart, an IEEE division by the pivot), so factor and applications are bit
// for bit those of the wavefront kernels in precond.cu and of the sequential
// reference.  Only the schedule differs.
//
// Schedule.  In a 3-D 7-point matrix numbered i + nx (j + ny k), row (i,j,k)
// of the forward sweep depends on (i,j,k-1), (i,j-1,k) and (i-1,j,k).  A CTA
// of 16 x 16 threads owns a 16 x 16 tile of z-lines, one thread per line, and
// walks the tile's diagonals: at step s thread (li,lj) computes cell
// k = s - li - lj.  Its k-1 input is its own previous value (a register), the
// i-1 and j-1 inputs were computed by neighbouring threads at step s-1 (shared
// memory, one named barrier per step).  Only the first line of a tile reads a
// value owned by another tile, 15 steps ahead in that tile's walk; those come
// through global memory (the sentinel values of sentinel.cuh), fetched by a
// ninth, polling warp that hands them over through shared memory.  Tiles
// are claimed from an atomic ticket in dependency order (a tile waits only on
// tiles with a smaller ticket), so no co-residency is needed.
//
// Walk layout.  At one step the 256 threads of a tile touch 31 different
// z-planes, so in natural order every warp access would be 32 separate cache
// lines, and a step would cost the LSU ~1.2 us instead of ~0.16 us (measured on
// B200 for this access pattern against the same walk on contiguous data).  The
// sweeps therefore read and write arrays stored in WALK order: index
// ((tile * nsteps + s) * 256 + thread), nsteps = nz + 30 rounded up to the
// prefetch depth, so one warp access is 32 consecutive doubles.  The factor
// bands are gathered into that order once at set-up; each application gathers
// y in (one bulk kernel), runs the two walks, and scatters z out (one bulk
// kernel) -- bulk kernels have the whole GPU to hide latency, a wavefront
// step does not.  Those two are transposes through shared memory
// (k_walk_gather_t / k_walk_scatter_t), contiguous on both sides; against
// element-wise gather/scatter they saved ~30 us per application at 192^3
// (14 ms per CG+ILU0 solve of 286 applications, measured before the poll
// warp below).
//
// The backward sweep is the forward walk run backwards: the U walk's thread
// (li,lj) of tile T at step s handles the cell the L walk handles at the
// mirrored position (15-li, 15-lj, ntiles-1-T, nsteps-1-s), whose walk index is
// walk_n - 1 - w (the U walk's cells then start nsteps - nz - 30 steps
// late).  So both walks use the same arrays, the U walk through the reversed
// index, and both are coalesced.  Its dependencies (+i, +j, +k) are
// then again "previous thread / previous tile / own previous step".
//
// The factorisation runs once per set-up on the natural-order bands with the
// same walk (pivots propagate; in a 7-point matrix ILU(0) changes only the
// diagonal and the L values).
//
// Measured on B200, one application at 192^3: 0.61 ms (gather + two walks +
// scatter; 0.97 ms before the poll warp), against 1.69 ms for the same walk
// on natural-order arrays and 3.45 ms for the wavefront schedule of
// precond.cu.  Values loaded per poll round: 4 steps (2: 0.63 ms, 3: 0.60,
// 8: 0.63, 16: 0.70).  The cluster walk further down (2 x 2 tiles a cluster,
// hand-offs inside a cluster through distributed shared memory, step inputs
// by bulk copy): 0.551 ms.
//
// Where the time goes (per-tile timestamps of one L walk at 192^3, 144
// tiles): a tile without upstream tiles steps in 0.265 us; tiles downstream
// step in 0.34-0.42 us, since every step waits for a value its neighbour
// produced 15 steps earlier plus the hand-off; a tile starts its walk ~8.5 us
// (16 neighbour steps + hand-off) after its upstream tile.  The critical path
// is 22 such lags plus one tile's walk: ~263 us.  The dependency depth
// (nx + ny + nz - 2 = 574 steps) at the lone tile's step time would be 152 us.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <type_traits>

#include "ab2_internal.cuh"
#include "precond.cuh"
#include "sentinel.cuh"

namespace ab2 {

namespace cg = cooperative_groups;

namespace {

constexpr int kTile = 16;
constexpr int kTileThreads = kTile * kTile;
constexpr int kWalkPrefetch = 8;  // steps a walk loads ahead; the walk length is padded to a multiple
// The sweeps' poll warp: steps whose neighbouring-tile values it loads per
// round (all in flight at once), and the shared-memory ring it hands them to
// the compute warps through.
constexpr int kPollDepth = 4;
constexpr int kBndRing = 16;
static_assert(kBndRing >= kPollDepth, "a poll round fits in the ring");

struct Geom {
  int nx, ny, nz, ntx, nty;
  long long nxny;
};

struct Bands {
  double *Lk, *Lj, *Li, *Ui, *Uj, *Uk, *P, *D;
};

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

// The factorisation walk (set-up only, natural-order bands): row (i,j,k)
// divides its L entries by the pivots of its -k, -j, -i neighbours and
// subtracts l * u (the neighbour's U entry towards this row) from its diagonal,
// columns ascending; the resulting pivot propagates.
struct PreF {
  double d, lk, lj, li, uk, uj, ui, bi, bj;
};

__global__ void __launch_bounds__(kTileThreads) k_stencil_factor(Geom g, Bands b, unsigned int* tickets, int* err) {
  constexpr int kPrefetch = 4;
  __shared__ double s_val[2][kTile][kTile + 1];
  __shared__ int s_tile;
  const int li = threadIdx.x % kTile, lj = threadIdx.x / kTile;
  const int ntiles = g.ntx * g.nty;
  const int nsteps = g.nz + 2 * (kTile - 1);
  double* wave = b.P;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(tickets, 1u);
    __syncthreads();
    const int tile = s_tile;
    if (tile >= ntiles) break;
    const int ai = (tile % g.ntx) * kTile + li;
    const int aj = (tile / g.ntx) * kTile + lj;
    const bool active = ai < g.nx && aj < g.ny;
    const long long line = active ? ai + (long long)g.nx * aj : 0;
    auto cell = [&](int s, long long& r) {
      const int ak = s - li - lj;
      if (!active || ak < 0 || ak >= g.nz) return -1;
      r = line + g.nxny * ak;
      return ak;
    };
    auto load = [&](int s, PreF& p) {
      long long r = 0;
      if (cell(s, r) < 0) return;
      if (lj == 0 && aj > 0) p.bj = ld_relaxed(wave + r - g.nx);
      if (li == 0 && ai > 0) p.bi = ld_relaxed(wave + r - 1);
      p.d = b.D[r];
      p.lk = b.Lk[r];
      p.lj = b.Lj[r];
      p.li = b.Li[r];
      p.uk = r >= g.nxny ? b.Uk[r - g.nxny] : 0.0;
      p.uj = r >= g.nx ? b.Uj[r - g.nx] : 0.0;
      p.ui = r >= 1 ? b.Ui[r - 1] : 0.0;
    };
    PreF pre[kPrefetch];
#pragma unroll
    for (int u = 0; u < kPrefetch; ++u) {
      pre[u] = PreF{0, 0, 0, 0, 0, 0, 0, 0, 0};
      load(u, pre[u]);
    }
    double own = 0.0;
    for (int s0 = 0; s0 < nsteps; s0 += kPrefetch) {
#pragma unroll
      for (int u = 0; u < kPrefetch; ++u) {
        const int s = s0 + u;
        if (s < nsteps) {
          const PreF c = pre[u];
          load(s + kPrefetch, pre[u]);
          long long r = 0;
          const int ak = cell(s, r);
          double val = 0.0;
          if (ak >= 0) {
            const double* prev = &s_val[(s + 1) & 1][0][0];
            double vi = 0.0, vj = 0.0;
            if (aj > 0)
              vj = lj > 0 ? prev[(lj - 1) * (kTile + 1) + li]
                          : (is_sentinel(c.bj) ? wait_value(wave + r - g.nx, err) : c.bj);
            if (ai > 0)
              vi = li > 0 ? prev[lj * (kTile + 1) + li - 1] : (is_sentinel(c.bi) ? wait_value(wave + r - 1, err) : c.bi);
            double d = c.d;  // a_ik /= pivot_k, then a_ii -= a_ik a_ki, columns ascending (-k, -j, -i)
            if (ak > 0) {
              const double l = c.lk / own;
              d = mul_sub_rn(l, c.uk, d);
              b.Lk[r] = l;
            }
            if (aj > 0) {
              const double l = c.lj / vj;
              d = mul_sub_rn(l, c.uj, d);
              b.Lj[r] = l;
            }
            if (ai > 0) {
              const double l = c.li / vi;
              d = mul_sub_rn(l, c.ui, d);
              b.Li[r] = l;
            }
            val = d;
            st_relaxed(wave + r, not_sentinel(val));
            own = val;
          }
          s_val[s & 1][lj][li] = val;
          __syncthreads();
        }
      }
    }
  }
}

// ------------------------------------------------------------------ walk layout
struct Walk {
  int nx, ny, nz, ntx, nty, nsteps;
  long long nxny, nw;  // nw = ntx nty nsteps 256
};

// The natural row handled at walk index w of the L walk, or -1 (padding).
__device__ __forceinline__ long long walk_row(const Walk& g, long long w) {
  const int t = (int)(w & (kTileThreads - 1));
  const long long q = w >> 8;
  const int s = (int)(q % g.nsteps);
  const int tile = (int)(q / g.nsteps);
  const int li = t & (kTile - 1), lj = t >> 4;
  const int i = (tile % g.ntx) * kTile + li, j = (tile / g.ntx) * kTile + lj, k = s - li - lj;
  if (i >= g.nx || j >= g.ny || k < 0 || k >= g.nz) return -1;
  return i + (long long)g.nx * j + g.nxny * k;
}

// dst[w] = src[row(w)] (0 on padding), rounded to T (the FP32 walk arrays
// are gathered from the FP64 factor).
template <class S, class T>
__global__ void k_walk_gather(Walk g, const S* __restrict__ src, T* __restrict__ dst) {
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < g.nw; w += (long long)gridDim.x * blockDim.x) {
    const long long r = walk_row(g, w);
    dst[w] = r >= 0 ? (T)__ldg(src + r) : T(0);
  }
}

// dst[row(w)] = src[w], and src[w] back to the sentinel for the next walk
// (element-wise; the FP32 walk's scatter).
template <class T>
__global__ void k_walk_scatter(Walk g, T* __restrict__ src, T* __restrict__ dst) {
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < g.nw; w += (long long)gridDim.x * blockDim.x) {
    const long long r = walk_row(g, w);
    if (r >= 0) {
      dst[r] = src[w];
      src[w] = sentinel_of<T>();
    }
  }
}

// Walk order <-> natural order for every application (y in, z out), both
// sides coalesced.  A thread keeps one grid line (li, lj) of a tile: at walk
// step s it owns cell k = s - li - lj, so at one step a warp touches 32
// consecutive walk entries, and at one plane k a warp touches two runs of 16
// consecutive natural rows.  Each thread stages its own cells in a ring of
// planes in shared memory (its own column: no barrier) and moves a plane
// once every lane has it.  One CTA per (tile, kTrPlanes planes).
// Measured per application at 192^3 (planes a CTA / batch): 64/4 550 us,
// 64/8 598, 64/16 555, 96/8 583, 96/12 542, 96/16 542, 96/20 551, 96/24 553,
// 96/32 561, 128/16 551, 128/24 564, 192/16 560.
constexpr int kTrPlanes = 96;
constexpr int kTrBatch = 12;                         // steps (planes) per batch
constexpr int kTrRing = 2 * (kTile - 1) + kTrBatch;  // planes live at once per thread

template <class T>
constexpr int tr_smem() {
  return kTrRing * kTileThreads * (int)sizeof(T);
}

// dst[row(w)] = src[w], and src[w] back to the sentinel for the next walk.
template <class T>
__global__ void __launch_bounds__(kTileThreads) k_walk_scatter_t(Walk g, T* __restrict__ src, T* __restrict__ dst) {
  extern __shared__ unsigned char tr_smem_raw[];
  T* ring = reinterpret_cast<T*>(tr_smem_raw);
  const int nch = (g.nz + kTrPlanes - 1) / kTrPlanes;
  const int tile = blockIdx.x / nch, ch = blockIdx.x - tile * nch;
  const int t = threadIdx.x, li = t & (kTile - 1), lj = t >> 4, d = li + lj;
  const int i = (tile % g.ntx) * kTile + li, j = (tile / g.ntx) * kTile + lj;
  const bool line = i < g.nx && j < g.ny;
  const int k0 = ch * kTrPlanes, k1 = min(g.nz, k0 + kTrPlanes);
  const long long wb = (long long)tile * g.nsteps * kTileThreads + t;
  const long long rb = i + (long long)g.nx * j;
  int out = k0;
  for (int s0 = k0; s0 < k1 + 2 * (kTile - 1); s0 += kTrBatch) {
    // the batch's loads first (all in flight together), then the stores
    T v[kTrBatch];
#pragma unroll
    for (int u = 0; u < kTrBatch; ++u) {
      const int k = s0 + u - d;
      v[u] = (line && k >= k0 && k < k1) ? __ldcs(src + wb + (long long)(s0 + u) * kTileThreads) : T(0);
    }
#pragma unroll
    for (int u = 0; u < kTrBatch; ++u) {
      const int k = s0 + u - d;
      if (line && k >= k0 && k < k1) {
        ring[(k % kTrRing) * kTileThreads + t] = v[u];
        src[wb + (long long)(s0 + u) * kTileThreads] = sentinel_of<T>();
      }
    }
    const int last = min(k1, s0 + kTrBatch - 2 * (kTile - 1));  // planes every lane has read
    for (; out < last; ++out)
      if (line) dst[rb + g.nxny * out] = ring[(out % kTrRing) * kTileThreads + t];
  }
}

// dst[w] = src[row(w)] for the cells of the grid (padding entries are left
// as they are: zero since set-up).
template <class T>
__global__ void __launch_bounds__(kTileThreads) k_walk_gather_t(Walk g, const T* __restrict__ src, T* __restrict__ dst) {
  extern __shared__ unsigned char tr_smem_raw[];
  T* ring = reinterpret_cast<T*>(tr_smem_raw);
  const int nch = (g.nz + kTrPlanes - 1) / kTrPlanes;
  const int tile = blockIdx.x / nch, ch = blockIdx.x - tile * nch;
  const int t = threadIdx.x, li = t & (kTile - 1), lj = t >> 4, d = li + lj;
  const int i = (tile % g.ntx) * kTile + li, j = (tile / g.ntx) * kTile + lj;
  const bool line = i < g.nx && j < g.ny;
  const int k0 = ch * kTrPlanes, k1 = min(g.nz, k0 + kTrPlanes);
  const long long wb = (long long)tile * g.nsteps * kTileThreads + t;
  const long long rb = i + (long long)g.nx * j;
  int s = k0;  // next step to write
  for (int p0 = k0; p0 < k1 + 2 * (kTile - 1); p0 += kTrBatch) {
    T v[kTrBatch];
#pragma unroll
    for (int u = 0; u < kTrBatch; ++u) {
      const int k = p0 + u;
      v[u] = (line && k < k1) ? __ldcs(src + rb + g.nxny * k) : T(0);
    }
#pragma unroll
    for (int u = 0; u < kTrBatch; ++u) {
      const int k = p0 + u;
      if (line && k < k1) ring[(k % kTrRing) * kTileThreads + t] = v[u];
    }
    const int last = p0 + kTrBatch;  // steps whose cells every lane has read
    for (; s < last; ++s) {
      const int k = s - d;
      if (line && k >= k0 && k < k1) dst[wb + (long long)s * kTileThreads] = ring[(k % kTrRing) * kTileThreads + t];
    }
  }
}

template <class T>
void set_transpose_smem() {
  AB2_CUDA(cudaFuncSetAttribute(k_walk_scatter_t<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, tr_smem<T>()));
  AB2_CUDA(cudaFuncSetAttribute(k_walk_gather_t<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, tr_smem<T>()));
}

template <class T>
struct WalkArrays {
  const T *Lk, *Lj, *Li, *Ui, *Uj, *Uk, *P;
};

// Per-step inputs of a compute thread, loaded kWalkPrefetch steps ahead: the
// right-hand side, three band values (L: -k,-j,-i ; U: +i,+j,+k) and the
// pivot (U walk).
template <class T>
struct PreW {
  T y, a1, a2, a3, piv;
};

__device__ __forceinline__ void compute_bar() { asm volatile("bar.sync 1, %0;" ::"n"(kTileThreads) : "memory"); }

template <class T>
__device__ __forceinline__ T quiet_nan();
template <>
__device__ __forceinline__ double quiet_nan<double>() {
  return __longlong_as_double(0x7FF8000000000000LL);
}
template <>
__device__ __forceinline__ float quiet_nan<float>() {
  return __uint_as_float(0x7FC00000u);
}

// One triangular sweep in walk layout.  UP = false: forward sweep
// x_i = y_i - sum_{k<dcol} l_ik x_k (solveL, ILU0Preconditioner.h:181-198) from
// `in` into `wave`.  UP = true: backward sweep x_i = (y_i - sum_{k>dcol} u_ik x_k)
// / u_ii (solveU, :200-231), reading `in` through the reversed index and
// putting it back to the sentinel.  `wave` must hold the sentinel on entry.
//
// A CTA is 8 compute warps (the 16 x 16 lines of a tile, synchronised per
// step on named barrier 1) and one poll warp.  The 32 values a step needs
// from the two neighbouring tiles (the first line's inputs: lane l < 16 the
// j-side value of line (l, 0), lane 16 + l the i-side value of line (0, l))
// are fetched by the poll warp: each round it loads the next kPollDepth
// steps' values at once, publishes the leading steps whose values have all
// arrived into a ring in shared memory (s_ready = last published step), and
// reloads the rest in the next round.  A compute thread on the first line
// spins on s_ready in shared memory, not on a global load.  Why: a tile's
// first steps run right behind its neighbour's; a compute warp that found
// the sentinel and polled L2 itself paid a full round trip inside every such
// step (about 1 us against a 0.26 us step), and the next tile waits on those
// steps -- at 192^3 that cost 16-18 us per tile boundary on the critical
// path.  With the polls in flight beside the compute, a step waits only for
// the value's arrival.
//
// Every wait is bounded (kWaitCycles without progress): the poll warp then
// records the error and publishes quiet NaNs, so the compute warps and the
// kernel always finish.
//
// Compute warps: a step is a handful of instructions per thread, and every
// array is reached through a per-thread pointer that moves once per group of
// kWalkPrefetch steps, with constant offsets inside the unrolled group.
template <bool UP, class T>
__global__ void __launch_bounds__(kTileThreads + 32, 1) k_walk_sweep(Walk g, WalkArrays<T> b, T* in, T* wave,
                                                                   unsigned int* tickets, int* err) {
  constexpr int kPre = kWalkPrefetch;
  constexpr long long kStep = UP ? -kTileThreads : kTileThreads;  // element stride of one step
  __shared__ T s_val[2][kTile][kTile + 1];
  __shared__ T s_bnd[kBndRing][2 * kTile];
  __shared__ int s_tile;
  __shared__ volatile int s_ready;  // last step whose neighbouring values are in s_bnd
  __shared__ volatile int s_done;   // last step the compute warps have finished
  const bool poller = threadIdx.x >= kTileThreads;
  const int lane = threadIdx.x & 31;
  // The line this thread computes (compute warps) or feeds (poll warp).
  const int li = poller ? (lane < kTile ? lane : 0) : threadIdx.x % kTile;
  const int lj = poller ? (lane < kTile ? 0 : lane - kTile) : threadIdx.x / kTile;
  const int ntiles = g.ntx * g.nty;
  const int nsteps = g.nsteps;
  // Walk coordinates of the grid's first cell (the U walk's tiles are the
  // mirror images of the L walk's, so a partial tile comes first, and its
  // cells start nsteps - nz - 30 steps into the walk).
  const int ox = UP ? g.ntx * kTile - g.nx : 0;
  const int oy = UP ? g.nty * kTile - g.ny : 0;
  const int oz = UP ? nsteps - g.nz - 2 * (kTile - 1) : 0;
  auto phys = [&](long long w) { return UP ? g.nw - 1 - w : w; };

  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      s_tile = (int)atomicAdd(tickets + (UP ? 2 : 1), 1u);
      s_ready = -1;
      s_done = -1;
    }
    __syncthreads();
    const int tile = s_tile;
    if (tile >= ntiles) break;
    const int ai = (tile % g.ntx) * kTile + li;
    const int aj = (tile / g.ntx) * kTile + lj;
    const bool active = ai >= ox && ai < ox + g.nx && aj >= oy && aj < oy + g.ny;
    const bool has_i = ai > ox, has_j = aj > oy;  // walk predecessor along i / j
    const bool bnd_i = li == 0 && has_i, bnd_j = lj == 0 && has_j;  // that predecessor is in another tile
    // valid steps: s_lo <= s < s_hi (cell k = s - li - lj - oz in [0, nz))
    const int s_lo = active ? li + lj + oz : nsteps;
    const int s_hi = active ? s_lo + g.nz : nsteps;
    const long long tbase = (long long)tile * nsteps * kTileThreads;

    if (poller) {
      // Neighbouring tile's cell at the same k: 15 steps further in that
      // tile's walk (its last line along i, resp. j).
      const bool need = lane < kTile ? bnd_j : bnd_i;
      if (!__any_sync(0xffffffffu, need)) continue;  // first tile row and column: nothing to fetch
      const long long w_nb =
          lane < kTile ? phys(tbase - (long long)g.ntx * nsteps * kTileThreads + 15 * kTileThreads + 15 * kTile + li)
                       : phys(tbase - (long long)nsteps * kTileThreads + 15 * kTileThreads + lj * kTile + 15);
      const T* p_nb = wave + (need ? w_nb : 0);
      long long t_last = clock64();
      bool failed = false;
      for (int t = 0; t < nsteps;) {
        // ring space: slot (t + d) % kBndRing is free once step t + d - kBndRing is done
        const int space = __shfl_sync(0xffffffffu, s_done, 0) + kBndRing - t + 1;
        if (space <= 0) {
          __nanosleep(64);
          bool stop = (clock64() - t_last > kWaitCycles) || *(volatile int*)err;
          if (__any_sync(0xffffffffu, stop)) {  // the compute warps stopped progressing: give up
            if (lane == 0) atomicOr(err, 1);
            break;
          }
          continue;
        }
        T v[kPollDepth];
#pragma unroll
        for (int d = 0; d < kPollDepth; ++d) {
          const int st = t + d;
          v[d] = (need && st >= s_lo && st < s_hi && !failed) ? ld_relaxed(p_nb + (long long)st * kStep) : T(0);
        }
        int first_missing = kPollDepth;
#pragma unroll
        for (int d = kPollDepth - 1; d >= 0; --d) {
          const int st = t + d;
          if (need && st >= s_lo && st < s_hi && is_sentinel(v[d]) && !failed) first_missing = d;
        }
        int n_pub = __reduce_min_sync(0xffffffffu, first_missing);
        if (n_pub == 0) {
          bool stop = (clock64() - t_last > kWaitCycles) || *(volatile int*)err;
          if (__any_sync(0xffffffffu, stop)) {
            // give up on the missing values: quiet NaNs from here on
            if (lane == 0) atomicOr(err, 1);
            failed = true;
          }
          continue;
        }
        n_pub = min(n_pub, space);
#pragma unroll
        for (int d = 0; d < kPollDepth; ++d) {
          const int st = t + d;
          if (d < n_pub && need && st >= s_lo && st < s_hi)
            s_bnd[st % kBndRing][lane] = failed ? quiet_nan<T>() : v[d];
        }
        __syncwarp();
        if (lane == 0) {
          __threadfence_block();
          s_ready = t + n_pub - 1;
        }
        t += n_pub;
        t_last = clock64();
      }
      continue;
    }

    // Compute warps.  Step-0 pointers: own cell at walk index tbase + thread.
    const long long w_own = phys(tbase + threadIdx.x);
    const T* p_y = in + w_own;
    const T* p_a1 = (UP ? b.Ui : b.Lk) + w_own;
    const T* p_a2 = (UP ? b.Uj : b.Lj) + w_own;
    const T* p_a3 = (UP ? b.Uk : b.Li) + w_own;
    const T* p_piv = b.P + w_own;
    T* p_in = in + w_own;
    T* p_out = wave + w_own;

    // Loads of step s (offset o = s * kStep from the step-0 pointers).
    auto load = [&](int s, long long o, PreW<T>& p) {
      if (s < s_lo || s >= s_hi) return;
      // Read-only path: none of these is written during the walk except
      // in[] by the U walk, after its one read here.
      p.y = __ldg(p_y + o);
      p.a1 = __ldg(p_a1 + o);
      p.a2 = __ldg(p_a2 + o);
      p.a3 = __ldg(p_a3 + o);
      if (UP) p.piv = __ldg(p_piv + o);
    };
    // The step's neighbouring-tile values, from the poll warp's ring.
    auto boundary = [&](int s, T& vi, T& vj) {
      if (s_ready < s) {
        const long long t0 = clock64();
        for (unsigned it = 1; s_ready < s; ++it) {
          if ((it & 255) == 0 && (clock64() - t0 > kWaitCycles || *(volatile int*)err)) {
            atomicOr(err, 1);
            vi = vj = quiet_nan<T>();
            return;
          }
        }
      }
      __threadfence_block();
      if (bnd_j) vj = s_bnd[s % kBndRing][li];
      if (bnd_i) vi = s_bnd[s % kBndRing][kTile + lj];
    };

    PreW<T> pre[kPre];
#pragma unroll
    for (int u = 0; u < kPre; ++u) {
      pre[u] = PreW<T>{0, 0, 0, 0, 0};
      load(u, u * kStep, pre[u]);
    }
    T own = 0;
    for (int s0 = 0; s0 < nsteps; s0 += kPre) {  // nsteps is a multiple of kPre
      const long long o0 = (long long)s0 * kStep;
#pragma unroll
      for (int u = 0; u < kPre; ++u) {
        const int s = s0 + u;
        const long long o = o0 + u * kStep;
        const PreW<T> c = pre[u];
        load(s + kPre, o + kPre * kStep, pre[u]);
        T val = 0;
        if (s >= s_lo && s < s_hi) {
          const T* prev = &s_val[(s + 1) & 1][0][0];
          T vi = 0, vj = 0;
          if (bnd_i || bnd_j) boundary(s, vi, vj);
          if (has_j && lj > 0) vj = prev[(lj - 1) * (kTile + 1) + li];
          if (has_i && li > 0) vi = prev[lj * (kTile + 1) + li - 1];
          const bool has_k = s > s_lo;
          T acc = c.y;
          if (!UP) {  // columns ascending: -k, -j, -i
            if (has_k) acc = mul_sub_rn(c.a1, own, acc);
            if (has_j) acc = mul_sub_rn(c.a2, vj, acc);
            if (has_i) acc = mul_sub_rn(c.a3, vi, acc);
            val = acc;
          } else {  // columns ascending: +i, +j, +k
            if (has_i) acc = mul_sub_rn(c.a1, vi, acc);
            if (has_j) acc = mul_sub_rn(c.a2, vj, acc);
            if (has_k) acc = mul_sub_rn(c.a3, own, acc);
            p_in[o] = sentinel_of<T>();  // the L walk's output, ready for the next application
            val = acc / c.piv;
          }
          st_relaxed(p_out + o, not_sentinel(val));
          own = val;
        }
        s_val[s & 1][lj][li] = val;
        compute_bar();
        if (threadIdx.x == 0) {
          __threadfence_block();
          s_done = s;
        }
      }
    }
  }
  // Hand the other sweep its ticket back (it does not run concurrently).
  if (blockIdx.x == 0 && threadIdx.x == 0) tickets[UP ? 1 : 2] = 0u;
}

// ------------------------------------------------------------------ cluster walk
// The same sweep with the tiles grouped into thread-block clusters of CX x CY
// tiles, one tile per CTA.  Inside a cluster a tile's boundary values are
// pushed by the producing threads (the last line along i, resp. j) straight
// into the consuming CTA's shared memory, so a hand-off costs one store to a
// neighbouring SM instead of a store to L2 followed by a poll of L2.
// Hand-offs between clusters keep the poll warp's path through global memory.
//
// Every boundary value reaches the consuming compute thread through a buffer
// of one slot per walk step (nsteps x 32 words of dynamic shared memory: the
// j-side values of lines (l, 0) in lanes 0-15, the i-side values of lines
// (0, l) in lanes 16-31).  Each slot is written once per launch and holds the
// sentinel until its value arrives -- the value is the flag, as in global
// memory -- so neither side waits for space and nothing is reset.  The poll
// warp fills the slots of the sides whose upstream tile is in another
// cluster; the producers in the cluster fill the others.
//
// The step inputs (y and the three bands, plus the pivot in the backward
// sweep: 256 consecutive words per array and step in walk order) come by bulk
// copy (cp.async.bulk, no multicast) into a ring of kInRing steps in shared
// memory, issued by a tenth warp as soon as the compute warps free a slot and
// completed on one mbarrier per slot; every compute thread waits on the slot
// (bounded) and reads its words.  Against the single-CTA walk's register
// prefetch this frees the compute warps' registers and load instructions; the
// issuing warp is separate from the poll warp, whose rounds through L2 would
// otherwise hold the copies back.
//
// Clusters take super-tiles from a ticket in row-major order, so a cluster
// waits only on clusters that run or are done; the CTAs of one cluster run
// together by construction.  Every wait is bounded as in the single-CTA walk.
// A cluster barrier at the start makes every buffer valid before a peer
// writes to it, and one at the end keeps each CTA's shared memory alive until
// no peer can write to it any more; before it the issuing warp waits
// (bounded) for its copies still in flight.

// Shared-memory words by 32-bit address: this CTA's (shared::cta) and a
// peer's (shared::cluster, from mapa).
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned peer_addr(unsigned a, int rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
// No "memory" clobber: the value is its own flag, so no other access needs
// ordering against the store, and a clobber would pin the walk's prefetched
// loads in place (register spills in the FP64 backward sweep).
__device__ __forceinline__ void st_peer(unsigned a, double v) {
  asm volatile("st.relaxed.cluster.shared::cluster.b64 [%0], %1;" ::"r"(a),
               "l"((unsigned long long)__double_as_longlong(v)));
}
__device__ __forceinline__ void st_peer(unsigned a, float v) {
  asm volatile("st.relaxed.cluster.shared::cluster.b32 [%0], %1;" ::"r"(a), "r"(__float_as_uint(v)));
}
__device__ __forceinline__ double ld_slot(unsigned a, double) {
  unsigned long long v;
  asm volatile("ld.volatile.shared.b64 %0, [%1];" : "=l"(v) : "r"(a));
  return __longlong_as_double((long long)v);
}
__device__ __forceinline__ float ld_slot(unsigned a, float) {
  unsigned v;
  asm volatile("ld.volatile.shared.b32 %0, [%1];" : "=r"(v) : "r"(a));
  return __uint_as_float(v);
}

// A slot of this CTA's buffer: its value, waited for (bounded) if it has not
// arrived yet.
template <class T>
__device__ __noinline__ T wait_slot(unsigned a, int* err) {
  const long long t0 = clock64();
  for (unsigned it = 1;; ++it) {
    const T v = ld_slot(a, T());
    if (!is_sentinel(v)) return v;
    if ((it & 255) == 0 && (clock64() - t0 > kWaitCycles || *(volatile int*)err)) {
      atomicOr(err, 1);
      return quiet_nan<T>();
    }
  }
}

template <class T>
__device__ __forceinline__ T take_slot(unsigned a, int* err) {
  const T v = ld_slot(a, T());
  return is_sentinel(v) ? wait_slot<T>(a, err) : v;
}

// Step inputs by bulk copy: each step's rows of the walk arrays (256
// consecutive words per array, in walk order) land in a ring of kInRing steps
// in shared memory, each slot completed on its own mbarrier.
constexpr int kInRing = 12;
template <bool UP>
constexpr int walk_in_fields() {
  return UP ? 5 : 4;  // y, three bands (and the pivot)
}

__device__ __forceinline__ void mbar_init(unsigned a, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned a, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned a, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(a), "r"(parity)
      : "memory");
  return done != 0;
}
// Global -> this CTA's shared memory, completing on the mbarrier (no
// multicast: the destination is this CTA's own window).
__device__ __forceinline__ void bulk_load(unsigned dst, const void* src, unsigned bytes, unsigned mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}
// The walk's output word, its own flag for the next tiles (no "memory"
// clobber: no other access needs ordering against it).
__device__ __forceinline__ void st_flag(double* p, double x) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"((unsigned long long)__double_as_longlong(x)));
}
__device__ __forceinline__ void st_flag(float* p, float x) {
  asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(__float_as_uint(x)));
}

// A word of the input ring (after the mbarrier wait, whose "memory" clobber
// keeps the load behind it).
__device__ __forceinline__ double ld_in(unsigned a, double) {
  unsigned long long v;
  asm("ld.shared.b64 %0, [%1];" : "=l"(v) : "r"(a) : "memory");
  return __longlong_as_double((long long)v);
}
__device__ __forceinline__ float ld_in(unsigned a, float) {
  unsigned v;
  asm("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
  return __uint_as_float(v);
}

// Waits for the phase of the given parity within the time bound only (the
// end-of-kernel drain of copies in flight); false if it gave up.
__device__ __noinline__ bool mbar_drain(unsigned a, unsigned parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(a, parity))
    if (clock64() - t0 > kWaitCycles) return false;
  return true;
}

// Waits (bounded) for the phase of the given parity; false if it gave up.
__device__ __noinline__ bool mbar_wait(unsigned a, unsigned parity, int* err) {
  const long long t0 = clock64();
  for (unsigned it = 1;; ++it) {
    if (mbar_try_wait(a, parity)) return true;
    if ((it & 15) == 0 && (clock64() - t0 > kWaitCycles || *(volatile int*)err)) {
      atomicOr(err, 1);
      return false;
    }
  }
}

// Dynamic shared memory of the cluster walk: the boundary buffer (nsteps x
// 32 words), the input ring (kInRing x fields x 256 words) and its mbarriers.
template <bool UP, class T>
constexpr size_t walk_cl_smem(int nsteps) {
  return ((size_t)nsteps * 2 * kTile + (size_t)kInRing * walk_in_fields<UP>() * kTileThreads) * sizeof(T) +
         kInRing * sizeof(unsigned long long);
}

template <bool UP, class T, int CX, int CY>
__global__ void __launch_bounds__(kTileThreads + 64, 1)
    k_walk_sweep_cl(Walk g, WalkArrays<T> b, T* in, T* wave, unsigned int* tickets, int* err) {
  constexpr int kPre = kWalkPrefetch;
  constexpr long long kStep = UP ? -kTileThreads : kTileThreads;
  constexpr int kLanes = 2 * kTile;
  constexpr int kF = walk_in_fields<UP>();
  constexpr unsigned kRowBytes = kTileThreads * sizeof(T);
  __shared__ T s_val[2][kTile][kTile + 1];
  __shared__ int s_tile;
  __shared__ volatile int s_done;  // last step the compute warps finished (the input ring's producer)
  extern __shared__ __align__(128) unsigned char walk_cl_raw[];
  T* s_bnd = reinterpret_cast<T*>(walk_cl_raw);                   // [step][lane]
  T* s_in = s_bnd + (size_t)g.nsteps * kLanes;                    // [slot][field][256]
  unsigned long long* s_mbar = reinterpret_cast<unsigned long long*>(s_in + (size_t)kInRing * kF * kTileThreads);
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int cx = rank % CX, cy = rank / CX;
  const int nsteps = g.nsteps;
  for (int q = threadIdx.x; q < nsteps * kLanes; q += blockDim.x) s_bnd[q] = sentinel_of<T>();
  if (threadIdx.x == 0) {
    s_done = -1;
    if (rank == 0) s_tile = (int)atomicAdd(tickets + (UP ? 2 : 1), 1u);
  }
  if (threadIdx.x == kTileThreads + 32) {
    for (int q = 0; q < kInRing; ++q) mbar_init(smem_addr(s_mbar + q), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  cl.sync();
  const int super = *cl.map_shared_rank(&s_tile, 0);
  const int nsx = (g.ntx + CX - 1) / CX;
  const int tx = (super % nsx) * CX + cx, ty = (super / nsx) * CY + cy;
  const unsigned mbar0 = smem_addr(s_mbar);

  if (tx < g.ntx && ty < g.nty) {
    const int tile = ty * g.ntx + tx;
    const bool copier = threadIdx.x >= kTileThreads + 32;
    const bool poller = !copier && threadIdx.x >= kTileThreads;
    const int lane = threadIdx.x & 31;
    const int li = poller ? (lane < kTile ? lane : 0) : threadIdx.x % kTile;
    const int lj = poller ? (lane < kTile ? 0 : lane - kTile) : (threadIdx.x / kTile) % kTile;
    const int ox = UP ? g.ntx * kTile - g.nx : 0;
    const int oy = UP ? g.nty * kTile - g.ny : 0;
    const int oz = UP ? nsteps - g.nz - 2 * (kTile - 1) : 0;
    auto phys = [&](long long w) { return UP ? g.nw - 1 - w : w; };
    const int ai = tx * kTile + li;
    const int aj = ty * kTile + lj;
    const bool active = ai >= ox && ai < ox + g.nx && aj >= oy && aj < oy + g.ny;
    const bool has_i = ai > ox, has_j = aj > oy;
    const bool bnd_i = li == 0 && has_i, bnd_j = lj == 0 && has_j;
    const int s_lo = active ? li + lj + oz : nsteps;
    const int s_hi = active ? s_lo + g.nz : nsteps;
    const long long tbase = (long long)tile * nsteps * kTileThreads;

    if (copier) {
      // Lane 0 issues each step's bulk copies once its slot is free.
      if (lane == 0) {
        const T* src[kF];
        src[0] = in;
        src[1] = UP ? b.Ui : b.Lk;
        src[2] = UP ? b.Uj : b.Lj;
        src[3] = UP ? b.Uk : b.Li;
        if constexpr (kF == 5) src[4] = b.P;
        // first word of step t's 256 in the arrays (the U walk reads its block reversed)
        auto row0 = [&](int t) { return UP ? g.nw - kTileThreads - tbase - (long long)t * kTileThreads
                                           : tbase + (long long)t * kTileThreads; };
        const unsigned in0 = smem_addr(s_in);
        int t_issue = 0;  // next step whose inputs are copied
        long long t_last = clock64();
        while (t_issue < nsteps) {
          const int lim = min(nsteps, s_done + kInRing + 1);
          if (t_issue < lim) {
            for (; t_issue < lim; ++t_issue) {
              const int q = t_issue % kInRing;
              const unsigned mb = mbar0 + q * 8;
              mbar_expect_tx(mb, kF * kRowBytes);
              const long long w0 = row0(t_issue);
#pragma unroll
              for (int f = 0; f < kF; ++f) bulk_load(in0 + (q * kF + f) * kRowBytes, src[f] + w0, kRowBytes, mb);
            }
            t_last = clock64();
          } else {
            __nanosleep(100);  // waiting for the compute warps to free a slot
            if (clock64() - t_last > kWaitCycles || *(volatile int*)err) {
              atomicOr(err, 1);
              break;
            }
          }
        }
        // Copies still in flight land before the CTA may leave (bounded by
        // time only: also after a failure, whatever the error flag says).
        for (int x = max(0, t_issue - kInRing); x < t_issue; ++x)
          if (!mbar_drain(mbar0 + (x % kInRing) * 8, (x / kInRing) & 1)) break;
      }
    } else if (poller) {
      // The sides whose upstream tile is in another cluster: global memory.
      const bool need = lane < kTile ? (bnd_j && cy == 0) : (bnd_i && cx == 0);
      if (__any_sync(0xffffffffu, need)) {
        const long long w_nb =
            lane < kTile ? phys(tbase - (long long)g.ntx * nsteps * kTileThreads + 15 * kTileThreads + 15 * kTile + li)
                         : phys(tbase - (long long)nsteps * kTileThreads + 15 * kTileThreads + lj * kTile + 15);
        const T* p_nb = wave + (need ? w_nb : 0);
        volatile T* slots = s_bnd + lane;
        int t = need ? s_lo : s_hi;  // next step this lane hands over
        long long t_last = clock64();
        bool failed = false;
        while (__any_sync(0xffffffffu, t < s_hi)) {
          T v[kPollDepth];
#pragma unroll
          for (int d = 0; d < kPollDepth; ++d) {
            const int st = t + d;
            v[d] = (st < s_hi && !failed) ? ld_relaxed(p_nb + (long long)st * kStep) : sentinel_of<T>();
          }
          int adv = 0;  // leading steps whose values arrived
#pragma unroll
          for (int d = 0; d < kPollDepth; ++d) {
            const int st = t + d;
            if (adv == d && st < s_hi && (failed || !is_sentinel(v[d]))) {
              slots[st * kLanes] = failed ? quiet_nan<T>() : v[d];
              ++adv;
            }
          }
          t += adv;
          if (__any_sync(0xffffffffu, adv > 0)) {
            t_last = clock64();
          } else {  // (warp-uniform) give up after the bound: quiet NaNs from here on
            const bool stop = __any_sync(0xffffffffu, clock64() - t_last > kWaitCycles || *(volatile int*)err != 0);
            if (stop && !failed) {
              if (lane == 0) atomicOr(err, 1);
              failed = true;
            }
          }
        }
      }
    } else {
      // In-cluster consumers of this tile's last lines.
      const bool feed_i = active && li == kTile - 1 && cx < CX - 1 && tx + 1 < g.ntx;
      const bool feed_j = active && lj == kTile - 1 && cy < CY - 1 && ty + 1 < g.nty;
      // 32-bit shared addresses of this thread's slots at step 0: own (read)
      // and the consumers' (written); a step is kLanes words further.
      const unsigned a_j = smem_addr(s_bnd + li), a_i = smem_addr(s_bnd + kTile + lj);
      const unsigned r_i = feed_i ? peer_addr(a_i, rank + 1) : 0u;  // consumer line (0, lj)
      const unsigned r_j = feed_j ? peer_addr(a_j, rank + CX) : 0u;  // consumer line (li, 0)
      constexpr unsigned kSlotStep = kLanes * sizeof(T);

      const long long w_own = phys(tbase + threadIdx.x);
      T* p_in = in + w_own;
      T* p_out = wave + w_own;
      // this thread's word of each input row in the ring (the U walk's rows are reversed)
      const unsigned a_in = smem_addr(s_in) + (UP ? kTileThreads - 1 - threadIdx.x : threadIdx.x) * sizeof(T);

      // Step s's inputs, once their slot's copies have landed.
      int f_slot = 0;
      unsigned f_par = 0;  // slot and phase parity of the next step to fetch
      auto fetch = [&](int s, PreW<T>& c) {
        (void)s;
        const int q = f_slot;
        const unsigned mb = mbar0 + q * 8, par = f_par;
        if (++f_slot == kInRing) {
          f_slot = 0;
          f_par ^= 1u;
        }
        if (!mbar_try_wait(mb, par)) mbar_wait(mb, par, err);
        const unsigned a = a_in + q * kF * kRowBytes;
        c.y = ld_in(a, T());
        c.a1 = ld_in(a + kRowBytes, T());
        c.a2 = ld_in(a + 2 * kRowBytes, T());
        c.a3 = ld_in(a + 3 * kRowBytes, T());
        if constexpr (kF == 5) c.piv = ld_in(a + 4 * kRowBytes, T());
      };

      T own = 0;
      PreW<T> nxt{0, 0, 0, 0, 0};
      fetch(0, nxt);
      for (int s0 = 0; s0 < nsteps; s0 += kPre) {
#pragma unroll
        for (int u = 0; u < kPre; ++u) {
          const int s = s0 + u;
          const long long o = (long long)s * kStep;
          const PreW<T> c = nxt;
          T val = 0;
          if (s >= s_lo && s < s_hi) {
            const T* prev = &s_val[(s + 1) & 1][0][0];
            T vi = 0, vj = 0;
            if (bnd_j) vj = take_slot<T>(a_j + s * kSlotStep, err);
            if (bnd_i) vi = take_slot<T>(a_i + s * kSlotStep, err);
            if (has_j && lj > 0) vj = prev[(lj - 1) * (kTile + 1) + li];
            if (has_i && li > 0) vi = prev[lj * (kTile + 1) + li - 1];
            const bool has_k = s > s_lo;
            T acc = c.y;
            if (!UP) {  // columns ascending: -k, -j, -i
              if (has_k) acc = mul_sub_rn(c.a1, own, acc);
              if (has_j) acc = mul_sub_rn(c.a2, vj, acc);
              if (has_i) acc = mul_sub_rn(c.a3, vi, acc);
              val = acc;
            } else {  // columns ascending: +i, +j, +k
              if (has_i) acc = mul_sub_rn(c.a1, vi, acc);
              if (has_j) acc = mul_sub_rn(c.a2, vj, acc);
              if (has_k) acc = mul_sub_rn(c.a3, own, acc);
              p_in[o] = sentinel_of<T>();
              val = acc / c.piv;
            }
            const T out = not_sentinel(val);
            st_flag(p_out + o, out);
            // the consumer's step: this one less the 15 lines between
            const int cs = s - (kTile - 1);
            if (feed_i) st_peer(r_i + cs * kSlotStep, out);
            if (feed_j) st_peer(r_j + cs * kSlotStep, out);
            own = val;
          }
          s_val[s & 1][lj][li] = val;
          // the next step's inputs, before the barrier (this step's slot is
          // handed back to the producer once s_done passes it)
          if (s + 1 < nsteps) fetch(s + 1, nxt);
          compute_bar();
          // (no fence: the only reader, the copy warp, reuses the slot of a
          // step whose words every thread read into registers before the
          // barrier; a fence here cost ~13 us per application at 192^3)
          if (threadIdx.x == 0) s_done = s;
        }
      }
    }
  }
  // Hand the other sweep its ticket back (it does not run concurrently).
  if (blockIdx.x == 0 && threadIdx.x == 0) tickets[UP ? 1 : 2] = 0u;
  cl.sync();
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

Walk walk_of(const Ilu0Data& d) {
  const Geom g = geom_of(d);
  Walk w;
  w.nx = g.nx;
  w.ny = g.ny;
  w.nz = g.nz;
  w.ntx = g.ntx;
  w.nty = g.nty;
  w.nsteps = (g.nz + 2 * (kTile - 1) + kWalkPrefetch - 1) / kWalkPrefetch * kWalkPrefetch;
  w.nxny = g.nxny;
  w.nw = (long long)g.ntx * g.nty * w.nsteps * kTileThreads;
  return w;
}

Bands bands_of(double* p, int n) {
  const size_t m = (size_t)n;
  return Bands{p, p + m, p + 2 * m, p + 3 * m, p + 4 * m, p + 5 * m, p + 6 * m, p + 7 * m};
}

// d_walk (and d_walk32): Lk Lj Li Ui Uj Uk P | y | L-walk output | U-walk output
enum { kWalkBands = 7, kWalkY = 7, kWalkL = 8, kWalkU = 9, kWalkArrays = 10 };

template <class T>
T* walk_array(T* base, const Ilu0Data& d, int a) {
  return base + (size_t)a * (size_t)d.walk_n;
}

template <class T>
WalkArrays<T> walk_bands(T* base, const Ilu0Data& d) {
  return WalkArrays<T>{walk_array(base, d, 0), walk_array(base, d, 1), walk_array(base, d, 2),
                       walk_array(base, d, 3), walk_array(base, d, 4), walk_array(base, d, 5),
                       walk_array(base, d, 6)};
}

int wave_grid(ab2_context* ctx, int ntiles) { return std::max(1, std::min(ntiles, ctx->num_sms * 2)); }

// The cluster walk: 2 x 2 tiles per cluster.  Measured at 192^3 (one ILU(0)
// application, B200): 2 x 2 0.581 ms, 2 x 4 0.588, 4 x 2 0.646, 4 x 4 0.642,
// against 0.609 for the single-CTA walk.  With one CTA an SM (the walk's
// shared memory), a GPC holds fewer large clusters than its SMs allow CTAs,
// and the remaining clusters start late.
constexpr int kClX = 2, kClY = 2;
// Its buffers live in shared memory: up to this many bytes (nz up to ~350 in
// FP64); longer walks take the single-CTA walk.
constexpr size_t kWalkClSmemMax = 216 * 1024;

template <bool UP, class T>
cudaLaunchConfig_t walk_cl_config(cudaStream_t stream, const Walk& w, cudaLaunchAttribute* attr) {
  const int nsx = (w.ntx + kClX - 1) / kClX, nsy = (w.nty + kClY - 1) / kClY;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kClX * kClY;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(nsx * nsy * kClX * kClY));
  cfg.blockDim = dim3(kTileThreads + 64);
  cfg.dynamicSmemBytes = walk_cl_smem<UP, T>(w.nsteps);
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

// Whether the device runs the cluster walk at all: both sweeps, at the
// shared-memory cap, asked once per device and word size (the kernels'
// shared-memory limit is raised to the cap on the way, so that no set-up can
// lower it under another factor's walk).
template <class T>
bool walk_cl_device_ok(ab2_context* ctx) {
  static std::atomic<int> ok[64];  // 0: not asked, 1: yes, 2: no
  const int dev = ctx->device;
  if (dev >= 0 && dev < 64 && ok[dev].load() != 0) return ok[dev].load() == 1;
  bool fits = true;
  Walk w{};
  w.ntx = w.nty = kClX * kClY;
  cudaLaunchAttribute attr[1];
  for (int up = 0; up < 2 && fits; ++up) {
    const void* k = up ? (const void*)k_walk_sweep_cl<true, T, kClX, kClY> : (const void*)k_walk_sweep_cl<false, T, kClX, kClY>;
    AB2_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWalkClSmemMax));
    cudaLaunchConfig_t cfg = up ? walk_cl_config<true, T>(nullptr, w, attr) : walk_cl_config<false, T>(nullptr, w, attr);
    cfg.dynamicSmemBytes = kWalkClSmemMax;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess || n < 1) {
      (void)cudaGetLastError();
      fits = false;
    }
  }
  if (dev >= 0 && dev < 64) ok[dev].store(fits ? 1 : 2);
  return fits;
}

// Whether this factor's walk can take the cluster walk (both word sizes: the
// mixed-precision solvers run the FP32 copy on the same schedule).
bool walk_cl_possible(ab2_context* ctx, const Walk& w) {
  const bool size_ok = walk_cl_smem<true, double>(w.nsteps) <= kWalkClSmemMax &&
                       walk_cl_smem<false, double>(w.nsteps) <= kWalkClSmemMax;
  return size_ok && walk_cl_device_ok<double>(ctx) && walk_cl_device_ok<float>(ctx);
}

template <bool UP, class T>
void launch_walk_cl(ab2_context* ctx, const Walk& w, const WalkArrays<T>& b, T* in, T* wave, unsigned int* tickets,
                    int* err) {
  cudaLaunchAttribute attr[1];
  const cudaLaunchConfig_t cfg = walk_cl_config<UP, T>(ctx->stream, w, attr);
  AB2_CUDA(cudaLaunchKernelEx(&cfg, k_walk_sweep_cl<UP, T, kClX, kClY>, w, b, in, wave, tickets, err));
}

// One sweep (UP: the backward one) on the factor's walk.
template <bool UP, class T>
void walk_sweep(ab2_context* ctx, const Ilu0Data& d, const Walk& w, const WalkArrays<T>& b, T* in, T* wave) {
  if (d.walk_cluster)
    launch_walk_cl<UP, T>(ctx, w, b, in, wave, d.d_tile_tickets, d.d_err);
  else
    k_walk_sweep<UP, T><<<wave_grid(ctx, w.ntx * w.nty), kTileThreads + 32, 0, ctx->stream>>>(
        w, b, in, wave, d.d_tile_tickets, d.d_err);
  check_launch(ctx, UP ? "walk_usweep" : "walk_lsweep");
}

int bulk_grid(ab2_context* ctx, long long n) {
  return (int)std::max(1LL, std::min((n + kThreads - 1) / kThreads, (long long)ctx->num_sms * 16));
}

}  // namespace

bool ilu_stencil_setup(ab2_context* ctx, const ab2_matrix* A, Ilu0Data& d, bool factored, int schedule) {
  const int n = A->n;
  if (n == 0) return false;
  // The 7-point geometry: kept by the matrix (AB2_FMT_STENCIL) or checked here.
  int nx = A->st_nx, ny = A->st_ny, nz = A->st_nz;
  if (nx == 0 && !stencil_geometry(ctx, A, &nx, &ny, &nz)) return false;
  d.st_nx = nx;
  d.st_ny = ny;
  d.st_nz = nz;
  const Geom g = geom_of(d);

  // Factorisation on natural-order bands.
  d.d_bands = dev_alloc<double>(ctx, (size_t)n * 8);
  d.d_tile_tickets = dev_alloc<unsigned int>(ctx, 3);
  AB2_CUDA(cudaMemsetAsync(d.d_tile_tickets, 0, 3 * sizeof(unsigned int), ctx->stream));
  const Bands b = bands_of(d.d_bands, n);
  if (factored) {
    // d_lu holds the factor: its diagonal is the pivot band.
    k_stencil_extract<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, g, A->d_rp, d.d_lu, b);
    check_launch(ctx, "stencil_extract");
    AB2_CUDA(cudaMemcpyAsync(b.P, b.D, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
  } else {
    k_stencil_extract<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, g, A->d_rp, A->d_v, b);
    check_launch(ctx, "stencil_extract");
    k_fill_bits<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, kSentinel, b.P);
    check_launch(ctx, "stencil_fill");
    k_stencil_factor<<<wave_grid(ctx, g.ntx * g.nty), kTileThreads, 0, ctx->stream>>>(g, b, d.d_tile_tickets,
                                                                                         d.d_err);
    check_launch(ctx, "stencil_factor");
    k_stencil_pack<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, g, A->d_rp, b, d.d_lu);
    check_launch(ctx, "stencil_pack");
  }

  // The sweeps' arrays in walk order.
  const Walk w = walk_of(d);
  d.walk_n = w.nw;
  d.d_walk = dev_alloc<double>(ctx, (size_t)kWalkArrays * (size_t)w.nw);
  const double* nat[kWalkBands] = {b.Lk, b.Lj, b.Li, b.Ui, b.Uj, b.Uk, b.P};
  for (int a = 0; a < kWalkBands; ++a) {
    k_walk_gather<<<bulk_grid(ctx, w.nw), kThreads, 0, ctx->stream>>>(w, nat[a], walk_array(d.d_walk, d, a));
    check_launch(ctx, "walk_gather");
  }
  AB2_CUDA(cudaMemsetAsync(walk_array(d.d_walk, d, kWalkY), 0, sizeof(double) * (size_t)w.nw, ctx->stream));
  k_fill_bits<<<bulk_grid(ctx, 2 * w.nw), kThreads, 0, ctx->stream>>>(2 * w.nw, kSentinel,
                                                                      walk_array(d.d_walk, d, kWalkL));
  check_launch(ctx, "walk_fill");
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  dev_free(ctx, d.d_bands);
  d.d_bands = nullptr;
  set_transpose_smem<double>();
  d.walk_cluster = schedule != AB2_ILU_STENCIL && walk_cl_possible(ctx, w);
  require(schedule != AB2_ILU_STENCIL_CLUSTER || d.walk_cluster,
          "ILU0 cluster schedule requested but its buffers do not fit shared memory (too many planes along z)");
  d.stencil = true;
  d.levels_l = d.levels_u = (int)(nx + ny + nz - 2);
  return true;
}

namespace {

template <class T>
void walk_apply(ab2_context* ctx, const Ilu0Data& d, T* base, const T* y, T* z) {
  const Walk w = walk_of(d);
  const WalkArrays<T> b = walk_bands(base, d);
  const int tiles = w.ntx * w.nty;
  T* yw = walk_array(base, d, kWalkY);
  T* lw = walk_array(base, d, kWalkL);
  T* uw = walk_array(base, d, kWalkU);
  // FP64: shared-memory transposes; FP32 (half the bytes): element-wise
  // kernels, which move them faster than the latency-bound transposes (both
  // measured back to back on one GPU).
  constexpr bool kTranspose = std::is_same<T, double>::value;
  const int tr_grid = tiles * ((w.nz + kTrPlanes - 1) / kTrPlanes);
  if (kTranspose) k_walk_gather_t<T><<<tr_grid, kTileThreads, tr_smem<T>(), ctx->stream>>>(w, y, yw);
  else k_walk_gather<<<bulk_grid(ctx, w.nw), kThreads, 0, ctx->stream>>>(w, y, yw);
  check_launch(ctx, "walk_gather");
  walk_sweep<false, T>(ctx, d, w, b, yw, lw);
  walk_sweep<true, T>(ctx, d, w, b, lw, uw);
  if (kTranspose) k_walk_scatter_t<T><<<tr_grid, kTileThreads, tr_smem<T>(), ctx->stream>>>(w, uw, z);
  else k_walk_scatter<<<bulk_grid(ctx, w.nw), kThreads, 0, ctx->stream>>>(w, uw, z);
  check_launch(ctx, "walk_scatter");
}

}  // namespace

// y -> walk order -> L walk -> U walk (reversed index) -> z.
void ilu_stencil_apply(ab2_context* ctx, const ab2_matrix* A, const Ilu0Data& d, const double* y, double* z) {
  (void)A;
  walk_apply(ctx, d, d.d_walk, y, z);
}

// FP32 walk arrays: the FP64 factor's bands rounded to float.
void ilu_stencil_enable_f32(ab2_context* ctx, Ilu0Data& d) {
  if (d.d_walk32) return;
  const Walk w = walk_of(d);
  d.d_walk32 = dev_alloc<float>(ctx, (size_t)kWalkArrays * (size_t)w.nw);
  op_to_f32(ctx, kWalkBands * w.nw, d.d_walk, d.d_walk32);
  AB2_CUDA(cudaMemsetAsync(walk_array(d.d_walk32, d, kWalkY), 0, sizeof(float) * (size_t)w.nw, ctx->stream));
  k_fill_bits32<<<bulk_grid(ctx, 2 * w.nw), kThreads, 0, ctx->stream>>>(2 * w.nw, kSentinel32,
                                                                        walk_array(d.d_walk32, d, kWalkL));
  check_launch(ctx, "walk_fill32");
}

void ilu_stencil_apply_f32(ab2_context* ctx, const Ilu0Data& d, const float* y, float* z) {
  require(d.d_walk32 != nullptr, "FP32 ILU0 arrays not built");
  walk_apply(ctx, d, d.d_walk32, y, z);
}

// After a failed application: the propagation arrays back to the sentinel
// (the tickets are reset by pc_reset).
void ilu_stencil_reset(ab2_context* ctx, const Ilu0Data& d) {
  if (d.d_walk) {
    k_fill_bits<<<bulk_grid(ctx, 2 * d.walk_n), kThreads, 0, ctx->stream>>>(2 * d.walk_n, kSentinel,
                                                                            walk_array(d.d_walk, d, kWalkL));
    check_launch(ctx, "walk_fill");
  }
  if (d.d_walk32) {
    k_fill_bits32<<<bulk_grid(ctx, 2 * d.walk_n), kThreads, 0, ctx->stream>>>(2 * d.walk_n, kSentinel32,
                                                                              walk_array(d.d_walk32, d, kWalkL));
    check_launch(ctx, "walk_fill32");
  }
}

}  // namespace ab2
