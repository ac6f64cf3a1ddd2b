// problems.cpp -- seeded synthetic systems (see include/ab2_problems.h).
// Host-only input preparation; nothing here is on the solve path.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "ab2.h"
#include "ab2_problems.h"

namespace {

inline uint64_t mix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
inline uint64_t key(uint64_t seed, uint64_t s) { return mix(seed + 0x632BE59BD9B4E019ull * (s + 1)); }
inline double u01(uint64_t u) { return (double)(u >> 11) * (1.0 / 9007199254740992.0); }
inline double normal(uint64_t k, uint64_t i) {
  const double a = 1.0 - u01(mix(k + mix(2 * i)));
  const double b = u01(mix(k + mix(2 * i + 1)));
  return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
}

template <class F>
void parallel_for(long long n, F&& f) {
  unsigned t = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  if (n < 65536) t = 1;
  std::vector<std::thread> pool;
  const long long chunk = (n + t - 1) / t;
  for (unsigned w = 0; w < t; ++w) {
    const long long a = w * chunk, b = std::min(n, a + chunk);
    if (a >= b) break;
    pool.emplace_back([&f, a, b] {
      for (long long i = a; i < b; ++i) f(i);
    });
  }
  for (auto& th : pool) th.join();
}

struct Builder {
  int nx, ny, nz, n;
  std::vector<int> rp;
  std::vector<int> ci;
  std::vector<double> v;
  explicit Builder(int nx_, int ny_, int nz_) : nx(nx_), ny(ny_), nz(nz_), n(nx_ * ny_ * nz_) {}
  int idx(int i, int j, int k) const { return i + nx * (j + ny * k); }
  // Row entries are generated in ascending column order by the callers.
  void layout(bool with_z) {
    rp.assign((size_t)n + 1, 0);
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          int c = 1;
          c += (i > 0) + (i < nx - 1) + (j > 0) + (j < ny - 1);
          if (with_z) c += (k > 0) + (k < nz - 1);
          rp[idx(i, j, k) + 1] = c;
        }
    for (int r = 0; r < n; ++r) rp[r + 1] += rp[r];
    ci.assign((size_t)rp[n], 0);
    v.assign((size_t)rp[n], 0.0);
  }
};

ab2_problem* finish(Builder& B, uint64_t seed, std::vector<double>* logk) {
  ab2_problem* p = new ab2_problem();
  std::memset(p, 0, sizeof(*p));
  p->n = B.n;
  p->nnz = B.rp[B.n];
  p->nx = B.nx;
  p->ny = B.ny;
  p->nz = B.nz;
  p->row_ptr = new int[(size_t)B.n + 1];
  p->cols = new int[(size_t)p->nnz];
  p->vals = new double[(size_t)p->nnz];
  p->x_true = new double[(size_t)B.n];
  p->b = new double[(size_t)B.n];
  std::memcpy(p->row_ptr, B.rp.data(), sizeof(int) * ((size_t)B.n + 1));
  std::memcpy(p->cols, B.ci.data(), sizeof(int) * (size_t)p->nnz);
  std::memcpy(p->vals, B.v.data(), sizeof(double) * (size_t)p->nnz);
  const uint64_t k0 = key(seed, 0);
  for (int i = 0; i < B.n; ++i) p->x_true[i] = 2.0 * u01(mix(k0 + mix((uint64_t)i))) - 1.0;
  int* rp = p->row_ptr;
  int* ci = p->cols;
  double* v = p->vals;
  double* xt = p->x_true;
  double* b = p->b;
  parallel_for(B.n, [&](long long r) {
    double acc = 0.0;
    for (int k = rp[r]; k < rp[r + 1]; ++k) acc = acc + v[k] * xt[ci[k]];  // product and sum rounded apart (-ffp-contract=off)
    b[r] = acc;
  });
  if (logk) {
    p->log10_k = new double[(size_t)B.n];
    std::memcpy(p->log10_k, logk->data(), sizeof(double) * (size_t)B.n);
  }
  return p;
}

// Separable Gaussian smoothing along one axis with reflective ends.
void smooth_axis(std::vector<double>& g, int nx, int ny, int nz, int axis, double sigma) {
  const int R = (int)std::ceil(4.0 * sigma);
  std::vector<double> w(2 * R + 1);
  double sw = 0;
  for (int t = -R; t <= R; ++t) sw += (w[t + R] = std::exp(-(double)t * t / (2 * sigma * sigma)));
  for (double& e : w) e /= sw;
  const int len = axis == 0 ? nx : axis == 1 ? ny : nz;
  const long long lines = (long long)nx * ny * nz / len;
  std::vector<double> out(g.size());
  auto reflect = [len](int j) {
    while (j < 0 || j >= len) j = j < 0 ? -j - 1 : 2 * len - j - 1;
    return j;
  };
  parallel_for(lines, [&](long long L) {
    // Line L: fixed coordinates on the two other axes.
    int i0 = 0, j0 = 0, k0 = 0;
    if (axis == 0) { j0 = (int)(L % ny); k0 = (int)(L / ny); }
    else if (axis == 1) { i0 = (int)(L % nx); k0 = (int)(L / nx); }
    else { i0 = (int)(L % nx); j0 = (int)(L / nx); }
    const long long stride = axis == 0 ? 1 : axis == 1 ? nx : (long long)nx * ny;
    const long long base = i0 + (long long)nx * (j0 + (long long)ny * k0);
    for (int t = 0; t < len; ++t) {
      double acc = 0;
      for (int d = -R; d <= R; ++d) acc += w[d + R] * g[base + stride * reflect(t + d)];
      out[base + stride * t] = acc;
    }
  });
  g.swap(out);
}

std::vector<double> gaussian_field(int nx, int ny, int nz, double sigma_out, double smooth_len, uint64_t seed) {
  const long long n = (long long)nx * ny * nz;
  std::vector<double> g((size_t)n);
  const uint64_t k1 = key(seed, 1);
  parallel_for(n, [&](long long i) { g[i] = normal(k1, (uint64_t)i); });
  if (smooth_len > 0) {
    if (nx > 1) smooth_axis(g, nx, ny, nz, 0, smooth_len);
    if (ny > 1) smooth_axis(g, nx, ny, nz, 1, smooth_len);
    if (nz > 1) smooth_axis(g, nx, ny, nz, 2, smooth_len);
  }
  double mean = 0;
  for (double e : g) mean += e;
  mean /= (double)n;
  double var = 0;
  for (double e : g) var += (e - mean) * (e - mean);
  var /= (double)n;
  const double s = var > 0 ? sigma_out / std::sqrt(var) : 0.0;
  for (double& e : g) e = (e - mean) * s;
  return g;
}

// Face transmissibilities t(P,Q) and Dirichlet terms assembled row by row.
template <class Face, class Bnd>
void assemble(Builder& B, bool with_z, Face&& face, Bnd&& bnd) {
  B.layout(with_z);
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  parallel_for(B.n, [&](long long r) {
    const int i = (int)(r % nx), j = (int)((r / nx) % ny), k = (int)(r / ((long long)nx * ny));
    int at = B.rp[r];
    double diag = 0;
    int dpos = -1;
    auto put = [&](int c, double a) {
      B.ci[at] = c;
      B.v[at] = a;
      ++at;
    };
    // Ascending columns: -z, -y, -x, self, +x, +y, +z.
    const int nb[6][3] = {{0, 0, -1}, {0, -1, 0}, {-1, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int f = 0; f < 6; ++f) {
      if (!with_z && nb[f][2] != 0) continue;
      if (f == 3) {
        dpos = at;
        put((int)r, 0.0);
      }
      const int ii = i + nb[f][0], jj = j + nb[f][1], kk = k + nb[f][2];
      const bool inside = ii >= 0 && ii < nx && jj >= 0 && jj < ny && kk >= 0 && kk < nz;
      double off = 0, dg = 0;
      if (inside) {
        face((int)r, B.idx(ii, jj, kk), i, j, k, f, off, dg);
        put(B.idx(ii, jj, kk), off);
      } else {
        bnd((int)r, i, j, k, f, dg);
      }
      diag += dg;
    }
    B.v[dpos] = diag;
  });
}

}  // namespace

extern "C" {

uint64_t ab2_rng_u64(uint64_t seed, uint64_t stream, uint64_t index) { return mix(key(seed, stream) + mix(index)); }
double ab2_rng_uniform(uint64_t seed, uint64_t stream, uint64_t index) {
  return 2.0 * u01(ab2_rng_u64(seed, stream, index)) - 1.0;
}

int ab2_problem_poisson(int nx, int ny, int nz, uint64_t seed, ab2_problem** out) {
  if (!out || nx < 1 || ny < 1 || nz < 1) return AB2_ERR_BAD_ARG;
  try {
    Builder B(nx, ny, nz);
    const bool with_z = nz > 1;
    const double d = with_z ? 6.0 : 4.0;
    assemble(
        B, with_z, [](int, int, int, int, int, int, double& off, double& dg) { off = -1.0; dg = 0.0; },
        [](int, int, int, int, int, double& dg) { dg = 0.0; });
    for (int r = 0; r < B.n; ++r)
      for (int k = B.rp[r]; k < B.rp[r + 1]; ++k)
        if (B.ci[k] == r) B.v[k] = d;
    *out = finish(B, seed, nullptr);
  } catch (const std::bad_alloc&) {
    return AB2_ERR_OOM;
  }
  return AB2_OK;
}

int ab2_problem_diffusion(int nx, int ny, int nz, double sigma_log10k, double smooth_len, uint64_t seed,
                          ab2_problem** out) {
  if (!out || nx < 1 || ny < 1 || nz < 1 || smooth_len < 0) return AB2_ERR_BAD_ARG;
  try {
    Builder B(nx, ny, nz);
    std::vector<double> g = gaussian_field(nx, ny, nz, sigma_log10k, smooth_len, seed);
    std::vector<double> kc(g.size());
    for (size_t i = 0; i < g.size(); ++i) kc[i] = std::pow(10.0, g[i]);
    assemble(
        B, nz > 1,
        [&](int p, int q, int, int, int, int, double& off, double& dg) {
          const double t = 2.0 * kc[p] * kc[q] / (kc[p] + kc[q]);
          off = -t;
          dg = t;
        },
        [&](int p, int, int, int, int, double& dg) { dg = 2.0 * kc[p]; });
    *out = finish(B, seed, &g);
  } catch (const std::bad_alloc&) {
    return AB2_ERR_OOM;
  }
  return AB2_OK;
}

int ab2_problem_convdiff(int nx, int ny, int nz, double peclet, int modes, uint64_t seed, ab2_problem** out) {
  if (!out || nx < 1 || ny < 1 || nz < 2 || modes < 1) return AB2_ERR_BAD_ARG;
  try {
    // Vector potential psi = sum_m a_m sin(2 pi k_m . X / L + phi_m), per component.
    const uint64_t k2 = key(seed, 2);
    std::vector<double> kv(modes * 3), amp(modes * 3), ph(modes * 3);
    uint64_t draw = 0;
    auto next = [&]() { return u01(mix(k2 + mix(draw++))); };
    for (int m = 0; m < modes; ++m) {
      double nk = 0;
      do {
        for (int c = 0; c < 3; ++c) kv[m * 3 + c] = (double)((int)(next() * 7.0) - 3);
        nk = std::sqrt(kv[m * 3] * kv[m * 3] + kv[m * 3 + 1] * kv[m * 3 + 1] + kv[m * 3 + 2] * kv[m * 3 + 2]);
      } while (nk == 0);
      for (int c = 0; c < 3; ++c) {
        const double a = 1.0 - next(), b = next();
        amp[m * 3 + c] = std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b) / nk;
        ph[m * 3 + c] = 6.283185307179586 * next();
      }
    }
    const double L = (double)std::max(nx, std::max(ny, nz));
    auto psi = [&](int c, double X, double Y, double Z) {
      double s = 0;
      for (int m = 0; m < modes; ++m)
        s += amp[m * 3 + c] *
             std::sin(6.283185307179586 * (kv[m * 3] * X + kv[m * 3 + 1] * Y + kv[m * 3 + 2] * Z) / L + ph[m * 3 + c]);
      return s;
    };
    // Edge integrals by the midpoint rule, on nodes (nx+1)(ny+1)(nz+1).
    const int NX = nx + 1, NY = ny + 1, NZ = nz + 1;
    auto nid = [&](int i, int j, int k) { return (size_t)i + (size_t)NX * ((size_t)j + (size_t)NY * k); };
    std::vector<double> Ex((size_t)NX * NY * NZ, 0.0), Ey(Ex.size(), 0.0), Ez(Ex.size(), 0.0);
    parallel_for((long long)NZ, [&](long long kk) {
      const int k = (int)kk;
      for (int j = 0; j < NY; ++j)
        for (int i = 0; i < NX; ++i) {
          if (i < nx) Ex[nid(i, j, k)] = psi(0, i + 0.5, j, k);
          if (j < ny) Ey[nid(i, j, k)] = psi(1, i, j + 0.5, k);
          if (k < nz) Ez[nid(i, j, k)] = psi(2, i, j, k + 0.5);
        }
    });
    // Face fluxes = circulation of psi around each face (Stokes), so every
    // cell's net outflow cancels edge by edge.
    auto Fx = [&](int i, int j, int k) {
      return Ey[nid(i, j, k)] + Ez[nid(i, j + 1, k)] - Ey[nid(i, j, k + 1)] - Ez[nid(i, j, k)];
    };
    auto Fy = [&](int i, int j, int k) {
      return Ez[nid(i, j, k)] + Ex[nid(i, j, k + 1)] - Ez[nid(i + 1, j, k)] - Ex[nid(i, j, k)];
    };
    auto Fz = [&](int i, int j, int k) {
      return Ex[nid(i, j, k)] + Ey[nid(i + 1, j, k)] - Ex[nid(i, j + 1, k)] - Ey[nid(i, j, k)];
    };
    double fmax = 0;
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i <= nx; ++i) fmax = std::max(fmax, std::fabs(Fx(i, j, k)));
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j <= ny; ++j)
        for (int i = 0; i < nx; ++i) fmax = std::max(fmax, std::fabs(Fy(i, j, k)));
    for (int k = 0; k <= nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) fmax = std::max(fmax, std::fabs(Fz(i, j, k)));
    const double scale = fmax > 0 ? peclet / fmax : 0.0;
    // Outward flux of cell (i,j,k) through face f (ordering -z,-y,-x,+x,+y,+z).
    auto outflux = [&](int i, int j, int k, int f) {
      switch (f) {
        case 0: return -Fz(i, j, k) * scale;
        case 1: return -Fy(i, j, k) * scale;
        case 2: return -Fx(i, j, k) * scale;
        case 3: return Fx(i + 1, j, k) * scale;
        case 4: return Fy(i, j + 1, k) * scale;
        default: return Fz(i, j, k + 1) * scale;
      }
    };
    Builder B(nx, ny, nz);
    assemble(
        B, true,
        [&](int, int, int i, int j, int k, int f, double& off, double& dg) {
          const double F = outflux(i, j, k, f);
          off = -1.0 + std::min(F, 0.0);
          dg = 1.0 + std::max(F, 0.0);
        },
        [&](int, int i, int j, int k, int f, double& dg) { dg = 2.0 + std::max(outflux(i, j, k, f), 0.0); });
    *out = finish(B, seed, nullptr);
  } catch (const std::bad_alloc&) {
    return AB2_ERR_OOM;
  }
  return AB2_OK;
}

int ab2_problem_destroy(ab2_problem* p) {
  if (!p) return AB2_ERR_BAD_ARG;
  delete[] p->row_ptr;
  delete[] p->cols;
  delete[] p->vals;
  delete[] p->x_true;
  delete[] p->b;
  delete[] p->log10_k;
  delete p;
  return AB2_OK;
}

}  // extern "C"
