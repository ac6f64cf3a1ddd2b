/*
 * ab2_problems.h -- seeded synthetic linear systems (host code in libab2).
 *
 * Alien's own driver assembles its matrix with MatrixProfiler +
 * ProfiledMatrixBuilder (examples/test_krylov.cpp:291-408, columns kept sorted
 * by MatrixProfilerT.h:95-113).  These generators produce the same kind of
 * SimpleCSR input -- n, row_ptr, sorted int32 columns, FP64 values -- for the
 * benchmark shapes, directly on the host, with a counter-based RNG so that any
 * cell's random numbers can be regenerated independently:
 *
 *   mix(z)        = splitmix64 finaliser
 *   key(seed, s)  = mix(seed + 0x632BE59BD9B4E019 * (s + 1))
 *   u64(seed,s,i) = mix(key(seed, s) + mix(i))
 *   uniform01     = (u64 >> 11) * 2^-53
 *   x_true[i]     = 2 * uniform01(seed, 0, i) - 1
 *   normal        = Box-Muller on draws 2i, 2i+1 of stream 1
 *
 * Cells are numbered i + nx*(j + ny*k); b = A x_true with the row-sequential
 * fma sum of the reference SpMV.
 */
#ifndef AB2_PROBLEMS_H
#define AB2_PROBLEMS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int n;
  long long nnz;
  int nx, ny, nz;
  int* row_ptr;    /* n+1 */
  int* cols;       /* nnz, ascending inside each row */
  double* vals;    /* nnz */
  double* x_true;  /* n */
  double* b;       /* n, = A x_true */
  double* log10_k; /* n cell coefficients (log10), NULL for constant ones */
} ab2_problem;

/* 7-point constant-coefficient Poisson, zero Dirichlet eliminated:
 * a_ii = 6, a_ij = -1 for neighbours inside the grid (nz == 1: 5-point, a_ii = 4). */
int ab2_problem_poisson(int nx, int ny, int nz, uint64_t seed, ab2_problem** out);

/* Heterogeneous diffusion, cell-centred finite volumes: log10 k = sigma *
 * (white noise smoothed by a separable Gaussian of std `smooth_len` cells,
 * truncated at 4 std, reflective ends, renormalised to mean 0 / std 1);
 * face transmissibility = harmonic mean 2 k_i k_j / (k_i + k_j); a Dirichlet
 * face adds 2 k to the diagonal.  nz == 1 gives the 2-D 5-point system. */
int ab2_problem_diffusion(int nx, int ny, int nz, double sigma_log10k, double smooth_len, uint64_t seed,
                          ab2_problem** out);

/* Convection-diffusion: unit diffusion (as above with k = 1) plus first-order
 * upwind convection by a discretely divergence-free velocity, the discrete
 * curl of a vector potential made of `modes` random Fourier modes, scaled so
 * that the largest face Peclet number |u| h / D equals `peclet`. */
int ab2_problem_convdiff(int nx, int ny, int nz, double peclet, int modes, uint64_t seed, ab2_problem** out);

int ab2_problem_destroy(ab2_problem* p);

/* MatrixMarket files (the reference reads them with
 * src/movesemantic/alien/move/impl/MatrixMarketReader.cc:58-157 and
 * benchmarks them through benchmark/src/alien/benchmark/MatrixMarketProblem.cpp).
 * Matrix: "%%MatrixMarket matrix coordinate real <symmetry>" -- any symmetry
 * but "general" is mirrored with the same value, duplicates are summed in
 * file order, columns come out ascending per row; square only.  rhs_path: an
 * "array real" file with one value per line, or NULL for b = 1.  x_true is
 * NULL and nx = n, ny = nz = 1.  Errors return AB2_ERR_BAD_ARG with the text
 * in ab2_matrix_market_error(). */
int ab2_problem_read_matrix_market(const char* matrix_path, const char* rhs_path, ab2_problem** out);
/* "coordinate real general" with 17 significant digits (exact round trip), and
 * b as "array real" (rhs_path may be NULL). */
int ab2_problem_write_matrix_market(const ab2_problem* p, const char* matrix_path, const char* rhs_path);
const char* ab2_matrix_market_error(void);

/* The generator's random streams, for tests. */
uint64_t ab2_rng_u64(uint64_t seed, uint64_t stream, uint64_t index);
double ab2_rng_uniform(uint64_t seed, uint64_t stream, uint64_t index); /* [-1, 1) */

#ifdef __cplusplus
}
#endif

#endif /* AB2_PROBLEMS_H */
