/*
 * ab2.h -- C ABI of libab2, the B200 (sm_100a) internal linear algebra and
 * Krylov solver backend for Alien.
 *
 * Every entry point takes plain pointers and sizes, returns AB2_OK (0) or a
 * negative AB2_ERR_* code, and never lets a C++ exception cross the boundary.
 * ab2_last_error_message() gives the text of the last failure on a context.
 *
 * Threading: a context owns one CUDA stream and is not thread safe; use one
 * context per host thread.  Every call is ordered on the context's stream.
 * Only calls that hand a value back to host memory synchronise
 * (ab2_vector_download, ab2_dot, ab2_norm*, ab2_scalar_get, ab2_solver_solve).
 *
 * Reference interfaces replaced (paths are inside arcaneframework/alien):
 *   algebra ops  src/core/alien/kernels/simple_csr/algebra/SimpleCSRInternalLinearAlgebra.h:55-173
 *                src/core/alien/kernels/sycl/algebra/SYCLInternalLinearAlgebra.h:46-141
 *   matrix/vec   src/core/alien/kernels/sycl/converters/SimpleCSRtoSYCLMatrixConverter.cc:74-104,
 *                SimpleCSRtoSYCLVectorConverter.cc, SYCLtoSimpleCSRVectorConverter.cc:60-70
 *   solvers      src/core/alien/expression/krylov/{CG.h:59-150, BiCGStab.h:152-300, Iteration.h:34-136}
 *   precond.     src/core/alien/expression/krylov/{DiagPreconditioner.h:49-68,
 *                ILU0Preconditioner.h:71-323, ChebyshevPreconditioner.h:73-202,392-444}
 *   status       src/core/alien/expression/solver/ILinearSolver.h:63-83 (SolverStatus)
 */
#ifndef AB2_H
#define AB2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ codes */
#define AB2_OK 0
#define AB2_ERR_CUDA (-1)          /* a CUDA runtime call failed */
#define AB2_ERR_OOM (-2)           /* device or pinned allocation failed */
#define AB2_ERR_BREAKDOWN (-3)     /* Krylov breakdown (NullValueException in CG.h/BiCGStab.h) */
#define AB2_ERR_NOT_CONVERGED (-4) /* reserved: solves report non-convergence in ab2_status */
#define AB2_ERR_TIMEOUT (-5)       /* a bounded device-side wait gave up */
#define AB2_ERR_BAD_ARG (-6)       /* null handle, size mismatch, bad enum */
#define AB2_ERR_UNSUPPORTED (-7)   /* valid request this build does not provide */

/* breakdown scalar, as the string passed to NullValueException */
#define AB2_BREAKDOWN_NONE 0
#define AB2_BREAKDOWN_ALPHA 1
#define AB2_BREAKDOWN_BETA 2
#define AB2_BREAKDOWN_RHO 3

/* matrix storage formats kept on the device (bit flags) */
#define AB2_FMT_CSR 1   /* CSR, int32 columns, as SimpleCSR */
#define AB2_FMT_ELL 2   /* sliced ELL (BEllPack) with 32-row slices */
#define AB2_FMT_F32 4   /* additionally keep an FP32 copy of the values */
#define AB2_FMT_STENCIL 8 /* when the profile is a 3-D 7-point stencil in lexicographic order
                             (row i + nx (j + ny k) holds exactly its in-grid neighbours), also keep
                             the values as 7 bands without column indices -- 4 bands when the matrix
                             is bit-for-bit symmetric; silently absent for other profiles (see
                             ab2_matrix_info.stencil_bands) */

/* SpMV variants (ab2_mult_variant) */
#define AB2_SPMV_AUTO 0
#define AB2_SPMV_CSR_SCALAR 1 /* one thread per row, values read straight from HBM */
#define AB2_SPMV_CSR_STAGED 2 /* row blocks staged through shared memory */
#define AB2_SPMV_ELL 3        /* sliced ELL, one thread per row, coalesced slots */
#define AB2_SPMV_CSR_VECTOR 4 /* FP64, 4/8/16/32 lanes per row by mean row length, 16-byte loads, lanes' partial
                                 sums combined by shuffles: for long rows; NOT the reference's row-sequential
                                 summation order (last-bit differences), so only ab2_mult_variant uses it --
                                 solvers and AUTO never do */
#define AB2_SPMV_STENCIL 5    /* the 7-point bands (AB2_FMT_STENCIL): one thread per row, no column indices,
                                 the row's terms in ascending column order as the CSR sum; AUTO's choice when
                                 present (falls back to ELL, then CSR, where the bands are absent) */

/* solvers / preconditioners (same names as the krylov example's options) */
#define AB2_SOLVER_CG 0
#define AB2_SOLVER_BICGSTAB 1

#define AB2_PC_NONE 0
#define AB2_PC_DIAG 1
#define AB2_PC_ILU0 2
#define AB2_PC_CHEB 3
#define AB2_PC_FILU0 4   /* FILU0Preconditioner.h: ILU(0) by fixed-point sweeps, Jacobi sweeps for L and U */
#define AB2_PC_NEUMANN 5 /* NeumannPolyPreconditioner.h: omega (I + G + ... + G^order) x, G = I - omega A */

/* ------------------------------------------------------------------ handles */
typedef struct ab2_context ab2_context;
typedef struct ab2_matrix ab2_matrix;
typedef struct ab2_vector ab2_vector;
typedef struct ab2_precond ab2_precond;
typedef struct ab2_solver ab2_solver;

/* ------------------------------------------------------------------ context */
int ab2_context_create(int device, ab2_context** ctx);
int ab2_context_destroy(ab2_context* ctx);
const char* ab2_last_error_message(const ab2_context* ctx);
/* cudaStream_t of the context, for callers that record events on it */
int ab2_context_stream(const ab2_context* ctx, void** stream);
int ab2_synchronize(ab2_context* ctx);
/* number of kernels libab2 has launched on this context since creation */
int ab2_context_launch_count(const ab2_context* ctx, long long* count);

/* Every dot product and norm is a grid reduction of reduction_threads-thread
 * blocks, one block per reduction_threads values up to reduction_max_blocks
 * blocks; each thread sums its strided values with fma, blocks and then the
 * block partials are combined by fixed shuffle trees.  The tree depends only
 * on n and the device, so results are reproducible bit for bit. */
typedef struct {
  int device;
  int num_sms;
  int reduction_threads;
  int reduction_max_blocks;
} ab2_context_info;
int ab2_context_get_info(const ab2_context* ctx, ab2_context_info* info);

/* Phase timers (the reference's StdTimer sentries under ALIEN_USE_PERF_TIMER,
 * utils/StdTimer.h): with timing on, every ABI operation records CUDA events
 * on the context's stream around its work and adds its device time to a
 * phase named as the reference's ("CSR-SPMV", "CSR-DOT", "CSR-AXPY", ...,
 * plus "PRECOND-<kind>", "SOLVER-CG", "DIST-SPMV", ...).  Nothing
 * synchronises until the times are read.  AB2_PERF_TIMER=1 in the environment
 * turns it on for every new context and prints the phases ("phase:seconds")
 * when the context is destroyed. */
typedef struct {
  char name[32];
  long long calls;
  double ms;
} ab2_phase_time;
int ab2_context_set_phase_timing(ab2_context* ctx, int on); /* on: (re)start at zero; 0: stop */
/* Writes up to cap phases, *count = phases recorded (synchronises on their events). */
int ab2_context_phase_times(ab2_context* ctx, ab2_phase_time* out, int cap, int* count);

/* ------------------------------------------------------------------ matrix */
/* Copies a host CSR matrix (columns sorted ascending inside each row, as
 * Alien's profilers produce) to the device in the requested formats.
 * The caller keeps ownership of the host arrays. */
int ab2_matrix_create_csr(ab2_context* ctx, int n, const int* row_ptr, const int* cols, const double* vals,
                          int formats, ab2_matrix** mat);
/* New values for the same profile (row_ptr[n] doubles). */
int ab2_matrix_update_values(ab2_context* ctx, ab2_matrix* mat, const double* vals);
int ab2_matrix_destroy(ab2_matrix* mat);

typedef struct {
  int n;
  long long nnz;
  long long ell_stored; /* slots in the sliced-ELL arrays, padding included (0 if absent) */
  int ell_slice;        /* rows per slice (32) */
  int formats;          /* AB2_FMT_* present */
  long long device_bytes;
  int stencil_bands;    /* 0 (no 7-point bands), 7, or 4 (bit-symmetric values) */
  int stencil_nx, stencil_ny, stencil_nz; /* grid of the 7-point profile, 0 when absent */
} ab2_matrix_info;
int ab2_matrix_get_info(const ab2_matrix* mat, ab2_matrix_info* info);

/* ------------------------------------------------------------------ vector */
int ab2_vector_create(ab2_context* ctx, int n, ab2_vector** vec);
int ab2_vector_destroy(ab2_vector* vec);
int ab2_vector_size(const ab2_vector* vec, int* n);
int ab2_vector_upload(ab2_context* ctx, ab2_vector* vec, const double* host);
int ab2_vector_download(ab2_context* ctx, const ab2_vector* vec, double* host);
/* raw device pointer (double*) of the vector's storage */
int ab2_vector_device_ptr(const ab2_vector* vec, void** dptr);

/* ------------------------------------------------------------------ algebra
 * Method-for-method the IInternalLinearAlgebra surface of SimpleCSR/SYCL.
 * All FP64.  Vector arguments must all have the matrix's row count. */
int ab2_mult(ab2_context* ctx, const ab2_matrix* A, const ab2_vector* x, ab2_vector* y);         /* y = A x */
int ab2_mult_variant(ab2_context* ctx, const ab2_matrix* A, const ab2_vector* x, ab2_vector* y, int variant);
int ab2_add_lmult(ab2_context* ctx, double alpha, const ab2_matrix* A, const ab2_vector* x, ab2_vector* y); /* y += a L x */
int ab2_add_umult(ab2_context* ctx, double alpha, const ab2_matrix* A, const ab2_vector* x, ab2_vector* y); /* y += a U x */
int ab2_compute_inv_diag(ab2_context* ctx, const ab2_matrix* A, ab2_vector* inv_diag);           /* d = 1/a_ii */
int ab2_mult_inv_diag(ab2_context* ctx, const ab2_matrix* A, ab2_vector* y);                      /* y = y / a_ii */
int ab2_axpy(ab2_context* ctx, double alpha, const ab2_vector* x, ab2_vector* y);                  /* y += a x */
int ab2_aypx(ab2_context* ctx, double alpha, ab2_vector* y, const ab2_vector* x);                  /* y = a y + x */
int ab2_copy(ab2_context* ctx, const ab2_vector* x, ab2_vector* y);                                /* y = x */
int ab2_scal(ab2_context* ctx, double alpha, ab2_vector* x);                                       /* x = a x */
int ab2_pointwise_mult(ab2_context* ctx, const ab2_vector* x, const ab2_vector* y, ab2_vector* w); /* w = x.y */
int ab2_assign(ab2_context* ctx, ab2_vector* x, double alpha);                                     /* x = a */
int ab2_diagonal(ab2_context* ctx, const ab2_matrix* A, ab2_vector* d);                            /* d = a_ii */
int ab2_reciprocal(ab2_context* ctx, ab2_vector* x);                                               /* x = 1/x */
/* reductions: result copied to host (synchronises) */
int ab2_dot(ab2_context* ctx, const ab2_vector* x, const ab2_vector* y, double* result);
int ab2_norm0(ab2_context* ctx, const ab2_vector* x, double* result); /* max |x_i| */
int ab2_norm1(ab2_context* ctx, const ab2_vector* x, double* result); /* sum |x_i| */
int ab2_norm2(ab2_context* ctx, const ab2_vector* x, double* result); /* sqrt(x.x) */

/* Device scalars: the "future" form of dot (SimpleCSRInternalLinearAlgebra.h:74-98).
 * ab2_dot_async enqueues x.y into a device slot without synchronising;
 * ab2_scalar_get waits for it. */
typedef struct ab2_scalar ab2_scalar;
int ab2_scalar_create(ab2_context* ctx, ab2_scalar** s);
int ab2_scalar_destroy(ab2_scalar* s);
int ab2_dot_async(ab2_context* ctx, const ab2_vector* x, const ab2_vector* y, ab2_scalar* result);
int ab2_scalar_get(ab2_context* ctx, const ab2_scalar* s, double* value);

/* Allocation-free dot product.  No counterpart in the reference: it exists for
 * callers that cannot allocate device memory when they need the reduction
 * (all free HBM handed to another allocator, or a loop that must not pay for
 * cudaMalloc/cudaFree and the device synchronisation they can cause).
 * x, y: device arrays of n doubles on the current device; result: one device
 * double, written on `stream` (a cudaStream_t, NULL for the default stream);
 * nothing is synchronised.  The scratch array used is that of the device that
 * is current on the calling thread (cudaSetDevice): make the device that holds
 * x, y and result current before the call.  The block partials live in a fixed 32 KB device
 * array inside libab2 (one per GPU, held until the process exits), which
 * limits n to 16,777,216; larger n returns AB2_ERR_BAD_ARG.  The first call on
 * each device looks that array up (cudaGetSymbolAddress): make it before any
 * stream capture.  All calls share the array: calls that overlap on the GPU
 * (unordered streams or host threads) race and give wrong results. */
int ab2_dot_noalloc(const double* x, const double* y, int n, double* result, void* stream);

/* ------------------------------------------------------------------ preconditioners */
/* ILU(0) schedules; all give the same factor and applications bit for bit.
 * WAVEFRONT: any CSR matrix; rows grouped by wavefront of the triangular
 *   graphs, one warp per 32 rows, cross-warp waits through global memory.
 * STENCIL: 3-D 7-point matrices in lexicographic order; 16x16 tiles of
 *   grid lines per CTA walk their diagonals through shared memory; values
 *   between tiles through global memory.
 * STENCIL_CLUSTER: the STENCIL walk with 2x2 tiles per thread-block cluster;
 *   values between the tiles of a cluster go straight into the neighbour's
 *   shared memory.  Its buffers must fit shared memory: up to ~350 planes
 *   along z (a request beyond that is refused).
 * AUTO: STENCIL_CLUSTER, else STENCIL when the matrix has that structure,
 *   else WAVEFRONT. */
#define AB2_ILU_AUTO 0
#define AB2_ILU_WAVEFRONT 1
#define AB2_ILU_STENCIL 2
#define AB2_ILU_STENCIL_CLUSTER 3

typedef struct {
  int kind;                 /* AB2_PC_* */
  double poly_factor;       /* Chebyshev: 0 = both bounds by power method; else alpha = beta/factor */
  int poly_order;           /* Chebyshev polynomial order (3 = three SpMVs per application) */
  int poly_factor_max_iter; /* Chebyshev: power-method steps per bound (Lanczos steps with cheb_lanczos) */
  int ilu_schedule;         /* AB2_ILU_* */
  int cheb_saad;    /* 0: ChebyshevPreconditioner<.., false> (_algo2, y starts at x, the reference default);
                       1: ChebyshevPreconditioner<.., true> (_algo1, y starts at 0: a symmetric operator) */
  int cheb_lanczos; /* 0: bounds by the reference's two power methods; 1: alpha = smallest and
                       beta = 1.1 x largest Ritz value of poly_factor_max_iter Lanczos steps on
                       D^-1/2 A D^-1/2 (no counterpart in the reference) */
  int filu_factor_iter; /* FILU0 "nb-factor-iter": 0 = the exact ILU(0) factor; k > 0 = k fixed-point
                           sweeps from A (FLUFactorisationAlgo::factorizeMultiIter) */
  int filu_solver_iter; /* FILU0 "nb-solver-iter": Jacobi sweeps per triangular solve (0: identity) */
  double filu_tol;      /* FILU0 "tol": accepted and unused, as in the reference */
} ab2_precond_options;

/* init(): Diag computes 1/a_ii; ILU0 factorises on the device; Chebyshev
 * estimates its bounds; FILU0 factorises (exactly or by fixed-point sweeps)
 * and stores L and U as sliced ELL; Neumann takes poly_factor as omega, or
 * (poly_factor = 0) 1 / the power-method estimate of |lambda_max| after
 * poly_factor_max_iter steps -- from a default-seeded std::mt19937 start vector
 * where NeumannPolyPreconditioner.h:143-145 seeds from std::random_device.
 * The matrix must outlive the preconditioner. */
int ab2_precond_create(ab2_context* ctx, const ab2_matrix* A, const ab2_precond_options* opts, ab2_precond** pc);
int ab2_precond_apply(ab2_context* ctx, const ab2_precond* pc, const ab2_vector* x, ab2_vector* y); /* y = M^-1 x */
int ab2_precond_destroy(ab2_precond* pc);

typedef struct {
  int kind;
  double cheb_alpha; /* lower bound used by Chebyshev */
  double cheb_beta;  /* upper bound used by Chebyshev */
  int ilu_levels_lower; /* wavefronts of the L sweep */
  int ilu_levels_upper; /* wavefronts of the U sweep */
  int ilu_schedule;     /* AB2_ILU_WAVEFRONT, AB2_ILU_STENCIL or AB2_ILU_STENCIL_CLUSTER as chosen */
  double neumann_factor; /* omega used by Neumann */
} ab2_precond_info;
int ab2_precond_get_info(const ab2_precond* pc, ab2_precond_info* info);
/* ILU(0) factor values in CSR order (row_ptr[n] doubles), for checking. */
int ab2_precond_ilu0_values(ab2_context* ctx, const ab2_precond* pc, double* lu);

/* ------------------------------------------------------------------ solver */
typedef struct {
  int solver;   /* AB2_SOLVER_* */
  int precond;  /* AB2_PC_* */
  double tol;   /* stop when r.r < tol^2 b.b (recursive residual, Iteration.h:83-90) */
  int max_iter;
  double poly_factor;
  int poly_order;
  int poly_factor_max_iter;
  int spmv_variant; /* AB2_SPMV_* used inside the loop */
  int use_graph;    /* 1: iteration loop in a CUDA graph with a device-side while condition */
  int ilu_schedule; /* AB2_ILU_* */
  int cheb_saad;    /* see ab2_precond_options */
  int cheb_lanczos;
  int filu_factor_iter; /* see ab2_precond_options */
  int filu_solver_iter;
  double filu_tol;
} ab2_solver_options;

typedef struct {
  int succeeded;          /* Iteration::getStatus() */
  int iterations;         /* Iteration::operator()() */
  int error;              /* AB2_OK, AB2_ERR_BREAKDOWN, AB2_ERR_TIMEOUT */
  int breakdown;          /* AB2_BREAKDOWN_* */
  double residual;        /* sqrt(last stop value / b.b): recursive relative residual */
  double true_residual;   /* ||b - A x|| / ||b|| recomputed after the solve */
  double nrm2_b;          /* b.b */
  double setup_ms;        /* preconditioner init + graph build of the last ab2_solver_create */
  double solve_ms;        /* device time of the last solve */
} ab2_status;

void ab2_solver_options_default(ab2_solver_options* opts);
int ab2_solver_create(ab2_context* ctx, const ab2_matrix* A, const ab2_solver_options* opts, ab2_solver** s);
/* x holds the initial guess on entry, the solution on exit. */
int ab2_solver_solve(ab2_solver* s, const ab2_vector* b, ab2_vector* x, ab2_status* status);
/* residual history: the stop test's r.r values of the last solve */
int ab2_solver_history(const ab2_solver* s, double* hist, int cap, int* len);
int ab2_solver_destroy(ab2_solver* s);

/* ------------------------------------------------------------------ mixed precision
 * FP32 Krylov inside FP64 iterative refinement.  No counterpart in the
 * reference (its solvers run in the matrix's value type); the inner solver is
 * the reference's CG.h / BiCGStab.h and preconditioners instantiated in float.
 * Each refinement step: r = b - A x and ||r|| in FP64; stop when
 * ||r|| / ||b|| < tol; inner solve A32 d = float(r / ||r||) from d = 0 to the
 * recursive residual inner_tol (FP32 values, FP32 accumulation, FP32
 * scalars); x += ||r|| d in FP64.  The matrix must carry FP32 values
 * (AB2_FMT_F32); the FP32 preconditioner is the FP64 set-up rounded. */
typedef struct ab2_mixed ab2_mixed;

typedef struct {
  int solver;          /* inner: AB2_SOLVER_CG or AB2_SOLVER_BICGSTAB */
  int precond;         /* inner, applied in FP32: AB2_PC_* */
  double tol;          /* outer: true relative residual ||b - A x|| / ||b||, FP64 */
  int max_outer;       /* refinement steps */
  double inner_tol;    /* inner: relative residual of each FP32 solve, in (0, 1) */
  int inner_max_iter;  /* inner: iterations per refinement step */
  double poly_factor;  /* Chebyshev settings as in ab2_precond_options */
  int poly_order;
  int poly_factor_max_iter;
  int cheb_saad;
  int cheb_lanczos;
  int ilu_schedule;    /* AB2_ILU_* */
  int spmv_variant;    /* AB2_SPMV_* for both precisions */
  int use_graph;       /* inner loop in a CUDA graph */
  int filu_factor_iter; /* see ab2_precond_options */
  int filu_solver_iter;
  double filu_tol;
  int jacobi_form;     /* CG + Diag only: AB2_MIXED_JACOBI_* */
} ab2_mixed_options;

/* How the mixed solver runs CG + Diag.  PLAIN: the FP32 Jacobi-PCG on A32.
 * SCALED: the same method in its symmetrically scaled form -- plain CG on
 * S A S (S = diag(1/sqrt(a_ii)), computed in FP64 then rounded: a unit
 * diagonal and three FP32 bands), with r32 = float(S r / ||r||) and
 * x += ||r|| S d; it needs a bit-symmetric 7-point matrix kept as bands
 * (AB2_FMT_STENCIL, ab2_matrix_info.stencil_bands == 4) with a positive
 * diagonal, and moves about half the bytes per inner iteration.  AUTO: SCALED
 * when the matrix allows it, else PLAIN.  ab2_mixed_status.jacobi_scaled
 * tells which ran. */
#define AB2_MIXED_JACOBI_AUTO 0
#define AB2_MIXED_JACOBI_PLAIN 1
#define AB2_MIXED_JACOBI_SCALED 2

typedef struct {
  int succeeded;          /* final true relative residual < tol */
  int outer_iterations;   /* refinement steps (inner solves) taken */
  int inner_iterations;   /* FP32 Krylov iterations over all steps */
  int error;              /* AB2_OK; AB2_ERR_NOT_CONVERGED (max_outer reached, or a step did not
                             reduce the true residual); AB2_ERR_BREAKDOWN (an inner solve broke
                             down before its first iteration); AB2_ERR_TIMEOUT */
  double true_residual;   /* final ||b - A x|| / ||b||, FP64 */
  double setup_ms;        /* FP64 preconditioner set-up + FP32 copies + graph build */
  double solve_ms;        /* device time of the last solve */
  int jacobi_scaled;      /* 1 when CG + Diag ran in the scaled form (AB2_MIXED_JACOBI_SCALED) */
} ab2_mixed_status;

void ab2_mixed_options_default(ab2_mixed_options* opts);
int ab2_mixed_create(ab2_context* ctx, const ab2_matrix* A, const ab2_mixed_options* opts, ab2_mixed** m);
/* x holds the initial guess on entry, the solution on exit (FP64). */
int ab2_mixed_solve(ab2_mixed* m, const ab2_vector* b, ab2_vector* x, ab2_mixed_status* status);
/* true relative residual before each refinement step and at the end of the last solve */
int ab2_mixed_history(const ab2_mixed* m, double* res, int cap, int* len);
int ab2_mixed_destroy(ab2_mixed* m);

/* ------------------------------------------------------------------ batched systems
 * Many independent systems of uneven sizes in ONE persistent launch.  No
 * counterpart in the reference (its solvers take one system at a time); the
 * per-system method is CG.h's Jacobi-PCG in FP32 inside FP64 refinement (as
 * ab2_mixed).  The systems are the diagonal blocks of one block-diagonal
 * matrix: system s is rows sys_offsets[s] .. sys_offsets[s+1]-1, and no row
 * may reference a column outside its block.  The matrix must carry FP32
 * values (AB2_FMT_F32).  A grid of thread-block clusters, as many as fit on
 * the GPU at once, takes systems largest first from a ticket; a cluster
 * solves its system to the per-system true relative residual tol, then takes
 * the next.  The inner SpMV format -- sliced ELL with 16, 32 or 64 rows per
 * slice, or CSR with 1, 2, 4 or 8 lanes per row -- the CTAs per system
 * (cluster size) and the threads per CTA are picked by timing candidates on
 * the batch at creation (the autotuner) unless fixed in the options. */
typedef struct ab2_batch ab2_batch;

typedef struct {
  double tol;          /* per system: ||b_s - A_s x_s|| / ||b_s|| (FP64) */
  int max_outer;       /* refinement steps per system */
  double inner_tol;    /* FP32 inner CG: relative recursive residual, in (0, 1) */
  int inner_max_iter;  /* FP32 iterations per refinement step */
  int spmv_variant;    /* AB2_SPMV_AUTO (autotune), AB2_SPMV_ELL or AB2_SPMV_CSR_SCALAR */
  int cluster_size;    /* CTAs per system: 0 (autotune), 1, 2, 4, 8 or 16 (16: where the GPU places it) */
  int threads;         /* threads per CTA: 0 (autotune) or 64..1024, a multiple of 32 */
  int tune_iters;      /* FP32 iterations per system in each autotuning trial (0: 8) */
  int ell_slice;       /* AB2_SPMV_ELL: rows per slice, 0 (autotune), 16, 32 or 64 */
  int lanes_per_row;   /* AB2_SPMV_CSR_SCALAR: lanes per row (rows per warp = 32 / it), 0 (autotune), 1, 2,
                          4 or 8; more than one sums a row in an xor-butterfly tree of per-lane partials */
} ab2_batch_options;

typedef struct {
  int spmv_variant, cluster_size, threads;
  float ms;            /* one trial's score: tune_iters FP32 iterations of every system plus
                          4 x tune_iters of the largest system alone (throughput + long pole) */
  int ell_slice, lanes_per_row;  /* the format's shape (0 where it does not apply) */
} ab2_batch_trial;

typedef struct {
  int nsys;
  long long rows;
  int spmv_variant, cluster_size, threads;  /* configuration in use */
  int tuned;            /* 1 if the autotuner chose it */
  double tune_ms;       /* time spent autotuning */
  double setup_ms;      /* creation, autotuning included */
  int trials;           /* number of autotuning trials (ab2_batch_trials) */
  int ell_slice, lanes_per_row;  /* the format's shape in use (0 where it does not apply) */
} ab2_batch_info;

typedef struct {
  int systems_converged;
  int max_outer;        /* most refinement steps any system took */
  long long inner_total;/* FP32 iterations, all systems */
  int inner_max;        /* most FP32 iterations any system took */
  double max_residual;  /* largest final true relative residual */
  double solve_ms;      /* device time of the solve (one launch) */
} ab2_batch_status;

void ab2_batch_options_default(ab2_batch_options* opts);
int ab2_batch_create(ab2_context* ctx, const ab2_matrix* A, int nsys, const int* sys_offsets,
                     const ab2_batch_options* opts, ab2_batch** batch);
/* x holds the initial guesses on entry, the solutions on exit (FP64). */
int ab2_batch_solve(ab2_batch* batch, const ab2_vector* b, ab2_vector* x, ab2_batch_status* status);
/* per-system results of the last solve (host arrays of nsys; any may be NULL) */
int ab2_batch_results(const ab2_batch* batch, int* converged, int* outer, int* inner, double* residual);
int ab2_batch_get_info(const ab2_batch* batch, ab2_batch_info* info);
int ab2_batch_trials(const ab2_batch* batch, ab2_batch_trial* trials, int cap);
int ab2_batch_destroy(ab2_batch* batch);

/* ------------------------------------------------------------------ learned preconditioner
 * No counterpart in the reference.  A message-passing network on the matrix
 * graph maps a residual r to z ~ A^-1 r, working on the diagonal-scaled
 * system D^-1/2 A D^-1/2 (unit diagonal):
 *   xr_i = r_i / sqrt(a_ii), s = rms(xr), x0_i = [xr_i / s, log(a_ii)/10]
 *   h1 = relu(W0 x0 + b0)                                                    (2 -> 64)
 *   4 layers: m_i = sum_j sigmoid(u e_ij + c) h_j,
 *             e_ij = log|a_ij| - (log a_ii + log a_jj)/2,
 *             h <- relu(W [h ; m] + b)                                       (128 -> 64)
 *   z_i = s (wd . h_i + bd + ws x0_i[0]) / sqrt(a_ii)
 * With wd = 0, bd = 0, ws = 1 the network is Jacobi (z = r / a_ii).
 * Weights are kept in FP32 for training and used as BF16 in the dense layers
 * (tensor cores, FP32 accumulation); activations are stored in BF16.
 * Training (on the GPU, hand-written backward kernels, Adam): pairs (r, e) of
 * a residual and the error it leaves, loss (z-e)^T A (z-e) / e^T A e.
 * Parameters: ab2_gnn_param_count() floats in the order W0 (64x2), b0, W1..W4
 * (64x128 each, row = output), b1..b4, u1..u4, c1..c4, wd, bd, ws.  The matrix
 * must have a positive diagonal and a structurally symmetric pattern. */
typedef struct ab2_gnn ab2_gnn;

int ab2_gnn_param_count(void);
/* params: NULL for a seeded He-style initialisation */
int ab2_gnn_create(ab2_context* ctx, const float* params, unsigned long long seed, ab2_gnn** gnn);
int ab2_gnn_get_params(const ab2_gnn* gnn, float* params);
int ab2_gnn_set_params(ab2_gnn* gnn, const float* params);
/* Layer kernels.  GATHER: any graph; a warp takes 16 nodes, copies their
 * neighbours' rows by index (cp.async) and runs both products on mma.sync.
 * GRID: a 3-D 7-point matrix in lexicographic order (rows i + nx (j + ny k));
 * 128 consecutive nodes a tile, each direction's neighbour rows one contiguous
 * block (bulk copies, no gather), the aggregation on the CUDA cores and the
 * dense layer on tcgen05 tensor cores with the accumulator in tensor memory.
 * AUTO (the default): GRID when the bound matrix has the 3-D 7-point profile,
 * else GATHER.  The two give the same network up to the order of the FP32
 * aggregation sums. */
#define AB2_GNN_LAYER_AUTO 0
#define AB2_GNN_LAYER_GATHER 1
#define AB2_GNN_LAYER_GRID 2
/* Takes effect at the next bind; GRID then fails with AB2_ERR_UNSUPPORTED on
 * a matrix without the 3-D 7-point profile. */
int ab2_gnn_set_layer(ab2_gnn* gnn, int layer);
/* The kernel the current binding uses (GATHER or GRID; AUTO when unbound). */
int ab2_gnn_get_layer(const ab2_gnn* gnn, int* layer);
/* Reads the graph features of A and sizes the activation buffers (A must outlive the binding). */
int ab2_gnn_bind(ab2_gnn* gnn, const ab2_matrix* A);
int ab2_gnn_apply(ab2_gnn* gnn, const ab2_vector* r, ab2_vector* z);   /* z = network(r), r != z */
/* loss of one (r, e) pair and its gradient (grad: host array of param_count floats, or NULL) */
int ab2_gnn_loss_grad(ab2_gnn* gnn, const ab2_vector* r, const ab2_vector* e, double* loss, float* grad);
/* one Adam step (beta1 0.9, beta2 0.999) on one pair; loss before the step */
int ab2_gnn_train_step(ab2_gnn* gnn, const ab2_vector* r, const ab2_vector* e, double lr, double* loss);
int ab2_gnn_destroy(ab2_gnn* gnn);

#define AB2_FCG_FALLBACK_STICKY 0 /* the fallback keeps the rest of the solve (direction window cleared) */
#define AB2_FCG_FALLBACK_STEP 1   /* the fallback preconditions the step after each failed network step */

/* Flexible CG with truncated A-orthogonalisation (Notay's FCG(m)): each new
 * direction p = z - sum_i (z . A p_i / p_i . A p_i) p_i over the last
 * `truncation` directions, alpha = p . r / p . A p, so that a preconditioner
 * that is not a fixed linear operator (the network) keeps the directions
 * conjugate.  The network is the preconditioner; a network step "fails" when
 * it reduces ||r|| by less than the factor fallback_ratio (1.0: a step that
 * does not reduce it at all).  Then the fallback (ILU(0)) takes over: for the
 * rest of the solve with the direction window cleared (STICKY), or for the
 * next step only, the network resuming after it (STEP, the default).
 * gnn = NULL: flexible CG with the fallback only.
 * Stops when ||r|| / ||b|| < tol (the true residual is reported after). */
typedef struct {
  double tol;
  int max_iter;
  double fallback_ratio;
  int truncation;       /* directions kept, 1..16 (1: PCG with a fixed SPD preconditioner) */
  int fallback_mode;    /* AB2_FCG_FALLBACK_STICKY or AB2_FCG_FALLBACK_STEP */
} ab2_fcg_options;

typedef struct {
  int succeeded;
  int iterations;
  int gnn_steps;        /* preconditioner applications by the network */
  int fallback_steps;   /* ... by the fallback */
  int switched_at;      /* iteration of the first failed network step, -1 if none failed */
  int error;            /* AB2_OK, AB2_ERR_NOT_CONVERGED, AB2_ERR_BREAKDOWN, AB2_ERR_TIMEOUT */
  double true_residual;
  double solve_ms;
} ab2_fcg_status;

void ab2_fcg_options_default(ab2_fcg_options* opts);
int ab2_fcg_solve(ab2_context* ctx, const ab2_matrix* A, ab2_gnn* gnn, const ab2_precond* fallback,
                  const ab2_vector* b, ab2_vector* x, const ab2_fcg_options* opts, ab2_fcg_status* status);

/* ------------------------------------------------------------------ self-test
 * Failure detection of the bounded device-side waits, without a fault: one
 * thread polls a sentinel word that nothing writes; the wait gives up after
 * its clock budget (~2 s), sets the error flag (*expired = 1) and the kernel
 * ends; *seconds is the wall time.  The context stays usable. */
int ab2_selftest_bounded_wait(ab2_context* ctx, int* expired, double* seconds);
/* The same for the mbarrier waits of the learned preconditioner's grid layer:
 * a wait on a barrier phase that nothing completes gives up after its clock
 * budget; *expired = 1 when it did. */
int ab2_selftest_mbarrier_wait(ab2_context* ctx, int* expired, double* seconds);
/* Host-side fault injection: the nth device allocation on ctx from now on
 * fails as AB2_ERR_OOM (once); 0 turns it off. */
int ab2_context_inject_alloc_failure(ab2_context* ctx, long long nth);

#ifdef __cplusplus
}
#endif

#endif /* AB2_H */
