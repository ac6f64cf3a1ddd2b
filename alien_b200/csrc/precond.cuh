// precond.cuh -- preconditioner state shared by precond.cu and krylov.cu.
#pragma once

#include <vector>

#include "ab2_internal.cuh"

struct ab2_matrix;

namespace ab2 {

struct Ilu0Data;

// ILU(0) on the device.  The factor keeps the CSR profile of A (L strictly
// below dcol with unit diagonal implied, U from dcol on), as
// LUFactorisationAlgo does (ILU0Preconditioner.h:51-178).
struct Ilu0Data {
  double* d_lu = nullptr;
  // Rows grouped by wavefront and padded with -1 to whole warps per wavefront,
  // so the 32 rows a warp takes never depend on each other.
  int* d_perm_l = nullptr;
  int* d_perm_u = nullptr;
  int len_l = 0, len_u = 0;
  int levels_l = 0, levels_u = 0;
  int widest_l = 1, widest_u = 1;   // chunks in the widest wavefront
  std::vector<int> lev_ptr_l;       // host: wavefront starts in perm_l (factorisation launches)
  std::vector<int> h_perm_l;
  double* d_tmp = nullptr;          // L-sweep output, left at the sentinel between applications
  unsigned int* d_counters = nullptr;  // [0]: L-sweep chunk ticket, [1]: U-sweep chunk ticket
  int* d_err = nullptr;             // set when a bounded wait gives up
  // 7-point lexicographic matrices: tile-walk schedule (ilu_stencil.cu)
  bool stencil = false;
  int st_nx = 0, st_ny = 0, st_nz = 0;
  double* d_bands = nullptr;            // set-up only: 8 n-vectors L(-k,-j,-i) U(+i,+j,+k) pivot diag
  unsigned int* d_tile_tickets = nullptr;  // factorisation, L sweep, U sweep
  // Walk layout (ilu_stencil.cu): 10 arrays of walk_n doubles -- the factor's
  // L(-k,-j,-i), U(+i,+j,+k) and pivot bands, the gathered right-hand side,
  // and the two sweeps' propagation arrays.
  long long walk_n = 0;
  double* d_walk = nullptr;
  float* d_walk32 = nullptr;  // the same arrays in FP32 (mixed-precision inner solves), built on demand
  bool walk_cluster = false;  // sweeps in 2 x 2-tile clusters (else one tile per CTA)
};

// Detects a 3-D 7-point matrix in lexicographic order and, if found,
// factorises it on the tile-walk schedule (bands + CSR copy in d_lu); with
// factored, d_lu already holds the factor and only the walk arrays are built.
// schedule (AB2_ILU_*): AB2_ILU_STENCIL keeps one tile per CTA; AUTO and
// AB2_ILU_STENCIL_CLUSTER take the cluster walk when it fits (the latter
// fails otherwise).
bool ilu_stencil_setup(ab2_context* ctx, const ab2_matrix* A, Ilu0Data& d, bool factored, int schedule);
void ilu_stencil_apply(ab2_context* ctx, const ab2_matrix* A, const Ilu0Data& d, const double* y, double* z);
// Puts the sweeps' propagation arrays back to the sentinel (after a failed application).
void ilu_stencil_reset(ab2_context* ctx, const Ilu0Data& d);
// FP32 copies of the walk arrays (the FP64 factor rounded) and the FP32 application.
void ilu_stencil_enable_f32(ab2_context* ctx, Ilu0Data& d);
void ilu_stencil_apply_f32(ab2_context* ctx, const Ilu0Data& d, const float* y, float* z);

struct ChebData {
  double alpha = 0, beta = 0;
  int order = 0;
  bool saad = false;
  std::vector<double> a;   // _algo2: alpha_i of each step (step 0: 2/d); _algo1: rho rho_old of step i
  std::vector<double> b;   // _algo2: beta_i of each step >= 1;          _algo1: 2 rho / delta of step i
  double inv_theta = 0;    // _algo1: 1 / theta
  double* d_p = nullptr;   // _algo2: p; _algo1: r
  double* d_y[2] = {nullptr, nullptr};  // _algo2: iterates; _algo1: w (ping-pong)
  double* d_xcopy = nullptr;
};

// FILU0 (FILU0Preconditioner.h): the factor in CSR order (exact ILU(0) or
// fixed-point sweeps), its strict L and strict U parts as sliced ELL (32-row
// slices, slot-major, column -1 for padding, CSR order kept inside each row)
// and 1/u_ii; the application is solver_iter Jacobi sweeps for L then for U.
struct FiluData {
  int factor_iter = 0, solver_iter = 0;
  double tol = 0;
  int* d_l_off = nullptr;  // slice offsets (in 32-row slot groups), n_slices + 1
  int* d_l_ci = nullptr;
  double* d_l_v = nullptr;
  int* d_u_off = nullptr;
  int* d_u_ci = nullptr;
  double* d_u_v = nullptr;
  double* d_inv = nullptr;        // 1/u_ii
  double* d_t[2] = {nullptr, nullptr};  // sweep work vectors
  float* d_l_v32 = nullptr;       // FP32 forms (pc_enable_f32)
  float* d_u_v32 = nullptr;
  float* d_inv32 = nullptr;
  float* d_t32 = nullptr;         // 2 n
};

// Neumann polynomial (NeumannPolyPreconditioner.h): omega and the order.
struct NeumannData {
  double omega = 0;
  int order = 0;
  double* d_t[3] = {nullptr, nullptr, nullptr};  // ping-pong iterates + a copy of an aliased input
  float* d_t32 = nullptr;                         // 3 n
};

// ILU(0) set-up into pc->ilu (precond.cu): factor plus the sweep schedule.
// With lu (device, A's CSR profile) the factor is taken as given -- the
// block-Jacobi factor of a distributed matrix -- and only the schedule is built.
void ilu_init(ab2_context* ctx, ab2_precond* pc, int schedule, const double* lu = nullptr);
void filu_init(ab2_context* ctx, ab2_precond* pc, const ab2_precond_options* o);
void neumann_init(ab2_context* ctx, ab2_precond* pc, const ab2_precond_options* o);
template <class T>
void filu_apply(ab2_context* ctx, const ab2_precond* pc, const T* x, T* y);
template <class T>
void neumann_apply(ab2_context* ctx, const ab2_precond* pc, const T* x, T* y);
void filu_enable_f32(ab2_context* ctx, ab2_precond* pc);
void neumann_enable_f32(ab2_context* ctx, ab2_precond* pc);
void filu_neumann_release(ab2_context* ctx, ab2_precond* pc);
// Keeps the ILU(0) factor (d_lu) and frees the sweep schedule's arrays.
void ilu_drop_schedule(ab2_context* ctx, Ilu0Data& d);

}  // namespace ab2

struct ab2_precond {
  ab2_context* ctx = nullptr;
  const ab2_matrix* A = nullptr;
  int kind = AB2_PC_NONE;
  int variant = AB2_SPMV_AUTO;
  double* d_inv = nullptr;  // 1/a_ii (Diag, Chebyshev)
  ab2::Ilu0Data ilu;
  ab2::ChebData cheb;
  ab2::FiluData fil;
  ab2::NeumannData neu;
  // FP32 form for the inner solves of the mixed-precision solver
  // (pc_enable_f32): the FP64 set-up's results rounded to float.
  bool f32 = false;
  float* d_inv32 = nullptr;
  float* d_lu32 = nullptr;    // wavefront ILU(0) factor
  float* d_tmp32 = nullptr;   // wavefront ILU(0) forward-sweep output (sentinel between applications)
  float* d_cheb32 = nullptr;  // Chebyshev work vectors p | y0 | y1 | xcopy
};

namespace ab2 {

// y = M^-1 x, stream ordered, capturable in a CUDA graph.
void pc_apply(ab2_context* ctx, const ab2_precond* pc, const double* x, double* y);
// Builds the FP32 form (the matrix must carry FP32 values for Chebyshev), and
// applies it: the same operations in float.
void pc_enable_f32(ab2_context* ctx, ab2_precond* pc);
void pc_apply_f32(ab2_context* ctx, const ab2_precond* pc, const float* x, float* y);
// Resets ILU0 sweep state after a failed (timed-out) application.
void pc_reset(ab2_context* ctx, const ab2_precond* pc);
int pc_error(ab2_context* ctx, const ab2_precond* pc);

}  // namespace ab2
