// precond.cuh -- preconditioner state shared by precond.cu and krylov.cu.
#pragma once

#include <vector>

#include "ab2_internal.cuh"

namespace ab2 {

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
};

struct ChebData {
  double alpha = 0, beta = 0;
  int order = 0;
  std::vector<double> a;   // alpha_i of each step (step 0: 2/d)
  std::vector<double> b;   // beta_i of each step >= 1
  double* d_p = nullptr;
  double* d_y[2] = {nullptr, nullptr};
  double* d_xcopy = nullptr;
};

}  // namespace ab2

struct ab2_precond {
  ab2_context* ctx = nullptr;
  const ab2_matrix* A = nullptr;
  int kind = AB2_PC_NONE;
  int variant = AB2_SPMV_AUTO;
  double* d_inv = nullptr;  // 1/a_ii (Diag, Chebyshev)
  ab2::Ilu0Data ilu;
  ab2::ChebData cheb;
};

namespace ab2 {

// y = M^-1 x, stream ordered, capturable in a CUDA graph.
void pc_apply(ab2_context* ctx, const ab2_precond* pc, const double* x, double* y);
// Resets ILU0 sweep state after a failed (timed-out) application.
void pc_reset(ab2_context* ctx, const ab2_precond* pc);
int pc_error(ab2_context* ctx, const ab2_precond* pc);

}  // namespace ab2
