// dist.cuh -- internal types of the row-block distribution (dist.cu,
// dist_solver.cu); not part of the ABI.
#pragma once

#include <vector>

#include "ab2_dist.h"
#include "ab2_internal.cuh"

namespace ab2 {

// Exchange plan of one distributed matrix on one rank.
struct HaloPlan {
  std::vector<int> recv_ranks, recv_off;  // ghost slice [recv_off[i], recv_off[i+1]) comes from recv_ranks[i]
  std::vector<int> send_ranks, send_off;  // send-buffer slice [send_off[j], send_off[j+1]) goes to send_ranks[j]
};

}  // namespace ab2

struct ab2_comm {
  int rank = 0, size = 1;
  ab2_context* ctx = nullptr;
  cudaStream_t cs = nullptr;        // transfers
  cudaEvent_t ev_ready = nullptr;   // context stream -> transfer stream
  cudaEvent_t ev_done = nullptr;    // transfer stream -> context stream
  double* d_gather = nullptr;       // size * kMaxRedComps gathered partials
  double* d_sum = nullptr;          // kMaxRedComps rank-ordered sums
  long long seq = 0;

  virtual ~ab2_comm() {}
  // Every rank's vector, in rank order (host data, set-up only).
  virtual std::vector<std::vector<int>> host_allgather(const std::vector<int>& mine) = 0;
  // Number the next collective; the returned parity selects the buffers it publishes.
  int next() {
    const int p = (int)(seq & 1);
    ++seq;
    before_publish(p);
    return p;
  }
  // The halo: sendbuf was packed on ctx->stream; ghosts receive.  Work queued
  // on ctx->stream after halo_finish() sees the ghosts.
  virtual void halo_start(const ab2::HaloPlan& plan, int parity, const double* sendbuf, double* ghosts) = 0;
  void halo_finish() { AB2_CUDA(cudaStreamWaitEvent(ctx->stream, ev_done, 0)); }
  // out[r k + j] = rank r's in[j] (ordered on ctx->stream).
  virtual void allgather(int parity, const double* in, int k, double* out) = 0;

 protected:
  virtual void before_publish(int parity) { (void)parity; }
};

struct ab2_dist_matrix {
  ab2_context* ctx = nullptr;
  ab2_comm* comm = nullptr;
  int global_n = 0, n_loc = 0, n_ghost = 0, first_upper_ghost = 0;
  std::vector<int> offsets;
  // host layout (DistStructInfo)
  std::vector<int> h_rp, h_ci, h_lrs, h_ghost_uids, h_iface, h_send_ids;
  std::vector<double> h_v;
  ab2::HaloPlan plan;
  ab2_matrix* local = nullptr;
  // device: exchange and interface rows
  int n_send = 0;
  int* d_send_ids = nullptr;
  double* d_send[2] = {nullptr, nullptr};
  int n_iface = 0;
  long long ghost_nnz = 0;
  int* d_iface = nullptr;
  int* d_gp = nullptr;
  int* d_gc = nullptr;
  double* d_gv = nullptr;
};

namespace ab2 {

// y = A x on the rank's rows (x has room for the ghosts); collective.
void dist_mult(ab2_context* ctx, const ab2_dist_matrix* A, double* x, double* y);
// out[0..k) = rank-ordered sums of every rank's in[0..k) (device); collective.
void dist_sum(ab2_context* ctx, ab2_comm* c, const double* in, int k, double* out);
// Block-Jacobi ILU(0) factor of the rank's rows in the diagonal block's CSR order.
double* dist_bj_factor(ab2_context* ctx, const ab2_dist_matrix* A);

}  // namespace ab2
