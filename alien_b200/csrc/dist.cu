// dist.cu -- row-block distribution of the algebra (include/ab2_dist.h).
//
// Communicators (ab2_comm):
//   * local group: several ranks in one process, one host thread and one
//     context each.  A collective is a host barrier plus device-to-device
//     copies ordered by CUDA events; no kernel waits on another rank.
//     Buffers a rank publishes (its halo send buffer, its partial sums) are
//     double-buffered by the parity of the collective's sequence number, so a
//     rank overwrites a buffer only after the peers' reads of it, queued two
//     collectives earlier, have completed (it waits on their "consumed"
//     events, recorded before the barrier it has since passed).
//   * NCCL: one rank per GPU; grouped ncclSend/ncclRecv for the halo and
//     ncclAllGather for partial sums, on a transfer stream beside the
//     context's stream.  libnccl is loaded at run time.
//
// The distributed matrix restates DistStructInfo::compute
// (kernels/simple_csr/DistStructInfo.cc:44-233) after sortGhostCols
// (SimpleCSRMatrix.h:215-258): local columns first in each row, then ghosts;
// ghost ids grouped by owner, ascending; exchange lists as m_send_info /
// m_recv_info.  The diagonal block is an ordinary ab2_matrix, so the local
// part of the SpMV, the Diag/ILU0 sweeps and the BLAS-1 run on the
// single-GPU kernels; the interface rows' ghost sums are one more kernel.
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "ab2_dist.h"
#include "ab2_internal.cuh"
#include "dist.cuh"
#include "precond.cuh"

namespace ab2 {
namespace {

// ------------------------------------------------------------------ local group
struct LocalGroup {
  int size = 0;
  double timeout_s = 120.0;
  std::mutex m;
  std::condition_variable cv;
  long long gen = 0;
  int arrived = 0;
  bool broken = false;
  struct Slot {
    cudaEvent_t produced[2] = {nullptr, nullptr};  // the rank's published data of that parity is written
    cudaEvent_t consumed[2] = {nullptr, nullptr};  // the rank has read the peers' data of that parity
    const double* send[2] = {nullptr, nullptr};
    const HaloPlan* plan[2] = {nullptr, nullptr};
    double* pub[2] = {nullptr, nullptr};            // kMaxRedComps partials
    char op[2] = {0, 0};                            // 'h' halo, 'g' gather: ranks must agree
    std::vector<int> host;
  };
  std::vector<Slot> slots;

  // All ranks meet; a rank that waits longer than timeout_s breaks the group
  // and every later barrier fails at once.
  void barrier() {
    std::unique_lock<std::mutex> lk(m);
    if (broken) throw Error{AB2_ERR_TIMEOUT, "local group: another rank gave up at a barrier"};
    const long long g = gen;
    if (++arrived == size) {
      arrived = 0;
      ++gen;
      cv.notify_all();
      return;
    }
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
    while (gen == g && !broken) {
      if (cv.wait_until(lk, deadline) == std::cv_status::timeout && gen == g) {
        broken = true;
        cv.notify_all();
        throw Error{AB2_ERR_TIMEOUT, "local group: barrier timed out waiting for the other ranks"};
      }
    }
    if (gen == g) throw Error{AB2_ERR_TIMEOUT, "local group: another rank gave up at a barrier"};
  }
};

struct LocalComm : ab2_comm {
  std::shared_ptr<LocalGroup> g;
  LocalGroup::Slot& me() { return g->slots[(size_t)rank]; }

  std::vector<std::vector<int>> host_allgather(const std::vector<int>& mine) override {
    me().host = mine;
    g->barrier();
    std::vector<std::vector<int>> all((size_t)size);
    for (int q = 0; q < size; ++q) all[(size_t)q] = g->slots[(size_t)q].host;
    g->barrier();  // nobody republishes before everybody has read
    return all;
  }

  // Every rank has to be in the same collective: a mismatch would read a
  // peer's buffers of another kind.
  void check_peers(int parity, char op) {
    for (int q = 0; q < size; ++q)
      require(g->slots[(size_t)q].op[parity] == op, "local group: ranks are in different collectives");
  }

  void before_publish(int parity) override {
    for (int q = 0; q < size; ++q)
      if (q != rank) AB2_CUDA(cudaStreamWaitEvent(ctx->stream, g->slots[(size_t)q].consumed[parity], 0));
  }

  void halo_start(const HaloPlan& plan, int parity, const double* sendbuf, double* ghosts) override {
    LocalGroup::Slot& s = me();
    s.send[parity] = sendbuf;
    s.plan[parity] = &plan;
    s.op[parity] = 'h';
    AB2_CUDA(cudaEventRecord(s.produced[parity], ctx->stream));
    g->barrier();
    check_peers(parity, 'h');
    // The ghost room is free once this rank's earlier work is done.
    AB2_CUDA(cudaStreamWaitEvent(cs, s.produced[parity], 0));
    for (size_t i = 0; i + 1 < plan.recv_off.size(); ++i) {
      const int q = plan.recv_ranks[i];
      const LocalGroup::Slot& ps = g->slots[(size_t)q];
      const HaloPlan& pp = *ps.plan[parity];
      size_t j = 0;
      while (j < pp.send_ranks.size() && pp.send_ranks[j] != rank) ++j;
      require(j < pp.send_ranks.size(), "local group: a neighbour does not send to this rank (inconsistent plans)");
      const int cnt = pp.send_off[j + 1] - pp.send_off[j];
      require(cnt == plan.recv_off[i + 1] - plan.recv_off[i], "local group: halo sizes disagree between ranks");
      AB2_CUDA(cudaStreamWaitEvent(cs, ps.produced[parity], 0));
      if (cnt > 0)
        AB2_CUDA(cudaMemcpyAsync(ghosts + plan.recv_off[i], ps.send[parity] + pp.send_off[j], sizeof(double) * cnt,
                                 cudaMemcpyDefault, cs));
    }
    AB2_CUDA(cudaEventRecord(s.consumed[parity], cs));
    AB2_CUDA(cudaEventRecord(ev_done, cs));
  }

  void allgather(int parity, const double* in, int k, double* out) override {
    LocalGroup::Slot& s = me();
    AB2_CUDA(cudaMemcpyAsync(s.pub[parity], in, sizeof(double) * k, cudaMemcpyDeviceToDevice, ctx->stream));
    s.op[parity] = 'g';
    AB2_CUDA(cudaEventRecord(s.produced[parity], ctx->stream));
    g->barrier();
    check_peers(parity, 'g');
    // out is this rank's buffer: the copies start after this rank's earlier
    // work, which includes the sum kernel that read out last time.
    AB2_CUDA(cudaStreamWaitEvent(cs, s.produced[parity], 0));
    for (int q = 0; q < size; ++q) {
      const LocalGroup::Slot& ps = g->slots[(size_t)q];
      AB2_CUDA(cudaStreamWaitEvent(cs, ps.produced[parity], 0));
      AB2_CUDA(cudaMemcpyAsync(out + (size_t)q * k, ps.pub[parity], sizeof(double) * k, cudaMemcpyDefault, cs));
    }
    AB2_CUDA(cudaEventRecord(s.consumed[parity], cs));
    AB2_CUDA(cudaEventRecord(ev_done, cs));
    AB2_CUDA(cudaStreamWaitEvent(ctx->stream, ev_done, 0));
  }

  ~LocalComm() override {
    LocalGroup::Slot& s = me();
    for (int p = 0; p < 2; ++p) {
      if (s.produced[p]) cudaEventDestroy(s.produced[p]);
      if (s.consumed[p]) cudaEventDestroy(s.consumed[p]);
      dev_free(ctx, s.pub[p]);
      s.produced[p] = s.consumed[p] = nullptr;
      s.pub[p] = nullptr;
    }
  }
};

// ------------------------------------------------------------------ NCCL
struct NcclApi {
  void* lib = nullptr;
  decltype(&ncclGetUniqueId) get_unique_id = nullptr;
  decltype(&ncclCommInitRank) comm_init_rank = nullptr;
  decltype(&ncclCommDestroy) comm_destroy = nullptr;
  decltype(&ncclSend) send = nullptr;
  decltype(&ncclRecv) recv = nullptr;
  decltype(&ncclGroupStart) group_start = nullptr;
  decltype(&ncclGroupEnd) group_end = nullptr;
  decltype(&ncclAllGather) all_gather = nullptr;
  decltype(&ncclGetErrorString) error_string = nullptr;
};

const NcclApi* nccl_api() {
  static const NcclApi api = [] {
    NcclApi a;
    a.lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    if (!a.lib) return a;
    bool ok = true;
    auto sym = [&](auto& fn, const char* name) {
      fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(a.lib, name));
      ok = ok && fn != nullptr;
    };
    sym(a.get_unique_id, "ncclGetUniqueId");
    sym(a.comm_init_rank, "ncclCommInitRank");
    sym(a.comm_destroy, "ncclCommDestroy");
    sym(a.send, "ncclSend");
    sym(a.recv, "ncclRecv");
    sym(a.group_start, "ncclGroupStart");
    sym(a.group_end, "ncclGroupEnd");
    sym(a.all_gather, "ncclAllGather");
    sym(a.error_string, "ncclGetErrorString");
    if (!ok) a.lib = nullptr;
    return a;
  }();
  return api.lib ? &api : nullptr;
}

void check_nccl(const NcclApi* api, ncclResult_t r, const char* what) {
  if (r != ncclSuccess) throw Error{AB2_ERR_CUDA, std::string(what) + ": " + api->error_string(r)};
}

struct NcclComm : ab2_comm {
  const NcclApi* api = nullptr;
  ncclComm_t comm = nullptr;

  std::vector<std::vector<int>> host_allgather(const std::vector<int>& mine) override {
    int* d_cnt = dev_alloc<int>(ctx, (size_t)size + 1);
    const int cnt = (int)mine.size();
    AB2_CUDA(cudaMemcpyAsync(d_cnt + size, &cnt, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    check_nccl(api, api->all_gather(d_cnt + size, d_cnt, 1, ncclInt32, comm, ctx->stream), "ncclAllGather");
    std::vector<int> cnts((size_t)size);
    AB2_CUDA(cudaMemcpyAsync(cnts.data(), d_cnt, sizeof(int) * size, cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    dev_free(ctx, d_cnt);
    const int mx = std::max(1, *std::max_element(cnts.begin(), cnts.end()));
    int* d_all = dev_alloc<int>(ctx, (size_t)mx * (size + 1));
    if (cnt) AB2_CUDA(cudaMemcpyAsync(d_all + (size_t)mx * size, mine.data(), sizeof(int) * cnt,
                                      cudaMemcpyHostToDevice, ctx->stream));
    check_nccl(api, api->all_gather(d_all + (size_t)mx * size, d_all, mx, ncclInt32, comm, ctx->stream),
               "ncclAllGather");
    std::vector<int> flat((size_t)mx * size);
    AB2_CUDA(cudaMemcpyAsync(flat.data(), d_all, sizeof(int) * flat.size(), cudaMemcpyDeviceToHost, ctx->stream));
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
    dev_free(ctx, d_all);
    std::vector<std::vector<int>> all((size_t)size);
    for (int q = 0; q < size; ++q) all[(size_t)q].assign(flat.begin() + (size_t)q * mx, flat.begin() + (size_t)q * mx + cnts[(size_t)q]);
    return all;
  }

  void halo_start(const HaloPlan& plan, int, const double* sendbuf, double* ghosts) override {
    AB2_CUDA(cudaEventRecord(ev_ready, ctx->stream));
    AB2_CUDA(cudaStreamWaitEvent(cs, ev_ready, 0));
    check_nccl(api, api->group_start(), "ncclGroupStart");
    for (size_t i = 0; i + 1 < plan.recv_off.size(); ++i)
      check_nccl(api, api->recv(ghosts + plan.recv_off[i], (size_t)(plan.recv_off[i + 1] - plan.recv_off[i]), ncclFloat64,
                                plan.recv_ranks[i], comm, cs), "ncclRecv");
    for (size_t j = 0; j + 1 < plan.send_off.size(); ++j)
      check_nccl(api, api->send(sendbuf + plan.send_off[j], (size_t)(plan.send_off[j + 1] - plan.send_off[j]), ncclFloat64,
                                plan.send_ranks[j], comm, cs), "ncclSend");
    check_nccl(api, api->group_end(), "ncclGroupEnd");
    AB2_CUDA(cudaEventRecord(ev_done, cs));
  }

  void allgather(int, const double* in, int k, double* out) override {
    check_nccl(api, api->all_gather(in, out, (size_t)k, ncclFloat64, comm, ctx->stream), "ncclAllGather");
  }

  ~NcclComm() override {
    if (comm && api) api->comm_destroy(comm);
  }
};

// Stream, events and buffers every communicator owns on its context.
void comm_attach(ab2_comm* c, ab2_context* ctx) {
  c->ctx = ctx_retain(ctx);
  AB2_CUDA(cudaSetDevice(ctx->device));
  AB2_CUDA(cudaStreamCreateWithFlags(&c->cs, cudaStreamNonBlocking));
  AB2_CUDA(cudaEventCreateWithFlags(&c->ev_ready, cudaEventDisableTiming));
  AB2_CUDA(cudaEventCreateWithFlags(&c->ev_done, cudaEventDisableTiming));
  c->d_gather = dev_alloc<double>(ctx, (size_t)c->size * kMaxRedComps);
  c->d_sum = dev_alloc<double>(ctx, kMaxRedComps);
}

// ------------------------------------------------------------------ kernels
__global__ void k_gather_rows(int m, const int* __restrict__ ids, const double* __restrict__ x, double* __restrict__ out) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) out[t] = x[ids[t]];
}

// y_i += sum of the ghost entries of interface row i (SimpleCSRMatrixMultT.h:117-127:
// tmpy starts at 0 and accumulates a*x, rounded apart, then y += tmpy).
__global__ void k_ghost_rows(int m, const int* __restrict__ rows, const int* __restrict__ gp,
                             const int* __restrict__ gc, const double* __restrict__ gv,
                             const double* __restrict__ xg, double* __restrict__ y) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = gp[t]; k < gp[t + 1]; ++k) s = mul_add_rn(gv[k], xg[gc[k]], s);
    const int i = rows[t];
    y[i] = add_rn(y[i], s);
  }
}

// out[j] = all[j] + all[k + j] + ... + all[(size-1) k + j], left to right.
__global__ void k_rank_sum(int size, int k, const double* __restrict__ all, double* __restrict__ out) {
  const int j = threadIdx.x;
  if (j >= k) return;
  double s = all[j];
  for (int r = 1; r < size; ++r) s = add_rn(s, all[(size_t)r * k + j]);
  out[j] = s;
}

// One wavefront of the parallel block-Jacobi factorisation
// (ILU0Preconditioner.h:93-119) on the rank's rows in the distributed layout:
// for each local k left of the diagonal, a_ik /= a_kk, then for positions j
// of row i from k+1 up to (not including) kcol[krow] + local_row_size[i] --
// the reference's bound -- a_ij -= a_ik a_kj where column j is a local column
// of row krow (the reference marks only those in m_work).
__global__ void k_bj_factor_level(const int* __restrict__ rows, int count, const int* __restrict__ rp,
                                  const int* __restrict__ ci, const int* __restrict__ dcol,
                                  const int* __restrict__ lrs, long long nnz, double* __restrict__ lu) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const int i = rows[t];
  const int di = dcol[i];
  for (int k = rp[i]; k < di; ++k) {
    const int kr = ci[k];
    const int dk = dcol[kr];
    const double piv = dk < nnz ? lu[dk] : 0.0;
    const double aik = lu[k] / piv;
    lu[k] = aik;
    int l = rp[kr];
    const int le = rp[kr] + lrs[kr];
    const int bound = rp[kr] + lrs[i];
    for (int j = k + 1; j < bound; ++j) {
      const int cj = ci[j];
      while (l < le && ci[l] < cj) ++l;
      if (l == le) break;
      if (ci[l] == cj) lu[j] = mul_sub_rn(aik, lu[l], lu[j]);
    }
  }
}

// The local parts of the rows (the diagonal block's CSR order).
__global__ void k_bj_extract(int n, const int* __restrict__ rp, const int* __restrict__ lrs,
                             const int* __restrict__ rp_loc, const double* __restrict__ lu, double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int p = 0; p < lrs[i]; ++p) out[rp_loc[i] + p] = lu[rp[i] + p];
}

}  // namespace
}  // namespace ab2

namespace ab2 {
namespace {

int owner_of(const std::vector<int>& offsets, int col) {
  // last r with offsets[r] <= col (offsets ascending, size+1 entries)
  return (int)(std::upper_bound(offsets.begin(), offsets.end() - 1, col) - offsets.begin()) - 1;
}

void dist_build(ab2_dist_matrix* A, const int* row_ptr, const int* cols, const double* vals, int formats) {
  ab2_context* ctx = A->ctx;
  ab2_comm* comm = A->comm;
  const int me = comm->rank, np = comm->size;
  const std::vector<int>& off = A->offsets;
  const int n = A->n_loc;
  const int base = off[(size_t)me];
  // Every rank reaches the exchange below, valid rows or not, so that a
  // rejection on one rank fails the call on all of them instead of leaving
  // the others waiting in the collective.
  std::string bad;
  if (row_ptr[0] != 0) bad = "row_ptr must start at 0";
  for (int i = 0; bad.empty() && i < n; ++i) {
    const int b = row_ptr[i], e = row_ptr[i + 1];
    if (b > e) bad = "row_ptr must be non-decreasing";
    else if (e > b && (!cols || !vals)) bad = "null cols or vals";
    for (int k = b; bad.empty() && k < e; ++k) {
      if (cols[k] < 0 || cols[k] >= A->global_n) bad = "column index out of range";
      else if (k > b && cols[k - 1] >= cols[k]) bad = "columns must be strictly ascending inside each row";
    }
  }
  if (!bad.empty()) {
    comm->host_allgather(std::vector<int>{1});
    throw Error{AB2_ERR_BAD_ARG, bad};
  }
  const long long nnz = row_ptr[n];
  // sortGhostCols: local columns first, ghosts after, each in their order
  A->h_rp.assign(row_ptr, row_ptr + n + 1);
  A->h_ci.resize((size_t)nnz);
  A->h_v.resize((size_t)nnz);
  A->h_lrs.assign((size_t)n, 0);
  std::vector<std::vector<int>> gids((size_t)np);
  std::vector<int> g_owner;  // per position: owner rank of a ghost column, -1 if local
  g_owner.assign((size_t)nnz, -1);
  for (int i = 0; i < n; ++i) {
    const int b = row_ptr[i], e = row_ptr[i + 1];
    int nl = 0;
    for (int k = b; k < e; ++k) {
      const int c = cols[k];
      if (c >= base && c < base + n) ++nl;
    }
    A->h_lrs[(size_t)i] = nl;
    int pl = b, pg = b + nl;
    for (int k = b; k < e; ++k) {
      const int c = cols[k];
      if (c >= base && c < base + n) {
        A->h_ci[(size_t)pl] = c - base;
        A->h_v[(size_t)pl++] = vals[k];
      } else {
        const int q = owner_of(off, c);
        g_owner[(size_t)pg] = q;
        A->h_ci[(size_t)pg] = c;  // global id until the ghosts are numbered
        A->h_v[(size_t)pg++] = vals[k];
        gids[(size_t)q].push_back(c);
      }
    }
  }
  // ghost numbering: by owner rank, ascending global id inside each owner
  std::vector<int> col_offset((size_t)np + 1, 0);
  for (int q = 0; q < np; ++q) {
    std::vector<int>& v = gids[(size_t)q];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    col_offset[(size_t)q + 1] = col_offset[(size_t)q] + (int)v.size();
  }
  A->n_ghost = col_offset[(size_t)np];
  A->h_ghost_uids.clear();
  for (int q = 0; q < np; ++q) A->h_ghost_uids.insert(A->h_ghost_uids.end(), gids[(size_t)q].begin(), gids[(size_t)q].end());
  for (long long k = 0; k < nnz; ++k) {
    const int q = g_owner[(size_t)k];
    if (q < 0) continue;
    const std::vector<int>& v = gids[(size_t)q];
    const int lid = (int)(std::lower_bound(v.begin(), v.end(), A->h_ci[(size_t)k]) - v.begin());
    A->h_ci[(size_t)k] = n + col_offset[(size_t)q] + lid;
  }
  // interface rows and their ghost entries
  A->h_iface.clear();
  std::vector<int> gp(1, 0), gc;
  std::vector<double> gv;
  for (int i = 0; i < n; ++i) {
    const int b = A->h_rp[(size_t)i] + A->h_lrs[(size_t)i], e = A->h_rp[(size_t)i + 1];
    if (b == e) continue;
    A->h_iface.push_back(i);
    for (int k = b; k < e; ++k) {
      gc.push_back(A->h_ci[(size_t)k] - n);
      gv.push_back(A->h_v[(size_t)k]);
    }
    gp.push_back((int)gc.size());
  }
  A->n_iface = (int)A->h_iface.size();
  A->ghost_nnz = (long long)gc.size();
  // receive plan and m_first_upper_ghost_index
  HaloPlan& P = A->plan;
  P.recv_ranks.clear();
  P.recv_off.assign(1, 0);
  int first_upper = 0;
  for (int q = 0; q < np; ++q)
    if (!gids[(size_t)q].empty()) {
      if (q < me) ++first_upper;
      P.recv_ranks.push_back(q);
      P.recv_off.push_back(P.recv_off.back() + (int)gids[(size_t)q].size());
    }
  A->first_upper_ghost = n + P.recv_off[(size_t)first_upper];
  // requests: status 0, then (owner, count, ids...) for every owner this rank needs values from
  std::vector<int> req(1, 0);
  for (int q = 0; q < np; ++q)
    if (!gids[(size_t)q].empty()) {
      req.push_back(q);
      req.push_back((int)gids[(size_t)q].size());
      req.insert(req.end(), gids[(size_t)q].begin(), gids[(size_t)q].end());
    }
  const std::vector<std::vector<int>> all = comm->host_allgather(req);
  for (int q = 0; q < np; ++q)
    if (all[(size_t)q].empty() || all[(size_t)q][0] != 0)
      throw Error{AB2_ERR_BAD_ARG, "rank " + std::to_string(q) + " rejected its rows"};
  P.send_ranks.clear();
  P.send_off.assign(1, 0);
  A->h_send_ids.clear();
  for (int q = 0; q < np; ++q) {
    const std::vector<int>& r = all[(size_t)q];
    for (size_t t = 1; t + 1 < r.size();) {
      const int owner = r[t], cnt = r[t + 1];
      require(cnt >= 0 && t + 2 + (size_t)cnt <= r.size(), "malformed ghost request");
      if (owner == me && q != me) {
        P.send_ranks.push_back(q);
        for (int u = 0; u < cnt; ++u) {
          const int id = r[t + 2 + (size_t)u] - base;
          require(id >= 0 && id < n, "a rank asked for a row this rank does not own (inconsistent offsets)");
          A->h_send_ids.push_back(id);
        }
        P.send_off.push_back((int)A->h_send_ids.size());
      }
      t += 2 + (size_t)cnt;
    }
  }
  A->n_send = (int)A->h_send_ids.size();
  // the diagonal block
  std::vector<int> rp_loc((size_t)n + 1, 0), ci_loc;
  std::vector<double> v_loc;
  ci_loc.reserve((size_t)nnz);
  v_loc.reserve((size_t)nnz);
  for (int i = 0; i < n; ++i) {
    for (int p = 0; p < A->h_lrs[(size_t)i]; ++p) {
      ci_loc.push_back(A->h_ci[(size_t)A->h_rp[(size_t)i] + p]);
      v_loc.push_back(A->h_v[(size_t)A->h_rp[(size_t)i] + p]);
    }
    rp_loc[(size_t)i + 1] = (int)ci_loc.size();
  }
  const int rc = ab2_matrix_create_csr(ctx, n, rp_loc.data(), ci_loc.data(), v_loc.data(), formats, &A->local);
  if (rc != AB2_OK) throw Error{rc, "local block: " + ctx->last_error};
  // device exchange and interface arrays
  A->d_send_ids = dev_alloc<int>(ctx, (size_t)A->n_send);
  A->d_send[0] = dev_alloc<double>(ctx, (size_t)A->n_send);
  A->d_send[1] = dev_alloc<double>(ctx, (size_t)A->n_send);
  A->d_iface = dev_alloc<int>(ctx, (size_t)A->n_iface);
  A->d_gp = dev_alloc<int>(ctx, gp.size());
  A->d_gc = dev_alloc<int>(ctx, gc.size());
  A->d_gv = dev_alloc<double>(ctx, gv.size());
  if (A->n_send)
    AB2_CUDA(cudaMemcpy(A->d_send_ids, A->h_send_ids.data(), sizeof(int) * A->n_send, cudaMemcpyHostToDevice));
  if (A->n_iface) AB2_CUDA(cudaMemcpy(A->d_iface, A->h_iface.data(), sizeof(int) * A->n_iface, cudaMemcpyHostToDevice));
  AB2_CUDA(cudaMemcpy(A->d_gp, gp.data(), sizeof(int) * gp.size(), cudaMemcpyHostToDevice));
  if (!gc.empty()) {
    AB2_CUDA(cudaMemcpy(A->d_gc, gc.data(), sizeof(int) * gc.size(), cudaMemcpyHostToDevice));
    AB2_CUDA(cudaMemcpy(A->d_gv, gv.data(), sizeof(double) * gv.size(), cudaMemcpyHostToDevice));
  }
}

void dist_free(ab2_dist_matrix* A) {
  ab2_context* ctx = A->ctx;
  if (ctx) {
    ctx_quiesce(ctx);
    for (void* p : {(void*)A->d_send_ids, (void*)A->d_send[0], (void*)A->d_send[1], (void*)A->d_iface, (void*)A->d_gp,
                    (void*)A->d_gc, (void*)A->d_gv})
      dev_free(ctx, p);
  }
  if (A->local) ab2_matrix_destroy(A->local);
  if (ctx) ctx_release(ctx);
  delete A;
}

}  // namespace

// y = A x on the rank's rows; x->d must have room for the ghosts.
void dist_mult(ab2_context* ctx, const ab2_dist_matrix* A, double* x, double* y) {
  ab2_comm* c = A->comm;
  const int p = c->next();
  if (A->n_send) {
    k_gather_rows<<<grid_for(A->n_send), kThreads, 0, ctx->stream>>>(A->n_send, A->d_send_ids, x, A->d_send[p]);
    check_launch(ctx, "dist_pack");
  }
  c->halo_start(A->plan, p, A->d_send[p], x + A->n_loc);
  op_spmv(ctx, A->local, x, y, AB2_SPMV_AUTO);
  c->halo_finish();
  if (A->n_iface) {
    k_ghost_rows<<<grid_for(A->n_iface), kThreads, 0, ctx->stream>>>(A->n_iface, A->d_iface, A->d_gp, A->d_gc, A->d_gv,
                                                                     x + A->n_loc, y);
    check_launch(ctx, "dist_ghost_rows");
  }
}

// out[0..k) = rank-ordered sums of every rank's in[0..k) (device, ctx->stream).
void dist_sum(ab2_context* ctx, ab2_comm* c, const double* in, int k, double* out) {
  const int p = c->next();
  c->allgather(p, in, k, c->d_gather);
  k_rank_sum<<<1, 32, 0, ctx->stream>>>(c->size, k, c->d_gather, out);
  check_launch(ctx, "dist_rank_sum");
}

}  // namespace ab2

using namespace ab2;

extern "C" {

int ab2_comm_local_group(ab2_context** ctxs, int size, double timeout_s, ab2_comm** comms) {
  if (!ctxs || !comms || size < 1 || !(timeout_s > 0)) return AB2_ERR_BAD_ARG;
  for (int r = 0; r < size; ++r) {
    if (!ctxs[r]) return AB2_ERR_BAD_ARG;
    comms[r] = nullptr;
  }
  auto g = std::make_shared<LocalGroup>();
  g->size = size;
  g->timeout_s = timeout_s;
  g->slots.resize((size_t)size);
  for (int r = 0; r < size; ++r) {
    LocalComm* c = new (std::nothrow) LocalComm();
    if (!c) return AB2_ERR_OOM;
    c->rank = r;
    c->size = size;
    c->g = g;
    const int rc = guard(ctxs[r], [&] {
      comm_attach(c, ctxs[r]);
      LocalGroup::Slot& s = c->me();
      for (int p = 0; p < 2; ++p) {
        AB2_CUDA(cudaEventCreateWithFlags(&s.produced[p], cudaEventDisableTiming));
        AB2_CUDA(cudaEventCreateWithFlags(&s.consumed[p], cudaEventDisableTiming));
        s.pub[p] = dev_alloc<double>(c->ctx, kMaxRedComps);
      }
    });
    comms[r] = c;
    if (rc != AB2_OK) {
      for (int q = 0; q <= r; ++q) {
        ab2_comm_destroy(comms[q]);
        comms[q] = nullptr;
      }
      return rc;
    }
  }
  return AB2_OK;
}

int ab2_comm_nccl_unique_id(unsigned char id[AB2_COMM_ID_BYTES]) {
  static_assert(sizeof(ncclUniqueId) == AB2_COMM_ID_BYTES, "ncclUniqueId size");
  if (!id) return AB2_ERR_BAD_ARG;
  const NcclApi* api = nccl_api();
  if (!api) return AB2_ERR_UNSUPPORTED;
  ncclUniqueId u;
  if (api->get_unique_id(&u) != ncclSuccess) return AB2_ERR_CUDA;
  std::memcpy(id, &u, sizeof(u));
  return AB2_OK;
}

int ab2_comm_nccl_create(ab2_context* ctx, const unsigned char id[AB2_COMM_ID_BYTES], int rank, int size,
                         ab2_comm** out) {
  if (!ctx || !id || !out || size < 1 || rank < 0 || rank >= size) return AB2_ERR_BAD_ARG;
  *out = nullptr;
  const NcclApi* api = nccl_api();
  if (!api) {
    ctx->last_error = "libnccl.so.2 could not be loaded";
    return AB2_ERR_UNSUPPORTED;
  }
  NcclComm* c = new (std::nothrow) NcclComm();
  if (!c) return AB2_ERR_OOM;
  c->api = api;
  c->rank = rank;
  c->size = size;
  const int rc = guard(ctx, [&] {
    comm_attach(c, ctx);
    ncclUniqueId u;
    std::memcpy(&u, id, sizeof(u));
    check_nccl(api, api->comm_init_rank(&c->comm, size, u, rank), "ncclCommInitRank");
  });
  if (rc != AB2_OK) {
    ab2_comm_destroy(c);
    return rc;
  }
  *out = c;
  return AB2_OK;
}

int ab2_comm_rank(const ab2_comm* c, int* rank) {
  if (!c || !rank) return AB2_ERR_BAD_ARG;
  *rank = c->rank;
  return AB2_OK;
}

int ab2_comm_size(const ab2_comm* c, int* size) {
  if (!c || !size) return AB2_ERR_BAD_ARG;
  *size = c->size;
  return AB2_OK;
}

int ab2_comm_destroy(ab2_comm* c) {
  if (!c) return AB2_ERR_BAD_ARG;
  ab2_context* ctx = c->ctx;
  cudaStream_t cs = c->cs;
  if (ctx) {
    ctx_quiesce(ctx);
    if (cs) cudaStreamSynchronize(cs);
    dev_free(ctx, c->d_gather);
    dev_free(ctx, c->d_sum);
  }
  if (c->ev_ready) cudaEventDestroy(c->ev_ready);
  if (c->ev_done) cudaEventDestroy(c->ev_done);
  delete c;  // a local-group rank frees its slot's events and buffers on its (still held) context
  if (cs) cudaStreamDestroy(cs);
  if (ctx) ctx_release(ctx);
  return AB2_OK;
}

int ab2_dist_matrix_create(ab2_context* ctx, ab2_comm* comm, const int* offsets, const int* row_ptr, const int* cols,
                           const double* vals, int formats, ab2_dist_matrix** out) {
  if (!ctx || !comm || !offsets || !row_ptr || !out || comm->ctx != ctx) return AB2_ERR_BAD_ARG;
  *out = nullptr;
  const int np = comm->size;
  for (int q = 0; q < np; ++q)
    if (offsets[q] > offsets[q + 1] || offsets[0] != 0) {
      ctx->last_error = "offsets must start at 0 and be non-decreasing";
      return AB2_ERR_BAD_ARG;
    }
  ab2_dist_matrix* A = new (std::nothrow) ab2_dist_matrix();
  if (!A) return AB2_ERR_OOM;
  A->ctx = ctx_retain(ctx);
  A->comm = comm;
  A->offsets.assign(offsets, offsets + np + 1);
  A->global_n = offsets[np];
  A->n_loc = offsets[comm->rank + 1] - offsets[comm->rank];
  const int rc = guard(ctx, [&] { dist_build(A, row_ptr, cols, vals, formats); });
  if (rc != AB2_OK) {
    dist_free(A);
    return rc;
  }
  *out = A;
  return AB2_OK;
}

int ab2_dist_matrix_get_info(const ab2_dist_matrix* A, ab2_dist_info* info) {
  if (!A || !info) return AB2_ERR_BAD_ARG;
  info->global_rows = A->global_n;
  info->local_rows = A->n_loc;
  info->ghost_rows = A->n_ghost;
  info->interface_rows = A->n_iface;
  info->recv_neighbours = (int)A->plan.recv_ranks.size();
  info->send_neighbours = (int)A->plan.send_ranks.size();
  info->send_count = A->n_send;
  info->first_upper_ghost_index = A->first_upper_ghost;
  info->ghost_nnz = A->ghost_nnz;
  info->local_nnz = (long long)A->h_ci.size() - A->ghost_nnz;
  return AB2_OK;
}

int ab2_dist_matrix_layout(const ab2_dist_matrix* A, int* row_ptr, int* cols, double* vals, int* lrs, int* ghost_uids,
                           int* iface) {
  if (!A) return AB2_ERR_BAD_ARG;
  if (row_ptr) std::copy(A->h_rp.begin(), A->h_rp.end(), row_ptr);
  if (cols) std::copy(A->h_ci.begin(), A->h_ci.end(), cols);
  if (vals) std::copy(A->h_v.begin(), A->h_v.end(), vals);
  if (lrs) std::copy(A->h_lrs.begin(), A->h_lrs.end(), lrs);
  if (ghost_uids) std::copy(A->h_ghost_uids.begin(), A->h_ghost_uids.end(), ghost_uids);
  if (iface) std::copy(A->h_iface.begin(), A->h_iface.end(), iface);
  return AB2_OK;
}

int ab2_dist_matrix_plan(const ab2_dist_matrix* A, int* recv_ranks, int* recv_offsets, int* send_ranks,
                         int* send_offsets, int* send_ids) {
  if (!A) return AB2_ERR_BAD_ARG;
  const HaloPlan& P = A->plan;
  if (recv_ranks) std::copy(P.recv_ranks.begin(), P.recv_ranks.end(), recv_ranks);
  if (recv_offsets) std::copy(P.recv_off.begin(), P.recv_off.end(), recv_offsets);
  if (send_ranks) std::copy(P.send_ranks.begin(), P.send_ranks.end(), send_ranks);
  if (send_offsets) std::copy(P.send_off.begin(), P.send_off.end(), send_offsets);
  if (send_ids) std::copy(A->h_send_ids.begin(), A->h_send_ids.end(), send_ids);
  return AB2_OK;
}

int ab2_dist_matrix_local(const ab2_dist_matrix* A, const ab2_matrix** local) {
  if (!A || !local) return AB2_ERR_BAD_ARG;
  *local = A->local;
  return AB2_OK;
}

int ab2_dist_matrix_destroy(ab2_dist_matrix* A) {
  if (!A) return AB2_ERR_BAD_ARG;
  dist_free(A);
  return AB2_OK;
}

int ab2_dist_vector_create(ab2_context* ctx, const ab2_dist_matrix* A, ab2_vector** out) {
  if (!ctx || !A || !out) return AB2_ERR_BAD_ARG;
  const int rc = ab2_vector_create(ctx, A->n_loc + A->n_ghost, out);
  if (rc != AB2_OK) return rc;
  (*out)->n = A->n_loc;  // the ghost room stays outside every other operation
  return AB2_OK;
}

int ab2_dist_mult(ab2_context* ctx, const ab2_dist_matrix* A, ab2_vector* x, ab2_vector* y) {
  if (!ctx || !A || !x || !y || x == y || x->n != A->n_loc || y->n != A->n_loc) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "DIST-SPMV");
  if (x->cap < A->n_loc + A->n_ghost) {
    ctx->last_error = "ab2_dist_mult: x has no room for the ghost values (create it with ab2_dist_vector_create)";
    return AB2_ERR_BAD_ARG;
  }
  return guard(ctx, [&] { dist_mult(ctx, A, x->d, y->d); });
}

}  // extern "C"

namespace {
template <class F>
int dist_scalar(ab2_context* ctx, ab2_comm* c, const ab2_vector* x, double* result, F&& local, bool root) {
  if (!ctx || !c || !x || !result || c->ctx != ctx) return AB2_ERR_BAD_ARG;
  return guard(ctx, [&] {
    RedSlot s = red_slot(ctx, 0);
    local(s.result);
    dist_sum(ctx, c, s.result, 1, c->d_sum);
    const double v = read_scalar(ctx, c->d_sum);
    *result = root ? std::sqrt(v) : v;
  });
}
}  // namespace

extern "C" {

int ab2_dist_dot(ab2_context* ctx, ab2_comm* c, const ab2_vector* x, const ab2_vector* y, double* result) {
  if (!y || !x || x->n != y->n) return AB2_ERR_BAD_ARG;
  PhaseScope phase_scope(ctx, "DIST-DOT");
  return dist_scalar(ctx, c, x, result, [&](double* out) { op_dot(ctx, x->n, x->d, y->d, out, 0); }, false);
}

int ab2_dist_norm1(ab2_context* ctx, ab2_comm* c, const ab2_vector* x, double* result) {
  PhaseScope phase_scope(ctx, "DIST-NORM1");
  return dist_scalar(ctx, c, x, result, [&](double* out) { op_norm1(ctx, x->n, x->d, out, 0); }, false);
}

int ab2_dist_norm2(ab2_context* ctx, ab2_comm* c, const ab2_vector* x, double* result) {
  PhaseScope phase_scope(ctx, "DIST-NORM2");
  return dist_scalar(ctx, c, x, result, [&](double* out) { op_dot(ctx, x->n, x->d, x->d, out, 0); }, true);
}

}  // extern "C"

namespace ab2 {

// Block-Jacobi ILU(0) factor of the rank's rows, in the diagonal block's CSR
// order (device, local_nnz doubles; the caller frees it).
double* dist_bj_factor(ab2_context* ctx, const ab2_dist_matrix* A) {
  const int n = A->n_loc;
  const std::vector<int>& rp = A->h_rp;
  const std::vector<int>& ci = A->h_ci;
  const std::vector<int>& lrs = A->h_lrs;
  const long long nnz = (long long)ci.size();
  // DistStructInfo::computeUpperDiagOffset: first local position with col >= row
  std::vector<int> dc((size_t)n);
  for (int i = 0; i < n; ++i) {
    int idx = rp[(size_t)i];
    for (int k = rp[(size_t)i]; k < rp[(size_t)i] + lrs[(size_t)i] && ci[(size_t)k] < i; ++k) ++idx;
    dc[(size_t)i] = idx;
  }
  // wavefronts of the local lower structure
  std::vector<int> lev((size_t)n, 0);
  int nlev = n > 0 ? 1 : 0;
  for (int i = 0; i < n; ++i) {
    int l = 0;
    for (int k = rp[(size_t)i]; k < dc[(size_t)i]; ++k) l = std::max(l, lev[(size_t)ci[(size_t)k]] + 1);
    lev[(size_t)i] = l;
    nlev = std::max(nlev, l + 1);
  }
  std::vector<int> cnt((size_t)nlev + 1, 0), perm((size_t)n);
  for (int i = 0; i < n; ++i) cnt[(size_t)lev[(size_t)i] + 1]++;
  for (int l = 0; l < nlev; ++l) cnt[(size_t)l + 1] += cnt[(size_t)l];
  std::vector<int> fill(cnt.begin(), cnt.end() - 1);
  for (int i = 0; i < n; ++i) perm[(size_t)fill[(size_t)lev[(size_t)i]]++] = i;

  int* d_rp = dev_alloc<int>(ctx, (size_t)n + 1);
  int* d_ci = dev_alloc<int>(ctx, (size_t)nnz);
  int* d_dc = dev_alloc<int>(ctx, (size_t)n);
  int* d_lrs = dev_alloc<int>(ctx, (size_t)n);
  int* d_perm = dev_alloc<int>(ctx, (size_t)n);
  double* d_lu = dev_alloc<double>(ctx, (size_t)nnz);
  double* d_out = dev_alloc<double>(ctx, (size_t)A->local->nnz);
  AB2_CUDA(cudaMemcpy(d_rp, rp.data(), sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice));
  if (nnz) {
    AB2_CUDA(cudaMemcpy(d_ci, ci.data(), sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice));
    AB2_CUDA(cudaMemcpy(d_lu, A->h_v.data(), sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice));
  }
  if (n) {
    AB2_CUDA(cudaMemcpy(d_dc, dc.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
    AB2_CUDA(cudaMemcpy(d_lrs, lrs.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
    AB2_CUDA(cudaMemcpy(d_perm, perm.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
  }
  for (int l = 1; l < nlev; ++l) {  // wavefront 0 has nothing left of the diagonal
    const int a = cnt[(size_t)l], b = cnt[(size_t)l + 1];
    if (b == a) continue;
    k_bj_factor_level<<<(b - a + 127) / 128, 128, 0, ctx->stream>>>(d_perm + a, b - a, d_rp, d_ci, d_dc, d_lrs, nnz,
                                                                    d_lu);
    check_launch(ctx, "dist_bj_factor");
  }
  if (n) {
    k_bj_extract<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, d_rp, d_lrs, A->local->d_rp, d_lu, d_out);
    check_launch(ctx, "dist_bj_extract");
  }
  AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  for (void* p : {(void*)d_rp, (void*)d_ci, (void*)d_dc, (void*)d_lrs, (void*)d_perm, (void*)d_lu}) dev_free(ctx, p);
  return d_out;
}

}  // namespace ab2

extern "C" int ab2_dist_precond_create(ab2_context* ctx, const ab2_dist_matrix* A, const ab2_precond_options* o,
                                       ab2_precond** out) {
  if (!ctx || !A || !o || !out) return AB2_ERR_BAD_ARG;
  *out = nullptr;
  // One rank: the matrix is not parallel (m_is_parallel = nproc > 1) and
  // ILU(0) is the sequential factorisation of the whole (local) matrix.
  if (o->kind == AB2_PC_NONE || o->kind == AB2_PC_DIAG || (o->kind == AB2_PC_ILU0 && A->comm->size == 1))
    return ab2_precond_create(ctx, A->local, o, out);
  if (o->kind != AB2_PC_ILU0) {
    ctx->last_error = "distributed preconditioners: NONE, DIAG and ILU0 (block Jacobi)";
    return AB2_ERR_UNSUPPORTED;
  }
  if (o->ilu_schedule < AB2_ILU_AUTO || o->ilu_schedule > AB2_ILU_STENCIL_CLUSTER) return AB2_ERR_BAD_ARG;
  ab2_precond* pc = new (std::nothrow) ab2_precond();
  if (!pc) return AB2_ERR_OOM;
  pc->ctx = ctx_retain(ctx);
  pc->A = A->local;
  pc->kind = AB2_PC_ILU0;
  double* lu = nullptr;
  const int rc = guard(ctx, [&] {
    lu = dist_bj_factor(ctx, A);
    ilu_init(ctx, pc, o->ilu_schedule, lu);
    AB2_CUDA(cudaStreamSynchronize(ctx->stream));
  });
  dev_free(ctx, lu);
  if (rc != AB2_OK) {
    ab2_precond_destroy(pc);
    return rc;
  }
  *out = pc;
  return AB2_OK;
}
