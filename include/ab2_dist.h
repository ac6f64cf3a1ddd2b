/*
 * ab2_dist.h -- row-block distribution of libab2's algebra over several ranks
 * (one rank per GPU, or several ranks on one GPU inside one process).
 *
 * Alien distributes a matrix by contiguous blocks of rows, one block per
 * rank, and runs the same Krylov templates on every rank with a parallel
 * algebra: the SpMV exchanges the ghost values its rows need, dot products
 * are summed over the ranks, and ILU(0) becomes block-Jacobi ILU(0) over each
 * rank's diagonal block.  This header is that algebra on libab2:
 *
 *   reference                                         here
 *   DistStructInfo::compute (kernels/simple_csr/       ab2_dist_matrix_create (collective)
 *     DistStructInfo.cc:44-233), sortGhostCols
 *     (SimpleCSRMatrix.h:215-258), MatrixProfilerT::
 *     computeProfile (handlers/profiler/
 *     MatrixProfilerT.h:131-190)
 *   SimpleCSRMatrixMultT::_parallelMult                ab2_dist_mult
 *     (algebra/SimpleCSRMatrixMultT.h:85-128) with
 *     SendRecvOp (SendRecvOp.h)
 *   CBLASMPIKernel::dot / nrm1 / nrm2                  ab2_dist_dot / ab2_dist_norm1 / ab2_dist_norm2
 *     (algebra/CBLASMPIKernel.h:85-125): local BLAS
 *     then mpAllReduce(ReduceSum)
 *   LUFactorisationAlgo::factorize + solveL/solveU     ab2_dist_precond_create (AB2_PC_ILU0)
 *     parallel branches (expression/krylov/
 *     ILU0Preconditioner.h:93-119,181-231)
 *   IMessagePassingMng (Arccore)                       ab2_comm
 *
 * Layout (as the reference's): a rank owns global rows [offsets[r],
 * offsets[r+1]).  Inside each row its local columns come first, ascending,
 * then its ghost columns, ascending.  Local columns are numbered 0..n_local-1
 * (global id - offsets[r]); ghost columns n_local.. in ascending global order
 * (grouped by owning rank, ascending).  A distributed vector holds the rank's
 * n_local values followed by room for the ghost values the SpMV receives.
 *
 * Results: the SpMV sums a row's local entries, then adds the sum of its
 * ghost entries (two roundings, as _parallelMult); a distributed dot is each
 * rank's libab2 dot of its local part, summed over the ranks in rank order
 * (p_0 + p_1 + ... left to right, identical on every rank: MPI leaves the
 * order of its sum open, this fixes one).  Block-Jacobi ILU(0) reproduces
 * the reference's parallel factorisation exactly, including the loop bound
 * of ILU0Preconditioner.h:107, which limits the elimination of row i by row
 * k to positions below kcol[k] + local_row_size[i]: on stencil matrices the
 * bound leaves only the divisions a_ik / a_kk (no diagonal updates).  With a
 * single rank the reference's matrix is not parallel (m_is_parallel is
 * nproc > 1) and ILU(0) is the sequential factorisation; so it is here.
 *
 * Collectives: ab2_dist_matrix_create, ab2_dist_mult, ab2_dist_dot,
 * ab2_dist_norm*, ab2_dist_precond_create (ILU0) and ab2_dist_solver_solve
 * must be called by every rank of the communicator, in the same order.
 */
#ifndef AB2_DIST_H
#define AB2_DIST_H

#include "ab2.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ab2_comm ab2_comm;
typedef struct ab2_dist_matrix ab2_dist_matrix;
typedef struct ab2_dist_solver ab2_dist_solver;

/* ------------------------------------------------------------------ communicators
 * Local group: `size` ranks inside this process, rank r bound to ctxs[r] (any
 * devices) and driven by its own host thread.  Ranks meet at host barriers
 * (which give up with AB2_ERR_TIMEOUT after timeout_s seconds) and move
 * data with device-to-device copies ordered by CUDA events; no kernel ever
 * waits for another rank.  comms receives one handle per rank. */
int ab2_comm_local_group(ab2_context** ctxs, int size, double timeout_s, ab2_comm** comms);
/* NCCL: one rank per process (or thread), the library loaded at run time
 * (libnccl.so.2; AB2_ERR_UNSUPPORTED when absent).  Rank 0 makes the id and
 * hands it to the others out of band (as ncclGetUniqueId / ncclCommInitRank). */
#define AB2_COMM_ID_BYTES 128
int ab2_comm_nccl_unique_id(unsigned char id[AB2_COMM_ID_BYTES]);
int ab2_comm_nccl_create(ab2_context* ctx, const unsigned char id[AB2_COMM_ID_BYTES], int rank, int size,
                         ab2_comm** comm);
int ab2_comm_rank(const ab2_comm* comm, int* rank);
int ab2_comm_size(const ab2_comm* comm, int* size);
int ab2_comm_destroy(ab2_comm* comm);

/* ------------------------------------------------------------------ distributed matrix
 * Collective.  offsets: size+1 global row offsets (the same on every rank);
 * row_ptr/cols/vals: this rank's rows, columns in GLOBAL numbering, ascending
 * inside each row; formats as ab2_matrix_create_csr (for the local block). */
int ab2_dist_matrix_create(ab2_context* ctx, ab2_comm* comm, const int* offsets, const int* row_ptr, const int* cols,
                           const double* vals, int formats, ab2_dist_matrix** A);
typedef struct {
  int global_rows;
  int local_rows;
  int ghost_rows;             /* DistStructInfo::m_ghost_nrow */
  int interface_rows;         /* m_interface_nrow: rows with at least one ghost column */
  int recv_neighbours;        /* ranks this one receives ghost values from */
  int send_neighbours;        /* ranks this one sends values to */
  int send_count;             /* values sent per SpMV */
  int first_upper_ghost_index;/* m_first_upper_ghost_index */
  long long local_nnz;        /* entries in local columns */
  long long ghost_nnz;        /* entries in ghost columns */
} ab2_dist_info;
int ab2_dist_matrix_get_info(const ab2_dist_matrix* A, ab2_dist_info* info);
/* The rank's rows in the distributed layout: row_ptr (local_rows+1), cols
 * (DistStructInfo::m_cols: local ids, then ghost ids n_local+g), vals in the
 * same order, local_row_size (m_local_row_size), ghost_uids (global id of
 * each ghost, m_recv_info.m_uids order), interface_rows (m_interface_rows).
 * Any pointer may be null. */
int ab2_dist_matrix_layout(const ab2_dist_matrix* A, int* row_ptr, int* cols, double* vals, int* local_row_size,
                           int* ghost_uids, int* interface_rows);
/* Exchange plan: recv_ranks/recv_offsets (recv_neighbours, +1; ghost slices),
 * send_ranks/send_offsets (send_neighbours, +1) and send_ids (send_count local
 * rows, m_send_info.m_ids).  Any pointer may be null. */
int ab2_dist_matrix_plan(const ab2_dist_matrix* A, int* recv_ranks, int* recv_offsets, int* send_ranks,
                         int* send_offsets, int* send_ids);
/* The rank's diagonal block (local rows x local columns) as an ordinary
 * matrix, owned by A. */
int ab2_dist_matrix_local(const ab2_dist_matrix* A, const ab2_matrix** local);
int ab2_dist_matrix_destroy(ab2_dist_matrix* A);

/* A vector of A's local rows with room for its ghosts (the reference resizes
 * x to local + ghost before the exchange: SimpleCSRMatrixMultT.h:89-90).
 * Every other libab2 vector operation works on its local part. */
int ab2_dist_vector_create(ab2_context* ctx, const ab2_dist_matrix* A, ab2_vector** v);

/* ------------------------------------------------------------------ distributed algebra */
/* y = A x: ghost values of x are received into x's ghost room while the
 * local block is multiplied, then the interface rows add their ghost sums. */
int ab2_dist_mult(ab2_context* ctx, const ab2_dist_matrix* A, ab2_vector* x, ab2_vector* y);
int ab2_dist_dot(ab2_context* ctx, ab2_comm* comm, const ab2_vector* x, const ab2_vector* y, double* result);
int ab2_dist_norm1(ab2_context* ctx, ab2_comm* comm, const ab2_vector* x, double* result);
int ab2_dist_norm2(ab2_context* ctx, ab2_comm* comm, const ab2_vector* x, double* result); /* sqrt(sum of local x.x) */

/* Preconditioners over the rank's rows: AB2_PC_NONE, AB2_PC_DIAG (1/a_ii of the
 * local rows) and AB2_PC_ILU0 (block-Jacobi ILU(0), the reference's parallel
 * factorisation; applied with the same sweeps as ab2_precond_apply, tile walk
 * included when the local block is a 3-D 7-point grid).  Others:
 * AB2_ERR_UNSUPPORTED (Chebyshev and Neumann need the distributed algebra in
 * their set-up: run the reference's templates on Alien::B200::DistAlgebra).
 * Apply with ab2_precond_apply on local vectors. */
int ab2_dist_precond_create(ab2_context* ctx, const ab2_dist_matrix* A, const ab2_precond_options* opts,
                            ab2_precond** pc);

/* ------------------------------------------------------------------ distributed solver
 * CG or BiCGStab (CG.h, BiCGStab.h, Iteration.h) with NONE, DIAG or ILU0 on
 * the distributed algebra above, device-resident: iterations are queued in
 * batches of check_every without host synchronisation; every rank computes
 * the same global scalars, so all ranks stop at the same iteration.
 * use_graph and spmv_variant of the options are ignored. */
int ab2_dist_solver_create(ab2_context* ctx, ab2_comm* comm, const ab2_dist_matrix* A, const ab2_solver_options* opts,
                           ab2_dist_solver** s);
int ab2_dist_solver_solve(ab2_dist_solver* s, const ab2_vector* b, ab2_vector* x, ab2_status* status);
int ab2_dist_solver_history(const ab2_dist_solver* s, double* hist, int cap, int* len);
int ab2_dist_solver_destroy(ab2_dist_solver* s);

#ifdef __cplusplus
}
#endif

#endif /* AB2_DIST_H */
