/* iga_dist.h - multi-rank MatMult and Krylov solve over the reference's
 * partition files, one rank per GPU, with NCCL moving the ghost values and
 * the dot products between the GPUs.
 *
 * The reference runs its matrix-free solve on every MPI rank over PETSc
 * ghosted vectors (matrix_free/iteration_number_fempc_mf.cpp:62-72,193-233):
 * per MatMult a forward ghost update of x (VecGhostUpdate INSERT/FORWARD,
 * matrix_free/src/GlobalAssemblyMF.cpp:161-162), the rank's element loop,
 * and a reverse add of the ghost rows into their owners (ADD/REVERSE,
 * :195-196); per Krylov iteration global dot products (MPI_Allreduce inside
 * PETSc). Here each rank holds one part (include/iga_part.h); the forward
 * update and the reverse add are grouped ncclSend/ncclRecv between the ranks
 * that share ghosts, the dots are ncclAllReduce of FP64 values, and the
 * vector updates, the part's MatMult and the preconditioner are this
 * library's kernels, all stream-ordered on the rank's GPU: the host only
 * reads the convergence test every few iterations.
 *
 * NCCL is loaded at run time (libnccl.so.2, the library the caller's
 * communicator comes from when it is already loaded); nothing here needs it
 * until the first iga_dist_* call.
 */
#ifndef IGA_DIST_H
#define IGA_DIST_H
#include <stdint.h>

#include "iga_part.h"
#include "iga_solve.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct iga_dist iga_dist;

/* NCCL communicator helpers for callers without NCCL headers: a 128-byte
 * unique id made on one rank (and sent to the others by the caller's own
 * means), then ncclCommInitRank on every rank with its GPU current. */
int iga_dist_unique_id(void *id128);
int iga_dist_comm_create(int nranks, int rank, const void *id128, int device, void **comm);
int iga_dist_comm_destroy(void *comm);

/* Exchange maps of rank `rank` (host only). offsets[nranks + 1]: the owned
 * range of rank q is offsets[q] .. offsets[q+1]-1 in the partition
 * numbering; ghost_counts[q] and ghosts (all ranks' ghost lists,
 * concatenated in rank order) as iga_part_ghosts gives them. Outputs:
 * recv_count[q] ghosts of this rank that q owns and recv_pos (nghost
 * entries): their positions in this rank's ghost list, grouped by owner
 * (ascending owner, ascending position); send_count[q] entries of this
 * rank that q holds as ghosts and send_idx (capacity send_cap): their
 * owned-local indices, grouped by peer (ascending peer, in the peer's
 * ghost-list order); *nsend the total. Fails (IGA_ERR_ARG) on a ghost that
 * no other rank owns. */
int iga_dist_exchange_maps(int nranks, int rank, const int64_t *offsets, const int *ghost_counts,
                           const int64_t *ghosts, int *recv_count, int *recv_pos, int *send_count, int *send_idx,
                           int64_t send_cap, int64_t *nsend);

/* Collective over the communicator's ranks: every rank calls it with its own
 * part (opened, NOT yet built) and the same communicator. Builds the part on
 * `device` with the SPD sign and identity Dirichlet rows (the form the
 * solver iterates on), exchanges the owned ranges and ghost lists (NCCL
 * all-gathers), builds the exchange maps and the block preconditioner (the
 * exact FEM inverse of the rank's own sub-patch, restricted to its owned
 * entries: block-diagonal and SPD globally, no communication). */
int iga_dist_create(iga_part *part, void *comm, int nranks, int rank, int device, iga_dist **out);
int iga_dist_destroy(iga_dist *d);

/* y_owned = K x_owned over all ranks (collective; owned entries of the
 * partition numbering, device arrays of nlocalfunc doubles). */
int iga_dist_apply(iga_dist *d, const double *x_owned, double *y_owned, void *stream);

/* Flexible PCG on K x = b from x = 0 (collective), owned entries only.
 * opts: rtol, max_it and pc (IGA_PC_NONE or IGA_PC_FEM_EXACT = the block
 * FEM preconditioner); the loop stops when the recurrence residual
 * ||r|| <= rtol ||b|| (global norms) and then checks the true residual.
 * Per iteration: one distributed MatMult (two ghost exchanges), three
 * all-reductions (b.b once; p.q; r.r, r.z, r.z_old). stats: iterations,
 * relres (true residual), seconds, status. */
int iga_dist_solve(iga_dist *d, const double *b_owned, double *x_owned, const iga_solve_opts *opts,
                   iga_solve_stats *stats, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* IGA_DIST_H */
