/* iga_part.h - one part of a partitioned mesh: the reference's partition
 * files and its ghosted MatMult, for multi-rank (one rank per GPU) use.
 *
 * The reference's preprocessor cuts the patch into part_num_1d x part_num_1d
 * parts (matrix_free/src/Partition.cpp:3-235) and writes, per rank r,
 * <base_name>_<r>.txt plus info.txt (matrix_free/src/FileManager.cpp:3-69,
 * 375-452). Its MatMult (matrix_free/src/GlobalAssemblyMF.cpp:141-210) runs
 * on a PETSc ghosted vector (matrix_free/iteration_number_fempc_mf.cpp:62-72,
 * VecCreateGhost): the local form holds the part's owned entries (a
 * contiguous range of the partition numbering) followed by its ghosts
 * (ghostID order); each rank loops over its own elements, adds the element
 * results into the rows ID >= 0 of owned and ghost entries, and PETSc adds
 * the ghost contributions into their owners.
 *
 * iga_part_apply is that per-rank loop on the GPU: it gathers the part's
 * rectangular block of control points from the local form, applies the
 * operator of the part's sub-patch (every row a full element sum, no boundary
 * rule), and scatters the block back to the local form, with the reference's
 * Dirichlet rule applied by the local ID. The ghost traffic stays with the
 * caller, exactly where the reference has it:
 *     VecGhostUpdateBegin/End(x, INSERT_VALUES, SCATTER_FORWARD);   ghosts of x
 *     iga_part_apply(part, x_local, y_local, stream);               local forms
 *     VecGhostUpdateBegin/End(y, ADD_VALUES, SCATTER_REVERSE);      ghost sums to owners
 * (or the torch.distributed exchange of parallel-computing_b200/iga_dist.py).
 *
 * Reading and validation are host-only; iga_part_build creates the device
 * state (a plan for the sub-patch, the maps).
 */
#ifndef IGA_PART_H
#define IGA_PART_H
#include <stdint.h>

#include "iga_mf.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct iga_part iga_part;

typedef struct {
    int p, q, nElemX, nElemY, part_num_1d, dim;  /* info.txt */
    double Lx, Ly;
    int rank, part_x, part_y;      /* this part: rank = part_y * part_num_1d + part_x */
    int nlocalfunc, nghost;        /* owned entries, ghost entries of the local form */
    int nlocalelemx, nlocalelemy;  /* the part's elements */
    int elem_x0, elem_y0;          /* first element of the part in the patch */
    int block_m, block_n;          /* control points of the sub-patch block: nlocalelem + degree */
    int64_t owned_offset;          /* partition-numbering index of the first owned entry */
    int64_t nfunc_global;          /* (nElemX + p) * (nElemY + q) */
} iga_part_info;

/* Reads info.txt (FileManager::ReadPreprocessInfo layout) and the partition
 * file of `rank` (FileManager::ReadPartition layout, IGA variant with ghostID
 * and the extraction operators), and checks them: sizes, the structured
 * element block, local IEN covering the block one-to-one, owned entries
 * inside the block. Host only. */
int iga_part_open(const char *info_file, const char *part_file, int rank, iga_part **out);
int iga_part_close(iga_part *part);
int iga_part_get_info(const iga_part *part, iga_part_info *info);
/* nghost partition-numbering indices of the ghosts, in local-form order. */
int iga_part_ghosts(const iga_part *part, int64_t *ghosts);
/* block_m * block_n local-form indices of the block's control points (x fastest). */
int iga_part_block_map(const iga_part *part, int32_t *block_to_local);
/* nlocalfunc + nghost entries of the file's ID (partition-numbering row, or -1 on Dirichlet). */
int iga_part_local_id(const iga_part *part, int32_t *id);
/* Mesh description of the sub-patch (arrays owned by the part, valid until close). */
int iga_part_mesh(const iga_part *part, iga_mesh_desc *mesh);

/* Device state for applies: a plan of the sub-patch with opts->precision
 * IGA_FP64 and opts->geometry / opts->device as given; opts->sign chooses
 * -K (reference) or +K; opts->bc chooses the Dirichlet rule of the local
 * rows: IGA_BC_REFERENCE (rows ID < 0 are zero, x read everywhere) or
 * IGA_BC_IDENTITY (x[ID < 0] taken as 0, owned rows ID < 0 give x, ghost rows 0). */
int iga_part_build(iga_part *part, const iga_opts *opts);
/* y_local = the part's contribution in local form (owned rows complete only
 * after the ghost rows of every part are added to their owners). Device
 * arrays of nlocalfunc + nghost doubles, stream-ordered. */
int iga_part_apply(iga_part *part, const double *x_local, double *y_local, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* IGA_PART_H */
