/* iga_batch.h - many independent Poisson solves advanced together.
 *
 * No counterpart in the reference (SeaVegetable/Parallel-Computing solves one
 * mesh per program run: matrix_free/iteration_number_fempc_mf.cpp:193-233).
 * A batch holds one plan per problem (meshes of any size; degrees 1..5 mixed
 * freely) and solves K_i x_i = b_i for every i with flexible PCG and the exact
 * bilinear-FEM preconditioner (fast diagonalisation), to the same per-problem
 * criterion as iga_solve: relative true residual ||b_i - K_i x_i|| / ||b_i||
 * <= rtol. Every kernel of an iteration covers the whole batch through work
 * lists (operator strips, reduction chunks, preconditioner GEMM tiles);
 * problems that have converged drop out of the work. The whole solve is one
 * CUDA graph launch whose conditional WHILE node runs the iterations on the
 * device until no problem is left.
 *
 * Vectors: a batch vector is the concatenation of the problems' vectors in
 * batch order, problem i at entries offsets[i] .. offsets[i+1]-1
 * (iga_batch_offsets), each in the layout of iga_mf.h. The operator is the
 * SPD one the solver uses (+K, identity rows on the boundary).
 *
 * Tile shapes: the element rows per warp strip of each problem and the warps
 * per CTA of each degree come from a tuning table (JSON) written by
 * iga_batch_autotune, which times the batched operator for candidate shapes
 * per (degree, precision, size bucket). Without a table, built-in defaults.
 */
#ifndef IGA_BATCH_H
#define IGA_BATCH_H
#include <stdint.h>

#include "iga_mf.h"
#include "iga_solve.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct iga_batch iga_batch;

typedef struct {
    int precision;          /* IGA_FP64 (FP64 PCG) or IGA_MIXED (FP32 PCG sweeps, FP64 refinement) */
    int device;
    const char *tune_file;  /* tuning table to read, or NULL for the built-in defaults */
} iga_batch_opts;

typedef struct {
    int status;                 /* IGA_OK when every problem met rtol, else the first failure's code */
    int converged;              /* problems that met rtol */
    int max_iterations;         /* largest per-problem PCG iteration count (all sweeps) */
    int64_t total_iterations;   /* sum over problems */
    int max_sweeps;             /* IGA_MIXED: most refinement sweeps any problem used */
    double max_relres;          /* largest ||b_i - K_i x_i|| / ||b_i|| (FP64 operator) */
    double seconds;             /* host wall time of iga_batch_solve */
} iga_batch_stats;

void iga_batch_opts_default(iga_batch_opts *opts);

/* Builds the plans of every problem (meshes as for iga_plan_create; kappa must
 * be NULL; at most 272 free control points in y, i.e. nElemY + q <= 274), the
 * work lists, and the preconditioner's 1-D eigenpairs (shared by problems with
 * equal 1-D FEM grids). */
int iga_batch_create(const iga_mesh_desc *meshes, int count, const iga_batch_opts *opts, iga_batch **out);
int iga_batch_destroy(iga_batch *batch);
/* count+1 entries: start of every problem's vector, then the total length. */
int iga_batch_offsets(const iga_batch *batch, int64_t *offsets);
/* The plan of problem i (owned by the batch), e.g. to apply one problem alone. */
iga_plan *iga_batch_plan(iga_batch *batch, int i);
/* Rows per strip of problem i and warps per CTA of its degree, as used. */
int iga_batch_shape(const iga_batch *batch, int i, int precision, int *rows_per_strip, int *warps_per_cta);

/* y = K x for every problem (SPD operator), device batch vectors of doubles
 * (IGA_FP64) or floats (IGA_FP32, MIXED batches only), stream-ordered. */
int iga_batch_apply(iga_batch *batch, int precision, const void *x, void *y, void *stream);
/* z = M^-1 r for every problem with the exact FEM preconditioner
 * (pc = IGA_PC_FEM_EXACT) or the identity (IGA_PC_NONE). */
int iga_batch_pc_apply(iga_batch *batch, int pc, int precision, const void *r, void *z, void *stream);

/* Solves every problem: b and x are device FP64 batch vectors. Uses o->rtol,
 * max_it (per problem, per sweep for MIXED), pc (IGA_PC_FEM_EXACT or
 * IGA_PC_NONE), sweep_rtol, max_sweeps and x0_nonzero; o = NULL: defaults
 * with pc = IGA_PC_FEM_EXACT. iterations / relres (count entries each, host)
 * receive the per-problem results when not NULL. Synchronises. */
int iga_batch_solve(iga_batch *batch, const double *b, double *x, const iga_solve_opts *o, iga_batch_stats *stats,
                    int *iterations, double *relres, void *stream);

/* Times the batched operator over these problems for candidate shapes (rows
 * per strip per size bucket, then warps per CTA per degree), precision
 * IGA_FP64 (tunes FP64 batches) or IGA_MIXED (tunes the FP32 operator of
 * MIXED batches), and merges the winners into tune_file (created if absent). */
int iga_batch_autotune(const iga_mesh_desc *meshes, int count, int precision, int device, const char *tune_file);
/* Shape the table gives a problem: rows per strip (0: no entry) and warps per
 * CTA (0: no entry). Host only; IGA_ERR_ARG if the file cannot be parsed. */
int iga_tune_lookup(const char *tune_file, int p, int precision, int nElemX, int nElemY, int *rows_per_strip,
                    int *warps_per_cta);

#ifdef __cplusplus
}
#endif
#endif /* IGA_BATCH_H */
