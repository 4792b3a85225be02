/* iga_solve.h - device-resident Krylov solve of the IGA Poisson system with
 * the bilinear-FEM preconditioner, and the FEM preconditioner's assembly.
 *
 * Replaces the reference's solve loop: PETSc KSPSolve on the MATSHELL with a
 * PCSHELL whose apply is an inner KSPCG + PCJACOBI solve of the bilinear FEM
 * matrix (matrix_free/iteration_number_fempc_mf.cpp:11-17,199-233), and the
 * GPU driver's FEM assembly (elem2coo + MATAIJCUSPARSE COO assembly:
 * matrix_free_gpu/src/Elem2COOGenerator.cpp:3-69, matrix_free_gpu/src/assembly.cu:41-99,
 * matrix_free_gpu/src/GlobalAssembly.cu:3-108).
 *
 * The system solved is the SPD form K u = b (boundary rows identity, b[Dir]
 * expected 0). The reference solves A_ref u = F with A_ref = -K, whose
 * solution is the negative of this one; pass -F to get the reference's
 * vector. Iteration counts are not strictly comparable with the reference:
 * it runs GMRES with a preconditioned-residual test; this runs flexible PCG
 * to a relative TRUE residual ||b - K u|| / ||b|| <= rtol.
 */
#ifndef IGA_SOLVE_H
#define IGA_SOLVE_H

#include <stdint.h>

#include "iga_mf.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    IGA_PC_NONE = 0,      /* unpreconditioned CG */
    IGA_PC_FEM_CG = 1,    /* reference: inner Jacobi-CG on the bilinear FEM matrix */
    IGA_PC_FEM_EXACT = 2  /* the same FEM matrix inverted exactly (tensor-product fast diagonalisation) */
};

enum {
    IGA_MIXED_PC = 3   /* solve precision: FP64 flexible PCG (FP64 operator and vectors) with the
                          preconditioner evaluated in FP32 (TF32 tensor-core GEMMs) */
};

typedef struct {
    int precision;     /* IGA_FP64: FP64 PCG. IGA_MIXED: FP32 PCG sweeps (FP32 operator and
                          preconditioner) wrapped in FP64 iterative refinement. IGA_MIXED_PC:
                          FP64 PCG, FP32 preconditioner (needs only the FP64 operator). */
    int pc;            /* IGA_PC_* */
    double rtol;       /* target relative true residual (FP64) */
    int max_it;        /* outer PCG iterations per solve / per FP32 sweep */
    double pc_rtol;    /* IGA_PC_FEM_CG inner tolerance (reference: 1e-10) */
    int pc_max_it;     /* IGA_PC_FEM_CG inner iteration cap (reference: 10000) */
    double sweep_rtol; /* IGA_MIXED: residual reduction asked of each FP32 sweep (default 1e-3:
                          shallow sweeps restart the Krylov space before FP32 rounding slows it);
                          a sweep asks for less when less is left to reach rtol */
    int max_sweeps;    /* IGA_MIXED: refinement sweeps */
    int x0_nonzero;    /* 1: use x as the initial guess, 0: start from x = 0 */
} iga_solve_opts;

typedef struct {
    int status;            /* IGA_OK or IGA_ERR_NOT_CONVERGED / BREAKDOWN / NONFINITE */
    int iterations;        /* outer PCG iterations (all sweeps) */
    int64_t pc_iterations; /* inner FEM-CG iterations (IGA_PC_FEM_CG) */
    int sweeps;            /* refinement sweeps (IGA_MIXED) */
    double relres;         /* final ||b - K x|| / ||b||, FP64 */
    double seconds;        /* wall time of the solve (device synchronised) */
} iga_solve_stats;

void iga_solve_opts_default(iga_solve_opts *opts);

/* Solve K x = b on the device (b, x: nfunc doubles, caller-owned). The plan
 * must hold the FP64 operator; IGA_MIXED needs a plan created with
 * precision IGA_MIXED (both operators); IGA_MIXED_PC runs on either. */
int iga_solve(iga_plan *plan, const double *b_dev, double *x_dev, const iga_solve_opts *opts,
              iga_solve_stats *stats, void *stream);

/* z = M^-1 r for one preconditioner (the PCSHELL apply MyPCApply,
 * matrix_free/iteration_number_fempc_mf.cpp:11-17): IGA_PC_FEM_CG runs the inner
 * Jacobi-CG to pc_rtol (at most pc_max_it iterations), IGA_PC_FEM_EXACT applies
 * K_fem^-1 exactly, IGA_PC_NONE copies. precision: IGA_FP64 (double arrays) or
 * IGA_FP32 (float arrays; FEM_EXACT then uses TF32 tensor-core GEMMs). */
int iga_pc_apply(iga_plan *plan, int pc, int precision, const void *r_dev, void *z_dev, double pc_rtol,
                 int pc_max_it, void *stream);

/* IGA_PC_FEM_EXACT splits its x transforms by parity (the FEM nodes of a
 * patch side are symmetric about its middle, so every x eigenvector is
 * symmetric or antisymmetric and each transform costs half the flops).
 * enable = 0 makes the plan's solver use the full transforms instead, 1
 * restores the default; either drops the plan's solver state (rebuilt on
 * the next solve). A test hook: the two forms give the same z to rounding.
 * No counterpart in the reference. */
int iga_plan_set_pc_split(iga_plan *plan, int enable);

/* enable = 0 makes iga_solve run its PCG iterations from the host, kernel by
 * kernel, instead of inside one conditional-loop graph (per-kernel profilers
 * do not see the kernels of conditional graphs); 1 restores the default.
 * Same kernels and arithmetic per iteration; the host reads the convergence
 * test after each one. A profiling hook: no counterpart in the reference. */
int iga_plan_set_solver_graph(iga_plan *plan, int enable);

/* y = K_fem x, the SPD bilinear-FEM matrix of the preconditioner (boundary
 * rows identity), matrix-free from its 1-D tensor factors; precision of x/y
 * as for iga_apply_prec. */
int iga_fem_apply(iga_plan *plan, int precision, const void *x_dev, void *y_dev, void *stream);

/* The FEM preconditioner matrix assembled on the device in CSR form, one
 * thread per row, no atomics (replaces Elem2COOGenerator + the COO atomicAdd
 * assembly). sign = -1 gives the reference's matrix (-K_fem on free rows,
 * +1 on Dirichlet diagonals), +1 the SPD one. Call with NULL arrays to get
 * nnz; rowptr has nfunc+1 entries. */
int iga_fem_assemble_csr(iga_plan *plan, int sign, int32_t *rowptr_dev, int32_t *colidx_dev, double *vals_dev,
                         int64_t *nnz, void *stream);

/* Coefficient of -div(kappa grad u) = f at the quadrature points (device array,
 * element-major, qx fastest; nElemX*nElemY*(p+1)^2 doubles), replacing the
 * plan's current kappa (kappa = 1 in the reference). Recomputes the
 * precomputed geometry on the device; on-the-fly plans store kappa. The
 * solver's preconditioners are rescaled by the local mean of kappa. No
 * counterpart in the reference. */
int iga_plan_set_kappa(iga_plan *plan, const double *kappa_dev, void *stream);

/* Adjoint gradient (no counterpart in the reference): g_q = -(grad lambda .
 * grad u)(x_q) * JxW_q at every quadrature point (same layout as kappa), i.e.
 * dJ/dkappa_q when K(kappa) u = F and K lambda = dJ/du with lambda = 0 on the
 * boundary. u, lambda: nfunc doubles on the device. */
int iga_adjoint_grad(iga_plan *plan, const double *u_dev, const double *lambda_dev, double *g_dev, void *stream);

/* 1-D node coordinates of the FEM preconditioner grid (host arrays of
 * nElemX+p and nElemY+q entries): degree p-2 Greville abscissae of the
 * shortened knot vector (matrix_free/preprocess_fem.cpp:38-60) for p >= 3; the
 * reference divides by zero for p = 2, replaced by the degree-2 Greville
 * abscissae of the IGA knot vector. */
int iga_fem_nodes(const iga_plan *plan, double *gx, double *gy);

/* The same 1-D nodes without a plan (host only): ne + p coordinates of a
 * direction with ne elements of degree p and net length L (the mean polyline
 * length of the control net in that direction; L on an axis-aligned patch of
 * length L), for callers that hold only part of a patch (the partitioned
 * FEM matrix of a multi-rank preconditioner). */
int iga_fem_nodes_1d(int p, int ne, double L, double *g);

/* Extreme eigenvalues of the SPD operator K (pc = IGA_PC_NONE) or of the
 * preconditioned M^-1 K (pc = IGA_PC_FEM_EXACT or IGA_PC_FEM_CG) on the free
 * control points, from `steps` Lanczos steps: the coefficients of a standard
 * PCG (FP64, device) on a seeded random right-hand side form the Lanczos
 * matrix, whose extreme eigenvalues are returned (host). steps_done (may be
 * NULL) receives the steps taken (fewer when the Krylov space is exhausted).
 * The reference studies the same extremes with SLEPc's Lanczos SVD
 * (eigenvalue_problem/driver.cpp:252-411); condition numbers are
 * lam_max / lam_min. */
int iga_spectrum_estimate(iga_plan *plan, int pc, int steps, uint64_t seed, double *lam_min, double *lam_max,
                          int *steps_done);

#ifdef __cplusplus
}
#endif
#endif /* IGA_SOLVE_H */
