/* CPU oracle for the matrix-free IGA Poisson operator and its Krylov solve.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * algorithm (SeaVegetable/Parallel-Computing, matrix_free/), used solely as the
 * checker by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
 * The shipped CUDA path never links, calls or falls back to it.
 *
 * Pinning: tests/test_oracle_pin.py checks every function here against the
 * reference's own element code compiled into oracle/_ref/libigaref.so
 * (oracle/Makefile, target "ref"), through the committed golden vectors under
 * tests/golden/ (made by tests/golden/make_golden.py). The reference ships no
 * golden vectors of its own. Features the reference does not have (NURBS
 * weights, a coefficient kappa, the adjoint gradient, FP32, PCG itself) are
 * checked against this restatement only: "parity unpinned" for those with
 * respect to the reference.
 */
#ifndef IGA_ORACLE_H
#define IGA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* SplitMix64 counter stream: u53 = (splitmix64(seed + (i+1)*golden) >> 11) * 2^-53 */
void orc_uniform(uint64_t seed, double lo, double hi, double *out, long n);
void orc_normal(uint64_t seed, double *out, long n); /* Box-Muller on the stream above */

/* 1-D ingredients */
void orc_gauss01(int n, double *x, double *w);               /* Gauss-Legendre on [0,1] */
void orc_bernstein(int p, double xi, double *B, double *dB); /* dB = d/dxi on [0,1] */
int orc_open_knots(int p, int ne, double L, double *S);     /* returns length ne+2p+1 */
int orc_extraction(int p, const double *S, int nS, double *C); /* Borden Alg. 1; returns nElem */
void orc_greville(int p, const double *S, int nS, double *g);  /* nS-p-1 values */

/* Single tensor-product patch as the reference stores it. CP is (x,y)
 * interleaved with x fastest (index i + j*m, m = nex+p); C1 is nex blocks of
 * (p+1)^2 (row-major, N = C B), C2 ney blocks of (q+1)^2; h1/h2 element sizes.
 * W (per control point) and kappa (per quadrature point, element-major,
 * qx fastest) are optional extensions (NULL = reference behaviour). */
typedef struct {
    int p, q, nex, ney;
    const double *CP, *W, *C1, *C2, *h1, *h2, *kappa;
} orc_patch;

/* y = sign * K x with the reference's element algorithm
 * (ElementMF::GenerateElementSingleQP + LocalAssemblyMF::LocalMatMulMF, loop of
 * GlobalAssemblyMF::MatMulMF). sign = -1 is the reference operator. Boundary
 * rows: bc = 0 -> y[Dir] = 0 (matrix-free reference), bc = 1 -> y[Dir] = x[Dir]
 * with x[Dir] not read (the SPD operator the solver uses), bc = 2 -> no
 * boundary rule (every row the full element sum: one part's sub-patch). */
void orc_apply_mf(const orc_patch *P, const double *x, double *y, double sign, int bc);
/* Reference mult_sf formula (LocalAssemblyMFSF::LocalMatMulMF); y[Dir] = 0. */
void orc_apply_sf(const orc_patch *P, const double *x, double *y, double sign);
/* F = int R f, F[Dir] = 0. fkind 0: x(1-x)y(1-y) (reference), 1: 2 pi^2 sin(pi x) sin(pi y),
 * 2: annulus manufactured f for u = sin(pi r) sin(2 theta). */
void orc_rhs(const orc_patch *P, int fkind, double *F);
/* Physical coordinates (x, y interleaved) and JxW at every quadrature point,
 * element-major with qx fastest. */
void orc_qp_points(const orc_patch *P, double *xy, double *jxw);
/* u_h = sum_a R_a u_a at every quadrature point (same order). */
void orc_eval_qp(const orc_patch *P, const double *u, double *vals);
/* dJ/dkappa_q = -grad(lam).grad(u) * JxW_q at every quadrature point. */
void orc_adjoint_grad(const orc_patch *P, const double *u, const double *lam, double *g);

/* Bilinear FEM preconditioner grid (one node per IGA control point).
 * 1-D nodes: degree p-2 Greville abscissae of the shortened knot vector
 * (reference matrix_free/preprocess_fem.cpp:38-60); for p = 2 (reference: NaN)
 * the degree-2 Greville abscissae of the IGA knot vector. */
void orc_fem_nodes(int p, int ne, double L, double *nodes);
/* y = sign*K_fem x on the interior, y[Dir] = x[Dir] (bc identity rows). */
void orc_fem_matvec(int nfx, int nfy, const double *nx, const double *ny, const double *x,
                    double *y, double sign);

/* FP64 PCG on the SPD operator (orc_apply_mf with sign=+1, bc=1) with the FEM
 * preconditioner applied by an inner Jacobi-CG to inner_rtol. Stops on the
 * relative true residual ||b-Ax||/||b|| <= rtol. Returns iterations (<0: failure). */
int orc_pcg(const orc_patch *P, const double *fem_nx, const double *fem_ny, const double *b,
            double *x, double rtol, int maxit, double inner_rtol, int inner_maxit,
            double *relres_out);

#ifdef __cplusplus
}
#endif
#endif
