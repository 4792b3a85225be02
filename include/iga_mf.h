/* iga_mf.h - C ABI of the B200 matrix-free isogeometric Poisson operator.
 *
 * Drop-in boundary for the reference's matrix-free MatMult
 * (SeaVegetable/Parallel-Computing):
 *   - the PETSc MATSHELL MATOP_MULT callback MyMatMult
 *     (matrix_free/iteration_number_fempc_mf.cpp:46-60,
 *      matrix_free_gpu/matrixfreegpu.cu:52-66), which calls
 *   - GlobalAssemblyMF::MatMulMF (matrix_free/src/GlobalAssemblyMF.cpp:141-281,
 *     matrix_free_gpu/src/GlobalAssemblyMF.cu:126-242), which on the GPU calls
 *   - MatrixFreeMatMultCUDA (matrix_free_gpu/include/mult.cuh:16-24).
 *
 * Semantics kept from the reference (IGA_SIGN_REFERENCE, IGA_BC_REFERENCE):
 *   y = A_ref x with A_ref = -K (K the SPD stiffness), x gathered through the
 *   element connectivity (boundary values x[Dir] are read), y[Dir] = 0.
 * Vector layout: one entry per control point, index i + j*m with x fastest,
 * m = nElemX + p (the serial layout of the reference's partition files).
 *
 * Differences from the reference, all deliberate:
 *   - a plan owns every device table and is built once (the reference copies
 *     all mesh tables to the device on every MatMult);
 *   - calls are stream-ordered and return a status code (the reference calls
 *     exit() on any CUDA error and synchronises the device after each launch);
 *   - results are bitwise reproducible (no atomics in any reduction).
 *
 * No CUDA or C++ types cross this boundary: streams are passed as void*
 * (a cudaStream_t, NULL = the legacy default stream), device buffers as
 * plain pointers.
 */
#ifndef IGA_MF_H
#define IGA_MF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct iga_plan iga_plan;

/* Status codes; every entry point returns one (never exits). */
enum {
    IGA_OK = 0,
    IGA_ERR_ARG = 1,            /* invalid argument or mesh */
    IGA_ERR_UNSUPPORTED = 2,    /* valid input this library does not handle */
    IGA_ERR_CUDA = 3,           /* a CUDA runtime call failed */
    IGA_ERR_NOMEM = 4,          /* device allocation failed */
    IGA_ERR_NOT_CONVERGED = 5,  /* Krylov solve hit max_it */
    IGA_ERR_BREAKDOWN = 6,      /* Krylov breakdown (p.Ap <= 0, indefinite PC) */
    IGA_ERR_NONFINITE = 7,      /* NaN/Inf met in a solve */
    IGA_ERR_TIMEOUT = 8         /* a bounded device wait gave up */
};

enum { IGA_FP64 = 0, IGA_FP32 = 1, IGA_MIXED = 2 };          /* operator precision(s) */
enum { IGA_GEOM_PRECOMPUTED = 0, IGA_GEOM_ON_THE_FLY = 1 };  /* mult_sf / mult_mf paths */
enum { IGA_SIGN_REFERENCE = -1, IGA_SIGN_SPD = 1 };
/* y[Dir]=0 / y[Dir]=x[Dir] / no boundary rows: every row is the full sum over
 * the patch's elements and x is read everywhere (the sub-patch of one part of
 * a partitioned mesh, whose ring rows are partial sums; include/iga_part.h) */
enum { IGA_BC_REFERENCE = 0, IGA_BC_IDENTITY = 1, IGA_BC_NONE = 2 };
enum { IGA_F_REFERENCE = 0, IGA_F_SINSIN = 1, IGA_F_ANNULUS = 2 }; /* load functions */

/* One single-patch tensor-product mesh, in the reference's arrays (all HOST
 * pointers, read during iga_plan_create only). Optional arrays may be NULL. */
typedef struct {
    int p, q;             /* degrees; this library requires p == q, 1 <= p <= 5 */
    int nElemX, nElemY;
    const double *CP;     /* 2*nfunc, (x,y) interleaved, nfunc = (nElemX+p)*(nElemY+q) */
    const double *weights;/* nfunc NURBS weights or NULL (reference: no weights).
                             Weights must factor as w(i,j) = a(i) b(j). */
    const double *C1;     /* nElemX*(p+1)^2 row-major extraction operators (N = C B) or NULL:
                             generated from the open uniform knot vector */
    const double *C2;     /* nElemY*(q+1)^2 or NULL */
    const double *h1, *h2;/* element sizes; accepted for drop-in, the operator does not depend on them */
    const int *IEN;       /* nElem*(p+1)*(q+1) or NULL; if given it must be the structured patch */
    const int *ID;        /* nfunc or NULL; if given, -1 exactly on the boundary ring */
    const int *Dir;       /* nDir boundary indices or NULL; if given, the boundary ring */
    int nDir;
    const double *kappa;  /* coefficient per quadrature point, element-major, qx fastest, or NULL */
} iga_mesh_desc;

typedef struct {
    int precision;  /* IGA_FP64, IGA_FP32 or IGA_MIXED (both operators) */
    int geometry;   /* IGA_GEOM_PRECOMPUTED or IGA_GEOM_ON_THE_FLY */
    int sign;       /* IGA_SIGN_REFERENCE (default for the drop-in) or IGA_SIGN_SPD */
    int bc;         /* IGA_BC_REFERENCE, IGA_BC_IDENTITY or IGA_BC_NONE */
    int device;     /* CUDA device ordinal */
    int rows_per_strip; /* element rows per warp strip, 0 = default (tuned) */
} iga_opts;

typedef struct {
    int64_t nfunc;          /* vector length N */
    int64_t nelem;
    int64_t geom_bytes;     /* device bytes of precomputed geometry per precision (0 on the fly) */
    int64_t algo_bytes_f64; /* algorithmic HBM bytes of one FP64 apply */
    int64_t algo_bytes_f32; /* ... of one FP32 apply */
    int rows_per_strip;
    int warps_per_cta;
} iga_plan_info;

/* ------------------------------------------------------------- meshes */
/* Unit-square-type patch [0,Lx]x[0,Ly] of matrix_free/preprocess.cpp:37-83:
 * open uniform knots, control points at the Greville abscissae (the linear
 * parameterisation the reference's ControlPointGenerator solves for), Bezier
 * extraction operators. Output sizes: CP 2*(nElemX+p)*(nElemY+p),
 * C1 nElemX*(p+1)^2, C2 nElemY*(p+1)^2 (host arrays). */
int iga_mesh_unit_square(int p, int nElemX, int nElemY, double Lx, double Ly, double *CP, double *C1, double *C2);

/* Exact quarter annulus r in [r_in, r_out], theta in [0, pi/2] as a NURBS
 * patch (no counterpart in the reference, which has no rational geometry):
 * radial direction (index i, x-fastest) linear, angular direction the rational
 * quadratic arc with middle weight sqrt(2)/2, both degree-elevated to p >= 2
 * and refined by uniform knot insertion to nElemX x nElemY elements. Outputs:
 * CP 2*(nElemX+p)*(nElemY+p), W (nElemX+p)*(nElemY+p) weights, C1/C2
 * extraction operators as for iga_mesh_unit_square. */
int iga_mesh_quarter_annulus(int p, int nElemX, int nElemY, double r_in, double r_out, double *CP, double *W,
                             double *C1, double *C2);

/* ---------------------------------------------------------------- plans */
/* Build a plan: validate the mesh, upload the tables, precompute geometry. */
int iga_plan_create(const iga_mesh_desc *mesh, const iga_opts *opts, iga_plan **out);
int iga_plan_destroy(iga_plan *plan);
int iga_plan_get_info(const iga_plan *plan, iga_plan_info *info);
void iga_opts_default(iga_opts *opts);
const char *iga_status_str(int status);
/* Text of the last error recorded on the calling host thread. */
const char *iga_last_error(void);

/* ------------------------------------------------------------ operator */
/* y = A x on the device, stream-ordered (replaces MyMatMult ->
 * GlobalAssemblyMF::MatMulMF -> MatrixFreeMatMultCUDA). x and y are device
 * arrays of nfunc doubles (FP64 / MIXED plans) or floats (FP32 plans), must
 * not alias, and are owned by the caller. */
int iga_apply(iga_plan *plan, const void *x_dev, void *y_dev, void *stream);
/* Same, choosing the operator precision of a MIXED plan explicitly. */
int iga_apply_prec(iga_plan *plan, int precision, const void *x_dev, void *y_dev, void *stream);
/* Host-buffer MatMult (the MATSHELL callback on host vectors): copies x in,
 * applies the FP64 operator, copies y out, and synchronises. The patch goes
 * through in slabs of strip rows on the plan's own streams, so that the
 * copies in both directions overlap the kernels (pinned host buffers give
 * the overlap; pageable ones work, slower). Ordered after prior work on the
 * legacy default stream; the result is bitwise that of iga_apply. */
int iga_apply_host(iga_plan *plan, const double *x_host, double *y_host);

/* Synchronises `stream` (a cudaStream_t or NULL), then reads and clears the
 * plan's device error flag: IGA_OK, or the status a kernel recorded since the
 * last query (IGA_ERR_TIMEOUT: a bounded wait for a bulk copy gave up; the
 * kernel stopped, let its copies land and returned, and the plan stays usable).
 * The stream-ordered calls (iga_apply, iga_apply_prec, iga_rhs) cannot report
 * such errors themselves; iga_apply_host and the solver check the flag. No
 * counterpart in the reference, which calls exit() on any CUDA error
 * (matrix_free_gpu/include/memory.cuh:9-12). */
int iga_plan_device_status(iga_plan *plan, void *stream);
/* Polls each bounded wait of the plan's MatMult kernel makes before it gives
 * up with IGA_ERR_TIMEOUT: polls >= 0 sets the limit (0: every wait gives up
 * at once, for tests of the timeout path; the kernel still waits, with the
 * full limit, for the copies it issued before returning), polls < 0 restores
 * the default (2^24 polls, seconds of wall time). A test hook: no counterpart
 * in the reference. */
int iga_plan_set_wait_limit(iga_plan *plan, long long polls);

/* Load vector F = int R f with F[Dir] = 0 (GlobalAssemblyMF::AssemLoad,
 * matrix_free/src/GlobalAssemblyMF.cpp:26-80), FP64, device output. */
int iga_rhs(iga_plan *plan, int fkind, double *F_dev, void *stream);

/* Reference-shaped entry point: the argument list of MatrixFreeMatMultCUDA
 * (matrix_free_gpu/include/mult.cuh:16-24, all device pointers), synchronous
 * like the reference's (cudaDeviceSynchronize after the kernel,
 * matrix_free_gpu/src/mult.cu:550); the status covers the kernels' run.
 *   - d_IEN must be the structured single-patch connectivity the reference's
 *     IENGenerator::GenerateIEN2D writes (matrix_free/src/IENGenerator.cpp:
 *     68-103); anything else returns IGA_ERR_UNSUPPORTED. NULL: assumed.
 *   - d_ID is honoured as the reference kernel honours it
 *     (matrix_free_gpu/src/mult.cu:455-460): control point A's row goes to
 *     y[ID[A]] when ID[A] >= 0 and nowhere otherwise. ID values must lie below
 *     nfunc = (nElemX+p)*(nElemY+q) and name no row twice (else
 *     IGA_ERR_UNSUPPORTED). With the reference's serial numbering (-1 on the
 *     boundary ring, A elsewhere; or NULL) the boundary rows are written as
 *     zero (y[Dir] = 0, which the reference caller's DirichletBCCUDA does);
 *     with any other ID the entries of y no ID value names keep their
 *     contents, so the caller zeroes y first, as the reference's caller does
 *     (matrix_free_gpu/src/GlobalAssemblyMF.cu:210).
 *   - d_B1/d_B2/d_dB1/d_dB2 and qw1/qw2 (Bernstein values/derivatives at the
 *     p+1 Gauss points on [0,1], point-major, and the Gauss weights) are
 *     checked once against the rule this library integrates with
 *     (IGA_ERR_UNSUPPORTED if they differ); all NULL: the library's own.
 *   - h1/h2 are accepted and not needed (they cancel in the operator).
 *   - d_F_array_in / d_F_array_out: 8-byte aligned, nfunc doubles.
 * The first call with a given set of arrays on a device builds and caches a
 * plan (one device-to-host copy of CP and the extraction operators, a device
 * check of IEN/ID); later calls with the same pointers on the same device
 * reuse it and assume the arrays' contents unchanged: after rewriting any of
 * them in place (or freeing them and reusing the addresses), call
 * iga_MatrixFreeMatMultCUDA_release. Unlike the reference it does not exit on
 * error. */
int iga_MatrixFreeMatMultCUDA(int p, int q, int nlocalelemx, int nlocalelemy,
                              const double *d_B1, const double *d_B2,
                              const double *d_dB1, const double *d_dB2,
                              const double *d_nurbs_extraction1, const double *d_nurbs_extraction2,
                              const double *d_elem_size1, const double *d_elem_size2,
                              const int *d_IEN, const int *d_ID, const double *d_CP,
                              const double *qw1, const double *qw2,
                              const double *d_F_array_in, double *d_F_array_out);
/* Drop every plan cached by iga_MatrixFreeMatMultCUDA. */
int iga_MatrixFreeMatMultCUDA_release(void);

/* Allocation-free MatMult. No counterpart in the reference: added for callers
 * that cannot allocate device memory when they need a MatMult (their own memory
 * pool owns the GPU, or a cudaMalloc/cudaFree device synchronisation inside a
 * solver loop is not acceptable). Arguments are those of
 * iga_MatrixFreeMatMultCUDA plus a stream; every array is a caller-owned device
 * array, and d_B1/d_dB1 (d_B2/d_dB2) must hold the Bernstein values/derivatives
 * at the p+1 (q+1) Gauss points on [0,1], point-major, and qw1/qw2 the Gauss
 * weights (the arrays the reference uploads). Geometry is computed on the fly
 * from d_CP (no NURBS weights). Computes y = A_ref x; d_IEN and d_ID are
 * checked and honoured exactly as by iga_MatrixFreeMatMultCUDA (on every call,
 * before y is touched; NULL: the structured connectivity and the reference's
 * serial numbering, with y[Dir] = 0). Alignment: d_CP 16 bytes (it is read as
 * (x, y) pairs), the other double arrays 8 bytes, d_IEN/d_ID 4 bytes;
 * otherwise IGA_ERR_ARG before anything runs. p == q with 1 <= p <= 5, else
 * IGA_ERR_UNSUPPORTED. The call runs on `stream` and returns after the
 * stream's work is done (the kernels' error slot is read back: IGA_ERR_TIMEOUT
 * when a bounded wait gave up).
 * This entry point calls no cudaMalloc, cudaFree or other allocating routine:
 * its scratch (basis tables, seam frames, the IEN/ID check words) is a fixed
 * 16 MiB device array held by every GPU that loads the library until the
 * process exits. Meshes whose scratch would exceed 16 MiB are rejected with
 * IGA_ERR_UNSUPPORTED (p = 3 up to about 2048 x 2048 elements fits). The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress)
 * and sets the kernel's shared memory limit; make that first call before any
 * stream capture. All calls share the one array, so calls that overlap on the
 * GPU (other streams, other host threads) race and must be serialised by the
 * caller. */
int iga_MatrixFreeMatMultCUDA_noalloc(int p, int q, int nlocalelemx, int nlocalelemy,
                                      const double *d_B1, const double *d_B2,
                                      const double *d_dB1, const double *d_dB2,
                                      const double *d_nurbs_extraction1, const double *d_nurbs_extraction2,
                                      const double *d_elem_size1, const double *d_elem_size2,
                                      const int *d_IEN, const int *d_ID, const double *d_CP,
                                      const double *qw1, const double *qw2,
                                      const double *d_F_array_in, double *d_F_array_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* IGA_MF_H */
