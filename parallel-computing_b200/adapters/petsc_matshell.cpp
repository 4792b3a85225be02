// petsc_matshell.cpp - the reference's PETSc MATSHELL MatMult on this
// library, as a source file a maintainer adds to the reference's own build
// (it needs PETSc, which this repository does not build against).
//
// The reference registers MyMatMult as MATOP_MULT of a shell matrix
// (matrix_free/iteration_number_fempc_mf.cpp:46-60,193-197; the GPU driver:
// matrix_free_gpu/matrixfreegpu.cu:52-66) and hands the shell to KSPSolve.
// Here the shell's context holds an iga_plan (one patch, one rank) or an
// iga_part (one part of the reference's partition files, one rank of a
// multi-rank run), and MatMult is one call into the library:
//   * IgaMatCreateShell: y = A x on the rank's vector; device arrays
//     (VecCUDAGetArrayRead / VecCUDAGetArrayWrite) for CUDA vectors, host
//     arrays (iga_apply_host: upload, apply, download) otherwise;
//   * IgaMatCreateShellGhosted: the reference's ghosted layout (VecCreateGhost,
//     iteration_number_fempc_mf.cpp:62-72): forward ghost update of x
//     (INSERT_VALUES, SCATTER_FORWARD), the part's contribution on the local
//     forms (iga_part_apply), reverse add of the ghost rows of y (ADD_VALUES,
//     SCATTER_REVERSE), as GlobalAssemblyMF::MatMulMF does around its element
//     loop (matrix_free/src/GlobalAssemblyMF.cpp:161-162,195-196).
// The library's calls return a status; a non-zero one becomes PETSC_ERR_LIB
// with the library's message instead of the reference's exit().
//
// The library runs on the legacy default stream here and the call waits for
// it, so that the arrays PETSc gets back are complete (PETSc does not order
// its own work after another library's streams).
#include <cuda_runtime.h>
#include <petscmat.h>

#include "iga_mf.h"
#include "iga_part.h"

namespace {

struct IgaShellCtx {
    iga_plan *plan = nullptr;   // whole patch (IgaMatCreateShell)
    iga_part *part = nullptr;   // one part of a partition (IgaMatCreateShellGhosted)
    PetscInt nghost = 0;
};

PetscErrorCode lib_error(Mat A, int status)
{
    MPI_Comm comm;
    PetscCall(PetscObjectGetComm((PetscObject)A, &comm));
    SETERRQ(comm, PETSC_ERR_LIB, "iga_b200 status %d: %s", status, iga_last_error());
}

bool is_cuda(Vec v)
{
    PetscBool cuda = PETSC_FALSE;
    PetscObjectTypeCompareAny((PetscObject)v, &cuda, VECSEQCUDA, VECMPICUDA, VECCUDA, "");
    return cuda == PETSC_TRUE;
}

}  // namespace

extern "C" PetscErrorCode IgaMatMult(Mat A, Vec x, Vec y)
{
    IgaShellCtx *ctx = nullptr;
    PetscFunctionBeginUser;
    PetscCall(MatShellGetContext(A, &ctx));
    int st;
    if (is_cuda(x) && is_cuda(y)) {
        const PetscScalar *xa;
        PetscScalar *ya;
        PetscCall(VecCUDAGetArrayRead(x, &xa));
        PetscCall(VecCUDAGetArrayWrite(y, &ya));
        st = iga_apply(ctx->plan, xa, ya, nullptr);
        if (st == IGA_OK && cudaStreamSynchronize(nullptr) != cudaSuccess) st = IGA_ERR_CUDA;
        PetscCall(VecCUDARestoreArrayRead(x, &xa));
        PetscCall(VecCUDARestoreArrayWrite(y, &ya));
    } else {
        const PetscScalar *xa;
        PetscScalar *ya;
        PetscCall(VecGetArrayRead(x, &xa));
        PetscCall(VecGetArrayWrite(y, &ya));
        st = iga_apply_host(ctx->plan, xa, ya);
        PetscCall(VecRestoreArrayRead(x, &xa));
        PetscCall(VecRestoreArrayWrite(y, &ya));
    }
    if (st != IGA_OK) PetscCall(lib_error(A, st));
    PetscFunctionReturn(0);
}

// The reference's ghosted layout: x and y are VecCreateGhost vectors whose
// local forms hold the rank's owned entries then its ghosts, in the order of
// the partition file (iga_part_ghosts). CUDA ghosted vectors are used on the
// device, others through a device copy of the local forms.
extern "C" PetscErrorCode IgaMatMultGhosted(Mat A, Vec x, Vec y)
{
    IgaShellCtx *ctx = nullptr;
    PetscFunctionBeginUser;
    PetscCall(MatShellGetContext(A, &ctx));
    PetscCall(VecGhostUpdateBegin(x, INSERT_VALUES, SCATTER_FORWARD));
    PetscCall(VecGhostUpdateEnd(x, INSERT_VALUES, SCATTER_FORWARD));
    Vec xl, yl;
    PetscCall(VecGhostGetLocalForm(x, &xl));
    PetscCall(VecGhostGetLocalForm(y, &yl));
    PetscInt n = 0;
    PetscCall(VecGetLocalSize(xl, &n));
    int st = IGA_OK;
    if (is_cuda(xl) && is_cuda(yl)) {
        const PetscScalar *xa;
        PetscScalar *ya;
        PetscCall(VecCUDAGetArrayRead(xl, &xa));
        PetscCall(VecCUDAGetArrayWrite(yl, &ya));
        st = iga_part_apply(ctx->part, xa, ya, nullptr);
        if (st == IGA_OK && cudaStreamSynchronize(nullptr) != cudaSuccess) st = IGA_ERR_CUDA;
        PetscCall(VecCUDARestoreArrayRead(xl, &xa));
        PetscCall(VecCUDARestoreArrayWrite(yl, &ya));
    } else {
        const PetscScalar *xa;
        PetscScalar *ya;
        double *dx = nullptr, *dy = nullptr;
        PetscCall(VecGetArrayRead(xl, &xa));
        PetscCall(VecGetArrayWrite(yl, &ya));
        const size_t bytes = sizeof(double) * (size_t)n;
        if (cudaMalloc((void **)&dx, bytes) != cudaSuccess || cudaMalloc((void **)&dy, bytes) != cudaSuccess ||
            cudaMemcpy(dx, xa, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
            st = IGA_ERR_CUDA;
        if (st == IGA_OK) st = iga_part_apply(ctx->part, dx, dy, nullptr);
        if (st == IGA_OK && cudaMemcpy(ya, dy, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) st = IGA_ERR_CUDA;
        cudaFree(dx);
        cudaFree(dy);
        PetscCall(VecRestoreArrayRead(xl, &xa));
        PetscCall(VecRestoreArrayWrite(yl, &ya));
    }
    PetscCall(VecGhostRestoreLocalForm(x, &xl));
    PetscCall(VecGhostRestoreLocalForm(y, &yl));
    if (st != IGA_OK) PetscCall(lib_error(A, st));
    // the ghost rows' partial sums to their owners
    PetscCall(VecGhostUpdateBegin(y, ADD_VALUES, SCATTER_REVERSE));
    PetscCall(VecGhostUpdateEnd(y, ADD_VALUES, SCATTER_REVERSE));
    PetscFunctionReturn(0);
}

extern "C" PetscErrorCode IgaMatShellDestroy(Mat A)
{
    IgaShellCtx *ctx = nullptr;
    PetscFunctionBeginUser;
    PetscCall(MatShellGetContext(A, &ctx));
    delete ctx;   // the plan / part stay the caller's
    PetscFunctionReturn(0);
}

// A shell matrix of nfunc rows on one rank over an existing plan (the plan
// keeps its sign and Dirichlet rule: the reference's -K with zero rows by
// default, iga_opts_default).
extern "C" PetscErrorCode IgaMatCreateShell(MPI_Comm comm, iga_plan *plan, Mat *A)
{
    PetscFunctionBeginUser;
    iga_plan_info info;
    if (iga_plan_get_info(plan, &info) != IGA_OK) SETERRQ(comm, PETSC_ERR_ARG_WRONG, "iga_b200: %s", iga_last_error());
    IgaShellCtx *ctx = new IgaShellCtx();
    ctx->plan = plan;
    const PetscInt n = (PetscInt)info.nfunc;
    PetscCall(MatCreateShell(comm, n, n, PETSC_DETERMINE, PETSC_DETERMINE, ctx, A));
    PetscCall(MatShellSetOperation(*A, MATOP_MULT, (void (*)(void))IgaMatMult));
    PetscCall(MatShellSetOperation(*A, MATOP_DESTROY, (void (*)(void))IgaMatShellDestroy));
    PetscFunctionReturn(0);
}

// A shell matrix of one rank's part (built with iga_part_build) for the
// reference's multi-rank drivers: local size nlocalfunc, vectors created with
// VecCreateGhost over the part's ghost list (the reference's MyMatCreateVecs).
extern "C" PetscErrorCode IgaMatCreateShellGhosted(MPI_Comm comm, iga_part *part, Mat *A)
{
    PetscFunctionBeginUser;
    iga_part_info info;
    if (iga_part_get_info(part, &info) != IGA_OK) SETERRQ(comm, PETSC_ERR_ARG_WRONG, "iga_b200: %s", iga_last_error());
    IgaShellCtx *ctx = new IgaShellCtx();
    ctx->part = part;
    ctx->nghost = info.nghost;
    const PetscInt n = info.nlocalfunc;
    PetscCall(MatCreateShell(comm, n, n, (PetscInt)info.nfunc_global, (PetscInt)info.nfunc_global, ctx, A));
    PetscCall(MatShellSetOperation(*A, MATOP_MULT, (void (*)(void))IgaMatMultGhosted));
    PetscCall(MatShellSetOperation(*A, MATOP_DESTROY, (void (*)(void))IgaMatShellDestroy));
    PetscFunctionReturn(0);
}

// Ghosted vectors of the part's layout (the reference's MyMatCreateVecs,
// matrix_free/iteration_number_fempc_mf.cpp:62-72).
extern "C" PetscErrorCode IgaPartCreateVec(MPI_Comm comm, iga_part *part, Vec *v)
{
    PetscFunctionBeginUser;
    iga_part_info info;
    if (iga_part_get_info(part, &info) != IGA_OK) SETERRQ(comm, PETSC_ERR_ARG_WRONG, "iga_b200: %s", iga_last_error());
    PetscInt *ghosts = nullptr;
    PetscCall(PetscMalloc1(info.nghost > 0 ? info.nghost : 1, &ghosts));
    {
        int64_t *g64 = new int64_t[info.nghost > 0 ? info.nghost : 1];
        const int st = iga_part_ghosts(part, g64);
        for (int i = 0; i < info.nghost; ++i) ghosts[i] = (PetscInt)g64[i];
        delete[] g64;
        if (st != IGA_OK) SETERRQ(comm, PETSC_ERR_LIB, "iga_b200: %s", iga_last_error());
    }
    PetscCall(VecCreateGhost(comm, info.nlocalfunc, PETSC_DETERMINE, info.nghost, ghosts, v));
    PetscCall(PetscFree(ghosts));
    PetscFunctionReturn(0);
}
