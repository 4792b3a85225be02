// Drives parallel-computing_b200/adapters/petsc_matshell.cpp against the
// PETSc stand-in (petscmat.h here) and fake library entry points that record
// their calls: the MATSHELL MatMult on device and host vectors, the status
// mapping, and the ghosted MatMult's order (forward ghost update, part
// apply, reverse add). Prints "ok" and exits 0 when every check holds.
// Test infrastructure only.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "petscmat.h"
#include "iga_mf.h"
#include "iga_part.h"

extern "C" {
PetscErrorCode IgaMatCreateShell(MPI_Comm comm, iga_plan *plan, Mat *A);
PetscErrorCode IgaMatCreateShellGhosted(MPI_Comm comm, iga_part *part, Mat *A);
PetscErrorCode IgaPartCreateVec(MPI_Comm comm, iga_part *part, Vec *v);
}

static int g_status = IGA_OK;

extern "C" {
int iga_plan_get_info(const iga_plan *, iga_plan_info *info)
{
    *info = iga_plan_info{};
    info->nfunc = 5;
    return IGA_OK;
}
int iga_apply(iga_plan *, const void *x, void *y, void *)
{
    mock_log().add("iga_apply");
    for (int i = 0; i < 5; ++i) static_cast<double *>(y)[i] = -2.0 * static_cast<const double *>(x)[i];
    return g_status;
}
int iga_apply_host(iga_plan *, const double *x, double *y)
{
    mock_log().add("iga_apply_host");
    for (int i = 0; i < 5; ++i) y[i] = -2.0 * x[i];
    return g_status;
}
int iga_part_get_info(const iga_part *, iga_part_info *info)
{
    *info = iga_part_info{};
    info->nlocalfunc = 3;
    info->nghost = 2;
    info->nfunc_global = 10;
    return IGA_OK;
}
int iga_part_ghosts(const iga_part *, int64_t *g)
{
    g[0] = 7;
    g[1] = 8;
    return IGA_OK;
}
int iga_part_apply(iga_part *, const double *x, double *y, void *)
{
    mock_log().add("iga_part_apply");
    for (int i = 0; i < 5; ++i) y[i] = x[i];   // every local-form row its own value
    return g_status;
}
const char *iga_last_error(void) { return "fake failure"; }
}

static int failures = 0;
static void check(bool ok, const char *what)
{
    if (!ok) {
        std::printf("FAIL: %s\n", what);
        ++failures;
    }
}
static int find(const std::string &s)
{
    const auto &c = mock_log().calls;
    for (size_t i = 0; i < c.size(); ++i)
        if (c[i].find(s) == 0) return (int)i;
    return -1;
}

int main()
{
    int dummy_plan = 0, dummy_part = 0;
    iga_plan *plan = reinterpret_cast<iga_plan *>(&dummy_plan);
    iga_part *part = reinterpret_cast<iga_part *>(&dummy_part);

    // 1. device vectors: the device arrays go to iga_apply
    Mat A;
    check(IgaMatCreateShell(0, plan, &A) == 0, "create shell");
    check(A->m == 5, "shell local size = nfunc");
    _p_Vec x, y;
    x.type = y.type = "seqcuda";
    x.data = {1, 2, 3, 4, 5};
    y.data.assign(5, 0.0);
    mock_log().calls.clear();
    check(MatMult(A, &x, &y) == 0, "MatMult on device vectors");
    check(find("VecCUDAGetArrayRead") >= 0 && find("iga_apply") >= 0 && find("VecGetArrayRead") < 0,
          "device arrays and iga_apply");
    check(y.data[4] == -10.0, "y = A x");

    // 2. host vectors: iga_apply_host
    x.type = y.type = "seq";
    mock_log().calls.clear();
    check(MatMult(A, &x, &y) == 0, "MatMult on host vectors");
    check(find("iga_apply_host") >= 0 && find("VecCUDAGetArrayRead") < 0, "host arrays and iga_apply_host");

    // 3. a failing call becomes PETSC_ERR_LIB with the library's message
    g_status = IGA_ERR_ARG;
    mock_log().calls.clear();
    check(MatMult(A, &x, &y) == PETSC_ERR_LIB, "error status mapped to PETSC_ERR_LIB");
    check(find("error: iga_b200 status") >= 0 && mock_log().calls.back().find("fake failure") != std::string::npos,
          "error message carries the library's text");
    g_status = IGA_OK;
    check(MatDestroy(&A) == 0, "destroy shell");

    // 4. ghosted layout: forward update, part apply on the local forms, reverse add
    Mat G;
    check(IgaMatCreateShellGhosted(0, part, &G) == 0, "create ghosted shell");
    check(G->m == 3 && G->M == 10, "ghosted shell sizes");
    _p_Vec gx, gy;
    gx.nowned = gy.nowned = 3;
    gx.ghost_owner_index = gy.ghost_owner_index = {0, 2};
    gx.data = {1, 2, 3, 0, 0};
    gy.data.assign(5, 0.0);
    mock_log().calls.clear();
    check(MatMult(G, &gx, &gy) == 0, "ghosted MatMult");
    const int f = find("VecGhostUpdateBegin forward insert"), a = find("iga_part_apply"),
              r = find("VecGhostUpdateBegin reverse add");
    check(f >= 0 && a > f && r > a, "forward update, part apply, reverse add, in that order");
    check(gy.data[0] == 2.0 && gy.data[1] == 2.0 && gy.data[2] == 6.0, "ghost rows added to their owners");
    check(gy.data[3] == 0.0 && gy.data[4] == 0.0, "ghost slots cleared by the reverse add");
    check(MatDestroy(&G) == 0, "destroy ghosted shell");

    // 5. ghosted vectors of the part's layout
    Vec v = nullptr;
    mock_log().calls.clear();
    check(IgaPartCreateVec(0, part, &v) == 0, "create ghosted vector");
    check(find("VecCreateGhost 3 2 7 8") >= 0, "owned size, ghost count and ghost indices");
    delete v;

    if (failures) return 1;
    std::printf("ok\n");
    return 0;
}
