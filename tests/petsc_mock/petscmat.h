/* A stand-in for the few PETSc declarations that
 * parallel-computing_b200/adapters/petsc_matshell.cpp uses, so that a CPU
 * test can compile the adapter and drive it without PETSc. Vectors are plain
 * host arrays; a "ghosted" vector keeps its owned entries and ghosts in one
 * local form; the calls record themselves in a log the test reads. Test
 * infrastructure only. */
#ifndef PETSC_MOCK_PETSCMAT_H
#define PETSC_MOCK_PETSCMAT_H
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

typedef int PetscErrorCode;
typedef int PetscInt;
typedef double PetscScalar;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef int MPI_Comm;
typedef enum { INSERT_VALUES, ADD_VALUES } InsertMode;
typedef enum { SCATTER_FORWARD, SCATTER_REVERSE } ScatterMode;
typedef enum { MATOP_MULT, MATOP_DESTROY } MatOperation;
typedef const char *VecType;
#define VECSEQCUDA "seqcuda"
#define VECMPICUDA "mpicuda"
#define VECCUDA "cuda"
#define PETSC_DETERMINE (-1)
#define PETSC_ERR_LIB 76
#define PETSC_ERR_ARG_WRONG 62

struct MockLog {
    std::vector<std::string> calls;
    void add(const std::string &s) { calls.push_back(s); }
};
inline MockLog &mock_log()
{
    static MockLog log;
    return log;
}

struct _p_Vec {
    std::string type = "seq";           // "seqcuda" marks a device vector
    std::vector<double> data;            // owned entries, then ghosts (ghosted vectors)
    int nowned = 0;
    std::vector<int> ghost_owner_index;  // owned index (of the same vector) each ghost mirrors
    _p_Vec *local = nullptr;             // local form: the same storage
};
typedef _p_Vec *Vec;

struct _p_Mat {
    MPI_Comm comm = 0;
    void *ctx = nullptr;
    PetscErrorCode (*mult)(_p_Mat *, Vec, Vec) = nullptr;
    PetscErrorCode (*destroy)(_p_Mat *) = nullptr;
    int m = 0, n = 0, M = 0, N = 0;
};
typedef _p_Mat *Mat;
typedef void *PetscObject;

#define PetscFunctionBeginUser do { } while (0)
#define PetscFunctionReturn(x) return (x)
#define PetscCall(x)                       \
    do {                                   \
        PetscErrorCode ierr_ = (x);        \
        if (ierr_) return ierr_;           \
    } while (0)
#define SETERRQ(comm, code, ...)                         \
    do {                                                 \
        char msg_[256];                                  \
        std::snprintf(msg_, sizeof msg_, __VA_ARGS__);   \
        mock_log().add(std::string("error: ") + msg_);   \
        return (code);                                   \
    } while (0)

inline PetscErrorCode PetscObjectGetComm(PetscObject, MPI_Comm *c)
{
    *c = 0;
    return 0;
}

inline PetscErrorCode PetscObjectTypeCompareAny(PetscObject obj, PetscBool *match, const char *first, ...)
{
    const std::string &t = static_cast<Vec>(obj)->type;
    *match = PETSC_FALSE;
    va_list ap;
    va_start(ap, first);
    for (const char *name = first; name && *name; name = va_arg(ap, const char *))
        if (t == name) *match = PETSC_TRUE;
    va_end(ap);
    return 0;
}

template <typename T>
inline PetscErrorCode MatShellGetContext(Mat A, T **ctx)
{
    *ctx = static_cast<T *>(A->ctx);
    return 0;
}
inline PetscErrorCode MatCreateShell(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt M, PetscInt N, void *ctx, Mat *A)
{
    *A = new _p_Mat();
    (*A)->comm = comm;
    (*A)->ctx = ctx;
    (*A)->m = m;
    (*A)->n = n;
    (*A)->M = M;
    (*A)->N = N;
    mock_log().add("MatCreateShell " + std::to_string(m) + " " + std::to_string(M));
    return 0;
}
inline PetscErrorCode MatShellSetOperation(Mat A, MatOperation op, void (*f)(void))
{
    if (op == MATOP_MULT) A->mult = reinterpret_cast<PetscErrorCode (*)(Mat, Vec, Vec)>(f);
    if (op == MATOP_DESTROY) A->destroy = reinterpret_cast<PetscErrorCode (*)(Mat)>(f);
    return 0;
}
inline PetscErrorCode MatMult(Mat A, Vec x, Vec y) { return A->mult(A, x, y); }
inline PetscErrorCode MatDestroy(Mat *A)
{
    PetscErrorCode e = (*A)->destroy ? (*A)->destroy(*A) : 0;
    delete *A;
    *A = nullptr;
    return e;
}

inline PetscErrorCode VecGetLocalSize(Vec v, PetscInt *n)
{
    *n = (PetscInt)v->data.size();
    return 0;
}
#define MOCK_ARRAY(name, tag, T)                       \
    inline PetscErrorCode name(Vec v, T **a)           \
    {                                                  \
        *a = v->data.data();                           \
        mock_log().add(tag);                           \
        return 0;                                      \
    }
MOCK_ARRAY(VecGetArrayRead, "VecGetArrayRead", const PetscScalar)
MOCK_ARRAY(VecRestoreArrayRead, "VecRestoreArrayRead", const PetscScalar)
MOCK_ARRAY(VecGetArrayWrite, "VecGetArrayWrite", PetscScalar)
MOCK_ARRAY(VecRestoreArrayWrite, "VecRestoreArrayWrite", PetscScalar)
MOCK_ARRAY(VecCUDAGetArrayRead, "VecCUDAGetArrayRead", const PetscScalar)
MOCK_ARRAY(VecCUDARestoreArrayRead, "VecCUDARestoreArrayRead", const PetscScalar)
MOCK_ARRAY(VecCUDAGetArrayWrite, "VecCUDAGetArrayWrite", PetscScalar)
MOCK_ARRAY(VecCUDARestoreArrayWrite, "VecCUDARestoreArrayWrite", PetscScalar)
#undef MOCK_ARRAY

// Ghost updates of one process: forward copies each ghost's owned value into
// the ghost slot, reverse adds the ghost slots into their owners and clears them.
inline PetscErrorCode VecGhostUpdateBegin(Vec v, InsertMode im, ScatterMode sm)
{
    mock_log().add(std::string("VecGhostUpdateBegin ") + (sm == SCATTER_FORWARD ? "forward" : "reverse") +
                   (im == ADD_VALUES ? " add" : " insert"));
    return 0;
}
inline PetscErrorCode VecGhostUpdateEnd(Vec v, InsertMode im, ScatterMode sm)
{
    for (size_t g = 0; g < v->ghost_owner_index.size(); ++g) {
        double &slot = v->data[v->nowned + g];
        double &owner = v->data[v->ghost_owner_index[g]];
        if (sm == SCATTER_FORWARD) slot = owner;
        else {
            owner += slot;
            slot = 0.0;
        }
    }
    mock_log().add("VecGhostUpdateEnd");
    return 0;
}
inline PetscErrorCode VecGhostGetLocalForm(Vec v, Vec *l)
{
    *l = v;   // the mock keeps owned entries and ghosts in one array
    return 0;
}
inline PetscErrorCode VecGhostRestoreLocalForm(Vec, Vec *l)
{
    *l = nullptr;
    return 0;
}
inline PetscErrorCode VecCreateGhost(MPI_Comm, PetscInt n, PetscInt, PetscInt nghost, const PetscInt *ghosts, Vec *v)
{
    *v = new _p_Vec();
    (*v)->nowned = n;
    (*v)->data.assign((size_t)(n + nghost), 0.0);
    std::string s = "VecCreateGhost " + std::to_string(n) + " " + std::to_string(nghost);
    for (PetscInt i = 0; i < nghost; ++i) s += " " + std::to_string(ghosts[i]);
    mock_log().add(s);
    return 0;
}
template <typename T>
inline PetscErrorCode PetscMalloc1(PetscInt n, T **p)
{
    *p = static_cast<T *>(std::malloc(sizeof(T) * (size_t)(n > 0 ? n : 1)));
    return 0;
}
template <typename T>
inline PetscErrorCode PetscFree(T *p)
{
    std::free(p);
    return 0;
}
#endif /* PETSC_MOCK_PETSCMAT_H */
