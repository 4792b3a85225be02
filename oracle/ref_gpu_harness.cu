// Test infrastructure only: drives the reference's own GPU MatMult kernel
// (matrix_free_gpu/src/mult.cu, MatrixFreeMatMultCUDA, compiled in place
// from the reference tree with P_ORDER = Q_ORDER = 3 by `make -C oracle
// refgpu`) with its mesh tables uploaded once, for parity checks and for the
// "reference GPU kernel on the same box" timing. Nothing of the product calls
// this library.
//
// The reference's GlobalAssemblyMF::MatMulMF (matrix_free_gpu/src/
// GlobalAssemblyMF.cu:126-242) uploads every table on every call, zeroes y,
// runs the kernel and zeroes y[Dir]; here the uploads happen once, y is zeroed
// on the device, and the Dirichlet rows stay zero because the kernel skips
// rows with ID < 0 (the reference's DirichletBCCUDA is not called: it is
// handed a host pointer, GlobalAssemblyMF.cu:227).
#include <cuda_runtime.h>

#include <cstring>

#include "mult.cuh"

namespace {
struct RefGpu {
    int p, nex, ney;
    double *B1, *B2, *dB1, *dB2, *C1, *C2, *h1, *h2, *CP, *qw1, *qw2;
    int *IEN, *ID;
};

template <typename T>
int up(T **dst, const T *src, size_t n)
{
    if (cudaMalloc((void **)dst, n * sizeof(T)) != cudaSuccess) return 1;
    return cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess;
}
}  // namespace

extern "C" {

int refgpu_destroy(void *h);

// Host arrays in the reference's layouts: B, dB [(p+1) qps][(p+1)] Bernstein
// values / derivatives at the Gauss points, qw [p+1], C1 [nex (p+1)^2],
// C2 [ney (p+1)^2], h1 [nex], h2 [ney], IEN [nex ney (p+1)^2], ID [N],
// CP [2N] (x, y interleaved).
int refgpu_create(int p, int nex, int ney, const double *B, const double *dB, const double *qw, const double *C1,
                  const double *C2, const double *h1, const double *h2, const int *IEN, const int *ID,
                  const double *CP, void **out)
{
    if (p != P_ORDER || !out) return 1;
    RefGpu *r = new RefGpu{};
    r->p = p;
    r->nex = nex;
    r->ney = ney;
    const size_t nb = (size_t)(p + 1) * (p + 1), N = (size_t)(nex + p) * (ney + p);
    int e = up(&r->B1, B, nb) | up(&r->B2, B, nb) | up(&r->dB1, dB, nb) | up(&r->dB2, dB, nb) |
            up(&r->C1, C1, nb * nex) | up(&r->C2, C2, nb * ney) | up(&r->h1, h1, (size_t)nex) |
            up(&r->h2, h2, (size_t)ney) | up(&r->CP, CP, 2 * N) | up(&r->qw1, qw, (size_t)p + 1) |
            up(&r->qw2, qw, (size_t)p + 1) | up(&r->IEN, IEN, nb * nex * ney) | up(&r->ID, ID, N);
    *out = e ? nullptr : r;
    if (e) refgpu_destroy(r);
    return e;
}

// y = A_ref x (device arrays of N doubles): y zeroed, then the reference's
// MatrixFreeMatMultCUDA (its kernel, then cudaDeviceSynchronize).
int refgpu_apply(void *h, const double *d_in, double *d_out)
{
    RefGpu *r = (RefGpu *)h;
    const size_t N = (size_t)(r->nex + r->p) * (r->ney + r->p);
    if (cudaMemset(d_out, 0, N * sizeof(double)) != cudaSuccess) return 1;
    MatrixFreeMatMultCUDA(r->p, r->p, r->nex, r->ney, r->B1, r->B2, r->dB1, r->dB2, r->C1, r->C2, r->h1, r->h2,
                          r->IEN, r->ID, r->CP, r->qw1, r->qw2, d_in, d_out);
    return cudaGetLastError() != cudaSuccess;
}

int refgpu_destroy(void *h)
{
    RefGpu *r = (RefGpu *)h;
    if (!r) return 0;
    void *ps[] = {r->B1, r->B2, r->dB1, r->dB2, r->C1, r->C2, r->h1, r->h2, r->CP, r->qw1, r->qw2, r->IEN, r->ID};
    for (void *q : ps)
        if (q) cudaFree(q);
    delete r;
    return 0;
}

}  // extern "C"
