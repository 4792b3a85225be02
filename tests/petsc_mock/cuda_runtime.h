/* Host stand-ins for the CUDA runtime calls the PETSc adapter makes (device
 * memory is host memory here), so that the CPU adapter test needs no GPU.
 * Test infrastructure only. */
#ifndef PETSC_MOCK_CUDA_RUNTIME_H
#define PETSC_MOCK_CUDA_RUNTIME_H
#include <cstdlib>
#include <cstring>
typedef enum { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 } cudaError_t;
enum cudaMemcpyKind { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2 };
inline cudaError_t cudaMalloc(void **p, size_t n)
{
    *p = std::malloc(n ? n : 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline cudaError_t cudaFree(void *p)
{
    std::free(p);
    return cudaSuccess;
}
inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind)
{
    std::memcpy(d, s, n);
    return cudaSuccess;
}
inline cudaError_t cudaStreamSynchronize(void *) { return cudaSuccess; }
#endif
