// Device-resident flexible PCG for K u = b with the bilinear-FEM
// preconditioner (include/iga_solve.h).
//
// Reference loop (matrix_free/iteration_number_fempc_mf.cpp:193-233): PETSc
// KSPSolve on the MATSHELL operator, PCSHELL apply = inner KSPCG + PCJACOBI on
// the FEM matrix to rtol = abstol = 1e-10 (:210-224). Here every vector, every
// scalar (alpha, beta, dot products) and every convergence test lives on the
// device; the host only reads one flag per outer iteration. All reductions
// are deterministic (fixed-order block partials, summed by the last block).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <random>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/iga_solve.h"
#include "iga_fastdiag.hpp"
#include "iga_fem.hpp"
#include "iga_gemm.hpp"
#include "iga_plan.hpp"

namespace iga {

constexpr int kRedBlocks = 592;   // fixed grid of every reduction kernel (4 x 148 SMs)
constexpr int kThreads = 256;
constexpr int kChunk = 16;        // inner CG iterations per captured graph

struct DevScalars {
    double alpha, beta, rz, rzo, rr, rr0, tol2, bb; // outer PCG (rzo = r_new . z_old)
    double ialpha, ibeta, irz, irr, itol2;          // inner FEM-CG
    int done, breakdown, idone, iiters, ibreak, imax;
    int err;                                        // a bounded wait in a kernel gave up
    int it, maxit;                                  // outer PCG in a device-side loop
};

// ------------------------------------------------------------ reductions
// Block sums of K values; the last block to finish sums the per-block
// partials in block order and returns true (thread 0 holds the totals).
template <int K>
__device__ bool reduce_last(double (&v)[K], double *partials, unsigned *counter, double (&tot)[K])
{
    __shared__ double sh[K][kThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = v[k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) sh[k][wid] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) s += sh[k][w];
            partials[blockIdx.x * K + k] = s;
        }
        __threadfence();
        const unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // Last block: every thread sums a fixed subset of the partials in block
    // order, then a fixed-shape tree (warp shuffles, then warp 0) combines them.
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += kThreads) s += ((volatile double *)partials)[b * K + k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) sh[k][wid] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) s += sh[k][w];
            tot[k] = s;
        }
        *counter = 0u;
    }
    return true;
}

__device__ __forceinline__ bool bnd(int i, int j, int m, int n) { return i == 0 || j == 0 || i == m - 1 || j == n - 1; }

// ------------------------------------------------------------ FEM stencil
// K_fem = Kx (x) My + Mx (x) Ky on the free nodes (1-D linear-element
// stiffness K and mass M from the node coordinates; the 2x2-Gauss bilinear
// element matrices of matrix_free/src/ElementFEM.cpp:3-117 are exactly these
// tensor products), identity rows on the boundary.
template <typename T>
struct FemCoef {
    const T *kd, *ko, *md, *mo;   // x: diag / off-diagonal (i,i+1)
    const T *ld, *lo, *nd, *no;   // y: stiffness diag / off, mass diag / off
    int m, n;
};

template <typename T>
__device__ __forceinline__ T fem_row(const T *__restrict__ p, int i, int j, const FemCoef<T> &c)
{
    const T kx[3] = {c.ko[i - 1], c.kd[i], c.ko[i]}, mx[3] = {c.mo[i - 1], c.md[i], c.mo[i]};
    const T ky[3] = {c.lo[j - 1], c.ld[j], c.lo[j]}, my[3] = {c.no[j - 1], c.nd[j], c.no[j]};
    const bool xl = i - 1 >= 1, xr = i + 1 <= c.m - 2, yl = j - 1 >= 1, yr = j + 1 <= c.n - 2;
    T s = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        if ((b == 0 && !yl) || (b == 2 && !yr)) continue;
        const T *row = p + (size_t)(j + b - 1) * c.m;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if ((a == 0 && !xl) || (a == 2 && !xr)) continue;
            s += (kx[a] * my[b] + mx[a] * ky[b]) * row[i + a - 1];
        }
    }
    return s;
}

template <typename T>
__device__ __forceinline__ T fem_diag(int i, int j, const FemCoef<T> &c)
{
    return c.kd[i] * c.nd[j] + c.md[i] * c.ld[j];
}

template <typename T>
__global__ void fem_apply_kernel(const T *__restrict__ x, T *__restrict__ y, FemCoef<T> c)
{
    const long long N = (long long)c.m * c.n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % c.m), j = (int)(t / c.m);
        y[t] = bnd(i, j, c.m, c.n) ? x[t] : fem_row(x, i, j, c);
    }
}

// CSR rows of the FEM matrix (sorted columns); rowptr precomputed on the host.
__global__ void fem_csr_kernel(const int32_t *__restrict__ rowptr, int32_t *__restrict__ col, double *__restrict__ val,
                               FemCoef<double> c, double sign)
{
    const long long N = (long long)c.m * c.n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % c.m), j = (int)(t / c.m);
        int k = rowptr[t];
        if (bnd(i, j, c.m, c.n)) {
            col[k] = (int32_t)t;
            val[k] = 1.0;
            continue;
        }
        const double kx[3] = {c.ko[i - 1], c.kd[i], c.ko[i]}, mx[3] = {c.mo[i - 1], c.md[i], c.mo[i]};
        const double ky[3] = {c.lo[j - 1], c.ld[j], c.lo[j]}, my[3] = {c.no[j - 1], c.nd[j], c.no[j]};
        for (int b = 0; b < 3; ++b) {
            const int jj = j + b - 1;
            if (jj < 1 || jj > c.n - 2) continue;
            for (int a = 0; a < 3; ++a) {
                const int ii = i + a - 1;
                if (ii < 1 || ii > c.m - 2) continue;
                col[k] = (int32_t)((long long)jj * c.m + ii);
                val[k] = sign * (kx[a] * my[b] + mx[a] * ky[b]);
                ++k;
            }
        }
    }
}

// ------------------------------------------------------------ inner FEM-CG (the PC apply)
// Jacobi-preconditioned CG on K_fem z = r_in to ||r|| <= pc_rtol ||r_in||.
template <typename T>
struct InnerCG {
    T *z, *r, *p, *q;
    const T *rhs;
    FemCoef<T> c;
    DevScalars *s;
    double *partials;
    unsigned *counter;
};

template <typename T>
__global__ void icg_init_kernel(InnerCG<T> a, const T *__restrict__ rhs, double rtol, int maxit)
{
    const long long N = (long long)a.c.m * a.c.n;
    double v[2] = {0.0, 0.0};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % a.c.m), j = (int)(t / a.c.m);
        const T r = rhs[t];
        const T d = bnd(i, j, a.c.m, a.c.n) ? T(1) : fem_diag(i, j, a.c);
        const T zz = r / d;
        a.z[t] = 0;
        a.r[t] = r;
        a.p[t] = zz;
        v[0] += (double)r * (double)zz;
        v[1] += (double)r * (double)r;
    }
    double tot[2];
    if (reduce_last<2>(v, a.partials, a.counter, tot) && threadIdx.x == 0) {
        a.s->irz = tot[0];
        a.s->irr = tot[1];
        a.s->itol2 = rtol * rtol * tot[1];
        a.s->iiters = 0;
        a.s->imax = maxit;
        a.s->ibreak = 0;
        a.s->idone = (tot[1] == 0.0) ? 1 : 0;
    }
}

template <typename T>
__global__ void icg_q_kernel(InnerCG<T> a)
{
    if (a.s->idone) return;
    const long long N = (long long)a.c.m * a.c.n;
    double v[1] = {0.0};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % a.c.m), j = (int)(t / a.c.m);
        const T pv = a.p[t];
        const T qv = bnd(i, j, a.c.m, a.c.n) ? pv : fem_row(a.p, i, j, a.c);
        a.q[t] = qv;
        v[0] += (double)pv * (double)qv;
    }
    double tot[1];
    if (reduce_last<1>(v, a.partials, a.counter, tot) && threadIdx.x == 0) {
        if (!(tot[0] > 0.0)) {
            a.s->ibreak = 1;
            a.s->idone = 1;
        } else {
            a.s->ialpha = a.s->irz / tot[0];
        }
    }
}

template <typename T>
__global__ void icg_update_kernel(InnerCG<T> a)
{
    if (a.s->idone) return;
    const long long N = (long long)a.c.m * a.c.n;
    const T al = (T)a.s->ialpha;
    double v[2] = {0.0, 0.0};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % a.c.m), j = (int)(t / a.c.m);
        a.z[t] += al * a.p[t];
        const T r = a.r[t] - al * a.q[t];
        a.r[t] = r;
        const T d = bnd(i, j, a.c.m, a.c.n) ? T(1) : fem_diag(i, j, a.c);
        v[0] += (double)r * (double)(r / d);
        v[1] += (double)r * (double)r;
    }
    double tot[2];
    if (reduce_last<2>(v, a.partials, a.counter, tot) && threadIdx.x == 0) {
        a.s->ibeta = tot[0] / a.s->irz;
        a.s->irz = tot[0];
        a.s->irr = tot[1];
        a.s->iiters += 1;
        if (tot[1] <= a.s->itol2 || a.s->iiters >= a.s->imax || !(tot[1] == tot[1])) a.s->idone = 1;
    }
}

template <typename T>
__global__ void icg_p_kernel(InnerCG<T> a)
{
    if (a.s->idone) return;
    const long long N = (long long)a.c.m * a.c.n;
    const T be = (T)a.s->ibeta;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % a.c.m), j = (int)(t / a.c.m);
        const T d = bnd(i, j, a.c.m, a.c.n) ? T(1) : fem_diag(i, j, a.c);
        a.p[t] = a.r[t] / d + be * a.p[t];
    }
}

// ------------------------------------------------------------ outer PCG vector kernels
// Elementwise loops move 16 bytes per access (4 floats / 2 doubles) when every
// array of the kernel starts on a 16-byte boundary; the last N % VN entries
// (or all of them, for unaligned arrays) take scalar accesses. The thread that
// handles an entry depends only on N and the grid, so the reductions stay
// deterministic.
template <typename T>
struct alignas(16) Pk {
    static constexpr int n = 16 / sizeof(T);
    T v[n];
};

template <typename T>
__device__ __forceinline__ Pk<T> ldp(const T *a, long long i)
{
    return *reinterpret_cast<const Pk<T> *>(a + i);
}

template <typename T>
__device__ __forceinline__ void stp(T *a, long long i, const Pk<T> &v)
{
    *reinterpret_cast<Pk<T> *>(a + i) = v;
}

__device__ __forceinline__ bool al16(const void *a) { return ((uintptr_t)a & 15u) == 0; }

// Calls f(i, c) for the first entry i and count c of every pack this thread
// owns, then f(i, 1) for its scalar tail entries.
template <typename T, typename F>
__device__ __forceinline__ void vloop(long long N, bool vec, F &&f)
{
    constexpr int VN = Pk<T>::n;
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x, st = (long long)gridDim.x * blockDim.x;
    const long long nv = vec ? N / VN : 0;
    for (long long k = g; k < nv; k += st) f(k * VN, VN);
    for (long long i = nv * VN + g; i < N; i += st) f(i, 1);
}

// Loads c entries (a pack or one scalar) starting at i.
template <typename T>
__device__ __forceinline__ Pk<T> ldc(const T *a, long long i, int c)
{
    if (c > 1) return ldp(a, i);
    Pk<T> v;
    v.v[0] = a[i];
    return v;
}

template <typename T>
__device__ __forceinline__ void stc(T *a, long long i, int c, const Pk<T> &v)
{
    if (c > 1) stp(a, i, v);
    else a[i] = v.v[0];
}

template <typename T>
__global__ void dot_kernel(const T *__restrict__ a, const T *__restrict__ b, long long N, double *out, double *partials,
                           unsigned *counter)
{
    double v[1] = {0.0};
    vloop<T>(N, al16(a) && al16(b), [&](long long i, int c) {
        const Pk<T> x = ldc(a, i, c), y = ldc(b, i, c);
#pragma unroll
        for (int k = 0; k < Pk<T>::n; ++k)
            if (k < c) v[0] += (double)x.v[k] * (double)y.v[k];
    });
    double tot[1];
    if (reduce_last<1>(v, partials, counter, tot) && threadIdx.x == 0) *out = tot[0];
}

// alpha = rz / (p.q) from the device scalars
template <typename T>
__global__ void pcg_pq_kernel(const T *__restrict__ p, const T *__restrict__ q, long long N, DevScalars *s,
                              double *partials, unsigned *counter)
{
    pdl_begin();
    double v[1] = {0.0};
    vloop<T>(N, al16(p) && al16(q), [&](long long i, int c) {
        const Pk<T> a = ldc(p, i, c), b = ldc(q, i, c);
#pragma unroll
        for (int k = 0; k < Pk<T>::n; ++k)
            if (k < c) v[0] += (double)a.v[k] * (double)b.v[k];
    });
    double tot[1];
    if (reduce_last<1>(v, partials, counter, tot) && threadIdx.x == 0) {
        if (!(tot[0] > 0.0)) {
            s->breakdown = 1;
            s->alpha = 0.0;
        } else {
            s->alpha = s->rz / tot[0];
        }
    }
}

// x += alpha p, r -= alpha q; rr = r.r and rzo = r.z with the previous
// preconditioned residual z (the flexible beta's correction term, taken here
// so that z need not be kept). Returns the totals to the last block.
template <typename T>
__device__ __forceinline__ bool xr_update(T *__restrict__ x, T *__restrict__ r, const T *__restrict__ p,
                                          const T *__restrict__ q, const T *__restrict__ z, long long N,
                                          const DevScalars *s, double *partials, unsigned *counter, double (&tot)[2])
{
    const T al = (T)s->alpha;
    double v[2] = {0.0, 0.0};
    vloop<T>(N, al16(x) && al16(r) && al16(p) && al16(q) && al16(z), [&](long long i, int c) {
        Pk<T> xv = ldc(x, i, c), rv = ldc(r, i, c);
        const Pk<T> pv = ldc(p, i, c), qv = ldc(q, i, c), zv = ldc(z, i, c);
#pragma unroll
        for (int k = 0; k < Pk<T>::n; ++k) {
            if (k < c) {
                xv.v[k] += al * pv.v[k];
                rv.v[k] -= al * qv.v[k];
                v[0] += (double)rv.v[k] * (double)rv.v[k];
                v[1] += (double)rv.v[k] * (double)zv.v[k];
            }
        }
        stc(x, i, c, xv);
        stc(r, i, c, rv);
    });
    return reduce_last<2>(v, partials, counter, tot);
}

template <typename T>
__global__ void pcg_xr_kernel(T *__restrict__ x, T *__restrict__ r, const T *__restrict__ p, const T *__restrict__ q,
                              const T *__restrict__ z, long long N, DevScalars *s, double *partials, unsigned *counter)
{
    double tot[2];
    if (xr_update(x, r, p, q, z, N, s, partials, counter, tot) && threadIdx.x == 0) {
        s->rr = tot[0];
        s->rzo = tot[1];
    }
}

// Same update inside the device-side loop: counts the iteration and sets the
// loop's condition (continue while rr > tol2, it < maxit, no breakdown, finite).
template <typename T>
__global__ void pcg_xr_cond_kernel(T *__restrict__ x, T *__restrict__ r, const T *__restrict__ p,
                                   const T *__restrict__ q, const T *__restrict__ z, long long N, DevScalars *s,
                                   double *partials, unsigned *counter, cudaGraphConditionalHandle h)
{
    pdl_begin();
    double tot[2];
    if (xr_update(x, r, p, q, z, N, s, partials, counter, tot) && threadIdx.x == 0) {
        s->rr = tot[0];
        s->rzo = tot[1];
        s->it += 1;
        const bool go = tot[0] > s->tol2 && s->it < s->maxit && !s->breakdown && tot[0] == tot[0];
        cudaGraphSetConditional(h, go ? 1u : 0u);
    }
}

__global__ void loop_init_kernel(DevScalars *s, double tol2, int maxit)
{
    s->tol2 = tol2;
    s->maxit = maxit;
    s->it = 0;
    s->breakdown = 0;
}

// Flexible (Polak-Ribiere) beta = r.(z - z_old) / rz_old with r.z_old = rzo
// from the update kernel; rz = r.z.
template <typename T>
__global__ void pcg_beta_kernel(const T *__restrict__ r, const T *__restrict__ z, long long N, DevScalars *s,
                                double *partials, unsigned *counter)
{
    pdl_begin();
    double v[1] = {0.0};
    vloop<T>(N, al16(r) && al16(z), [&](long long i, int c) {
        const Pk<T> a = ldc(r, i, c), b = ldc(z, i, c);
#pragma unroll
        for (int k = 0; k < Pk<T>::n; ++k)
            if (k < c) v[0] += (double)a.v[k] * (double)b.v[k];
    });
    double tot[1];
    if (reduce_last<1>(v, partials, counter, tot) && threadIdx.x == 0) {
        s->beta = (tot[0] - s->rzo) / s->rz;
        s->rz = tot[0];
    }
}

template <typename T>
__global__ void pcg_p_kernel(T *__restrict__ p, const T *__restrict__ z, long long N, const DevScalars *s, int first)
{
    pdl_begin();
    const T be = first ? T(0) : (T)s->beta;
    vloop<T>(N, al16(p) && al16(z), [&](long long i, int c) {
        const Pk<T> zv = ldc(z, i, c);
        if (first) {   // the first direction never reads stale p
            stc(p, i, c, zv);
            return;
        }
        Pk<T> pv = ldc(p, i, c);
#pragma unroll
        for (int k = 0; k < Pk<T>::n; ++k) pv.v[k] = zv.v[k] + be * pv.v[k];
        stc(p, i, c, pv);
    });
}

// r = b - Ax (FP64), rr = r.r, bb = b.b
__global__ void residual_kernel(const double *__restrict__ b, const double *__restrict__ Ax, double *__restrict__ r,
                                long long N, DevScalars *s, double *partials, unsigned *counter)
{
    double v[2] = {0.0, 0.0};
    vloop<double>(N, al16(b) && al16(Ax) && al16(r), [&](long long i, int c) {
        const Pk<double> bv = ldc(b, i, c), av = ldc(Ax, i, c);
        Pk<double> rv;
#pragma unroll
        for (int k = 0; k < Pk<double>::n; ++k) {
            rv.v[k] = bv.v[k] - av.v[k];
            if (k < c) {
                v[0] += rv.v[k] * rv.v[k];
                v[1] += bv.v[k] * bv.v[k];
            }
        }
        stc(r, i, c, rv);
    });
    double tot[2];
    if (reduce_last<2>(v, partials, counter, tot) && threadIdx.x == 0) {
        s->rr = tot[0];
        s->bb = tot[1];
    }
}

// r = b - q, rr = r.r
template <typename T>
__global__ void sub_kernel(const T *__restrict__ b, const T *__restrict__ q, T *__restrict__ r, long long N,
                           DevScalars *s, double *partials, unsigned *counter)
{
    double v[1] = {0.0};
    vloop<T>(N, al16(b) && al16(q) && al16(r), [&](long long i, int c) {
        const Pk<T> bv = ldc(b, i, c), qv = ldc(q, i, c);
        Pk<T> rv;
#pragma unroll
        for (int k = 0; k < Pk<T>::n; ++k) {
            rv.v[k] = bv.v[k] - qv.v[k];
            if (k < c) v[0] += (double)rv.v[k] * (double)rv.v[k];
        }
        stc(r, i, c, rv);
    });
    double tot[1];
    if (reduce_last<1>(v, partials, counter, tot) && threadIdx.x == 0) s->rr = tot[0];
}

template <typename T>
__global__ void copy_kernel(T *__restrict__ dst, const T *__restrict__ src, long long N)
{
    pdl_begin();
    vloop<T>(N, al16(dst) && al16(src), [&](long long i, int c) { stc(dst, i, c, ldc(src, i, c)); });
}

template <typename T>
__global__ void zero_kernel(T *__restrict__ dst, long long N)
{
    Pk<T> zv;
#pragma unroll
    for (int k = 0; k < Pk<T>::n; ++k) zv.v[k] = T(0);
    vloop<T>(N, al16(dst), [&](long long i, int c) { stc(dst, i, c, zv); });
}

// FP32 sweep right-hand side r32 = r64 / scale.
__global__ void scale_down_kernel(const double *__restrict__ r, float *__restrict__ r32, long long N, const DevScalars *s)
{
    const double inv = s->rr > 0.0 ? 1.0 / sqrt(s->rr) : 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x)
        r32[t] = (float)(r[t] * inv);
}

// Refinement update x64 += scale * d32 (scale = ||r64|| of the sweep's rhs).
__global__ void refine_update_kernel(double *__restrict__ x, const float *__restrict__ d, long long N, double scale)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x)
        x[t] += scale * (double)d[t];
}

// Scale of an FP64 vector carried through an FP32 preconditioner: the input
// is divided by ||r|| (rr = r.r of the current residual) on the way down and
// the output multiplied by it on the way up, so FP32's exponent range holds
// any residual size. 1 when rr is zero or not finite.
__device__ __forceinline__ double pc_scale(const DevScalars *s)
{
    const double rr = s->rr;
    return (rr > 0.0 && rr < 1e300) ? sqrt(rr) : 1.0;
}

__global__ void to_fp32_kernel(const double *__restrict__ r, float *__restrict__ r32, long long N, const DevScalars *s)
{
    pdl_begin();
    const double inv = 1.0 / pc_scale(s);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x)
        r32[t] = (float)(r[t] * inv);
}

__global__ void from_fp32_kernel(const float *__restrict__ z32, double *__restrict__ z, long long N, const DevScalars *s)
{
    pdl_begin();
    const double sc = pc_scale(s);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x)
        z[t] = sc * (double)z32[t];
}

// ------------------------------------------------------------ exact FEM inverse (fast diagonalisation)
// ---- tridiagonal solves along y of the x-diagonalised FEM system
// For every x mode a < nx: (lx[a] My + Ky) t = w, w = column a of the nyp x nxp
// matrix Wt (y contiguous: element (b, a) at b + a nyp), in place. The LDL^T
// factors are precomputed per mode in the same layout: Lf_b = e_{b-1} / d_{b-1}
// (the unit lower factor's subdiagonal, Lf_0 = 0) and Dv_b = 1 / d_b, so
//   forward  u_b = w_b - Lf_b u_{b-1},       v_b = Dv_b u_b,
//   backward x_b = v_b - Lf_{b+1} x_{b+1}    (no term past the last free row).
// One warp per mode: lane l owns rows [l s, l s + s) with s odd, so that the
// lanes' shared-memory accesses fall in distinct banks. Each recurrence is
// composed per lane into an affine map c -> E + P c, the maps are combined by
// a warp shuffle scan, and each lane then runs its rows from its carry-in.
// Arithmetic in T. STAGED: the mode's column and factors are brought into
// shared memory by the bulk-copy engine and the result is written back with
// 16-byte stores; else (columns too long for shared memory) the kernel works
// on them in place.
constexpr int kTriMaxWarps = 16;

// inclusive scan of affine maps over lanes, lane order (forward) or reverse lane order
template <typename R>
__device__ __forceinline__ void affine_scan(R &E, R &P, int lane, bool reverse)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const R pe = reverse ? __shfl_down_sync(0xffffffffu, E, o) : __shfl_up_sync(0xffffffffu, E, o);
        const R pp = reverse ? __shfl_down_sync(0xffffffffu, P, o) : __shfl_up_sync(0xffffffffu, P, o);
        if (reverse ? lane + o < 32 : lane >= o) {
            E = E + P * pe;
            P = P * pp;
        }
    }
}

template <typename T, bool STAGED>
__global__ void __launch_bounds__(kTriMaxWarps * 32)
fd_tri_kernel(T *__restrict__ W, const T *__restrict__ Lf, const T *__restrict__ Dv, int nx, int ny, int nyp, int seg,
              DevScalars *sc)
{
    pdl_launch();
    extern __shared__ __align__(16) unsigned char tri_smem[];
    __shared__ uint64_t bar[kTriMaxWarps];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T *wb = nullptr, *lb = nullptr, *db = nullptr;
    if constexpr (STAGED) {
        wb = reinterpret_cast<T *>(tri_smem) + (size_t)wid * 3 * nyp;
        lb = wb + nyp;
        db = lb + nyp;
        if (lane == 0) mbar_init(&bar[wid], 1);
        fence_mbar_init();
        __syncwarp();
    }
    uint32_t phase = 0;
    const int b0 = lane * seg, b1 = min(b0 + seg, ny);
    const uint32_t bytes = (uint32_t)nyp * (uint32_t)sizeof(T);
    const int a0 = blockIdx.x * nw + wid;
    // the first mode's factors (constant) are requested before the wait for
    // the preceding grid, its column of W after it
    if (STAGED && lane == 0 && a0 < nx) {
        mbar_arrive_expect_tx(&bar[wid], 3u * bytes);
        bulk_g2s(lb, Lf + (size_t)a0 * nyp, bytes, &bar[wid]);
        bulk_g2s(db, Dv + (size_t)a0 * nyp, bytes, &bar[wid]);
    }
    pdl_wait();
    for (int a = a0; a < nx; a += gridDim.x * nw) {
        T *wg = W + (size_t)a * nyp;
        const T *lg = Lf + (size_t)a * nyp, *dg = Dv + (size_t)a * nyp;
        T *wp;
        const T *lp, *dp;
        if constexpr (STAGED) {
            if (lane == 0) {
                if (a != a0) {
                    mbar_arrive_expect_tx(&bar[wid], 3u * bytes);
                    bulk_g2s(lb, lg, bytes, &bar[wid]);
                    bulk_g2s(db, dg, bytes, &bar[wid]);
                }
                bulk_g2s(wb, wg, bytes, &bar[wid]);
            }
            if (!mbar_wait_bounded(&bar[wid], phase)) {
                if (lane == 0) sc->err = 1;
                mbar_wait_bounded(&bar[wid], phase);   // let the copies land before leaving
                return;
            }
            phase ^= 1u;
            wp = wb;
            lp = lb;
            dp = db;
        } else {
            wp = wg;
            lp = lg;
            dp = dg;
        }
        // forward: this lane's map, the scan, then its rows from the carry-in
        T E = 0, P = 1;
#pragma unroll 4
        for (int b = b0; b < b1; ++b) {
            const T l = lp[b];
            E = wp[b] - l * E;
            P = -l * P;
        }
        affine_scan(E, P, lane, false);
        T u = __shfl_up_sync(0xffffffffu, E, 1);
        if (lane == 0) u = 0;
#pragma unroll 4
        for (int b = b0; b < b1; ++b) {
            u = wp[b] - lp[b] * u;
            wp[b] = u * dp[b];
        }
        __syncwarp();
        // backward over the same rows, lanes in reverse order
        E = 0;
        P = 1;
#pragma unroll 4
        for (int b = b1 - 1; b >= b0; --b) {
            const T l = b + 1 < ny ? lp[b + 1] : T(0);
            E = wp[b] - l * E;
            P = -l * P;
        }
        affine_scan(E, P, lane, true);
        T x = __shfl_down_sync(0xffffffffu, E, 1);
        if (lane == 31) x = 0;
#pragma unroll 4
        for (int b = b1 - 1; b >= b0; --b) {
            const T l = b + 1 < ny ? lp[b + 1] : T(0);
            x = wp[b] - l * x;
            wp[b] = x;
        }
        if constexpr (STAGED) {
            __syncwarp();
            const int nv = (int)((size_t)nyp * sizeof(T) / 16);
            const uint4 *src = reinterpret_cast<const uint4 *>(wb);
            uint4 *dst = reinterpret_cast<uint4 *>(wg);
            for (int i = lane; i < nv; i += 32) dst[i] = src[i];
            fence_proxy_async_smem();   // order these generic accesses before the next bulk copy
            __syncwarp();
        }
    }
}

// Launch shape of fd_tri_kernel for columns of nyp entries of T: warps per
// CTA of the staged kernel (0 when a column and its factors do not fit in
// shared memory) and its dynamic shared memory.
static int tri_warps(int nyp, size_t esz, size_t &smem)
{
    const size_t per_warp = 3 * (size_t)nyp * esz, cap = 226 * 1024;   // leaves room for the static barriers
    const int w = (int)std::min<size_t>(kTriMaxWarps, cap / per_warp);
    smem = (size_t)w * per_warp;
    return w;
}

// Interior block of r (m x n grid, x fastest) into a zero-padded nxp x nyp
// column-major matrix (rows = x), and back: GEMM-friendly leading dimensions.
// Each thread moves 16 bytes of the padded matrix (nxp is a multiple of 16);
// blockIdx.y strides over the columns b, so no index division is needed. With
// sc (FP64 vectors, FP32 transform) the gather divides by pc_scale and the
// scatter multiplies by it.
// z = r on the boundary ring of the m x n grid (identity rows of K_fem),
// ring entries t0, t0 + stride, ...
template <typename T>
__device__ __forceinline__ void ring_copy(T *__restrict__ z, const T *__restrict__ r, int m, int n, long long t0,
                                          long long stride)
{
    const long long nb = 2LL * m + 2LL * (n - 2);
    for (long long t = t0; t < nb; t += stride) {
        long long idx;
        if (t < m) idx = t;
        else if (t < 2LL * m) idx = (long long)(n - 1) * m + (t - m);
        else {
            const long long u = t - 2LL * m;
            const long long j = 1 + u / 2;
            idx = j * m + ((u % 2) ? (m - 1) : 0);
        }
        z[idx] = r[idx];
    }
}

// The gather also copies the boundary ring of r into z (one launch fewer).
// With the parity split (kb > 0) column c of U is, for c < kb, the even fold
// r[c] + r[nx-1-c] (c < fo; the middle entry r[fo] alone when nx is odd) and,
// for c >= kb, the odd fold r[j] - r[nx-1-j] with j = c - kb < fo.
template <typename T, typename V>
__global__ void fd_gather_kernel(const V *__restrict__ r, T *__restrict__ U, V *__restrict__ z, int m, int n, int nx,
                                 int ny, int nxp, int nyp, int kb, int fo, const DevScalars *sc)
{
    pdl_begin();
    ring_copy(z, r, m, n, ((long long)blockIdx.y * gridDim.x + blockIdx.x) * blockDim.x + threadIdx.x,
              (long long)gridDim.x * gridDim.y * blockDim.x);
    constexpr int VN = Pk<T>::n;
    const double inv = sc ? 1.0 / pc_scale(sc) : 1.0;
    const int nv = nxp / VN;
    for (int b = blockIdx.y; b < nyp; b += gridDim.y) {
        const V *rb = r + (size_t)(b + 1) * m + 1;
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nv; k += gridDim.x * blockDim.x) {
            Pk<T> o;
#pragma unroll
            for (int c = 0; c < VN; ++c) {
                const int a = k * VN + c;
                double v = 0.0;
                if (b < ny) {
                    if (kb == 0) {
                        if (a < nx) v = (double)rb[a];
                    } else if (a < kb) {
                        if (a < fo) v = (double)rb[a] + (double)rb[nx - 1 - a];
                        else if (a == fo && (nx & 1)) v = (double)rb[a];
                    } else if (a - kb < fo) {
                        v = (double)rb[a - kb] - (double)rb[nx - 1 - (a - kb)];
                    }
                }
                o.v[c] = (T)(v * inv);
            }
            stp(U, (long long)b * nxp + (long long)k * VN, o);
        }
    }
}

// z's interior from the parity-split transform W [nyp][nxp] (even block
// Ze = columns 0 .. fe-1, odd block Zo = columns kb .. kb+fo-1):
// z[j] = Ze[j] + Zo[j], z[nx-1-j] = Ze[j] - Zo[j] (j < fo), and the middle
// entry z[fo] = Ze[fo] when nx is odd; times sqrt(*rr) when rr is set.
template <typename T, typename V>
__global__ void fd_unfold_kernel(const T *__restrict__ W, V *__restrict__ z, int m, int nx, int ny, int nxp, int kb,
                                 int fe, int fo, const double *rr)
{
    pdl_begin();
    double f = 1.0;
    if (rr) {
        const double v = *rr;
        f = (v > 0.0 && v < 1e300) ? sqrt(v) : 1.0;
    }
    for (int b = blockIdx.y; b < ny; b += gridDim.y) {
        const T *wb = W + (size_t)b * nxp;
        V *zb = z + (size_t)(b + 1) * m + 1;
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < fe; j += gridDim.x * blockDim.x) {
            const double e = (double)wb[j];
            if (j < fo) {
                const double o = (double)wb[kb + j];
                zb[j] = (V)(f * (e + o));
                zb[nx - 1 - j] = (V)(f * (e - o));
            } else {
                zb[j] = (V)(f * e);
            }
        }
    }
}

// 2-D launch of the gather / unfold: 128-thread blocks over the groups of a
// row, block rows striding over the rows. About one wave of blocks (16 per
// SM): one block per row made these kernels block-launch bound (the FP32
// unfold of a 2049 x 1025 half took 21 us in 18.4 K blocks of one row each).
static dim3 grid2d(int ngroups, int nrows, int nsm)
{
    const int gx = std::max(1, (ngroups + 127) / 128);
    const int gy = std::max(1, std::min({nrows, 65535, std::max(1, 16 * nsm / gx)}));
    return dim3((unsigned)gx, (unsigned)gy);
}

// z = r on the boundary ring (identity rows of K_fem).
template <typename T>
__global__ void boundary_copy_kernel(T *__restrict__ z, const T *__restrict__ r, int m, int n)
{
    pdl_begin();
    ring_copy(z, r, m, n, blockIdx.x * (long long)blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x);
}

// ------------------------------------------------------------ kappa scaling of the preconditioner
// s_i = 1 / sqrt(mean of kappa over the quadrature points of the elements
// supporting control point i); the preconditioner becomes S M^-1 S, which
// keeps the FEM matrix's shape and adds the coefficient's local magnitude.
__global__ void kappa_scale_kernel(const double *__restrict__ kappa, double *__restrict__ s64, float *__restrict__ s32,
                                   StripGrid g)
{
    const int P = g.P, NQ2 = (P + 1) * (P + 1);
    const long long N = (long long)g.m * g.n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int C = (int)(t % g.m), R = (int)(t / g.m);
        double sum = 0.0;
        int cnt = 0;
        for (int ey = max(0, R - P); ey <= min(R, g.ney - 1); ++ey)
            for (int ex = max(0, C - P); ex <= min(C, g.nex - 1); ++ex) {
                const double *k = kappa + ((size_t)ey * g.nex + ex) * NQ2;
                for (int q = 0; q < NQ2; ++q) sum += k[q];
                cnt += NQ2;
            }
        const double v = (cnt > 0 && sum > 0.0) ? 1.0 / sqrt(sum / cnt) : 1.0;
        s64[t] = v;
        s32[t] = (float)v;
    }
}

template <typename T>
__global__ void mul_kernel(T *__restrict__ out, const T *__restrict__ a, const T *__restrict__ b, long long N)
{
    pdl_begin();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x)
        out[t] = a[t] * b[t];
}

// ------------------------------------------------------------ host state
template <typename T>
struct PrecState {
    bool ready = false;
    T *kd = nullptr, *ko = nullptr, *md = nullptr, *mo = nullptr;
    T *ld = nullptr, *lo = nullptr, *nd = nullptr, *no = nullptr;
    T *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *b = nullptr;
    T *tz = nullptr;   // FP32 state: the preconditioner's output inside an FP64 (IGA_MIXED_PC) solve
    T *sc = nullptr;   // kappa-scaled preconditioner input
    T *iz = nullptr, *ir = nullptr, *ip = nullptr, *iq = nullptr;
    cudaGraphExec_t chunk = nullptr;
    // exact FEM inverse: x eigenvectors (column-major), eigenvalues, two work
    // matrices, and the LDL^T factors of the y systems of every x mode
    T *Vx = nullptr, *lx = nullptr, *W1 = nullptr, *W2 = nullptr, *Dv = nullptr;
    T *Lf = nullptr;   // LDL^T unit lower factor's subdiagonal per x mode (layout of Dv)
    int nxp = 0, nyp = 0;   // transform sizes padded to multiples of 16
    // parity split of the x transform (centrosymmetric x pencil): kb = the
    // padded even block (0: no split), fe / fo the even / odd mode counts;
    // nmodes = rows of the mode-major work matrix the y solves walk
    int kb = 0, fe = 0, fo = 0, nmodes = 0;
    GemmTF32 g1, g2;        // FP32: the two transforms' prepared tensor-core GEMMs
    int tri_w = 0;          // most warps per CTA of the staged tridiagonal kernel (0: in place)
    size_t tri_smem = 0;    // its shared memory at tri_w warps
    int nsm = 148;          // SMs of the plan's device
    // device-side PCG loop: a CUDA graph whose conditional WHILE node runs one
    // iteration per pass (built for one preconditioner / kappa-scaling choice)
    cudaGraphExec_t loop = nullptr;
    int loop_pc = -1, loop_scaled = -1, loop_prec = -1;
    bool loop_failed = false;   // the loop graph could not be instantiated: host-driven loop
    FemCoef<T> coef() const
    {
        FemCoef<T> c;
        c.kd = kd; c.ko = ko; c.md = md; c.mo = mo;
        c.ld = ld; c.lo = lo; c.nd = nd; c.no = no;
        return c;
    }
};

struct SolverState {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool fd_host = false;
    // host x eigenpairs (built once). Split by parity (fold): even modes
    // 0 .. fe-1 then odd modes, Vx = the fe x fe even block followed by the
    // fo x fo odd block, each row one mode's half vector; else n x n.
    bool fold = false;
    int fe = 0, fo = 0;
    std::vector<double> lamx, Vx;
    std::vector<double> Dv, Lf;               // host LDL^T factors of the y systems, [a][b]
    double *ks64 = nullptr;                   // kappa scaling of the preconditioner
    float *ks32 = nullptr;
    int kappa_version = 0;
    DevScalars *s = nullptr;
    DevScalars *h = nullptr;   // pinned mirror
    double *partials = nullptr;
    unsigned *counter = nullptr;
    double *r64 = nullptr, *q64 = nullptr;   // refinement residual / operator output
    PrecState<double> d;
    PrecState<float> f;
    std::vector<double> gx, gy;
};

}  // namespace iga

using namespace iga;

namespace iga {

void fem_1d(const std::vector<double> &g, std::vector<double> &kd, std::vector<double> &ko,
                   std::vector<double> &md, std::vector<double> &mo)
{
    const int n = (int)g.size();
    kd.assign(n, 0.0);
    md.assign(n, 0.0);
    ko.assign(n, 0.0);
    mo.assign(n, 0.0);
    for (int e = 0; e + 1 < n; ++e) {   // linear element [g_e, g_e+1], 2-point Gauss is exact
        const double h = g[e + 1] - g[e];
        kd[e] += 1.0 / h;
        kd[e + 1] += 1.0 / h;
        ko[e] = -1.0 / h;
        md[e] += h / 3.0;
        md[e + 1] += h / 3.0;
        mo[e] = h / 6.0;
    }
}

std::vector<double> fem_nodes_1d(int p, int ne, double L)
{
    if (p >= 3) {   // matrix_free/preprocess_fem.cpp:38-60
        std::vector<double> S;
        const double h = L / (ne + 2);
        for (int i = 0; i < p - 1; ++i) S.push_back(0.0);
        for (int i = 1; i < ne + 2; ++i) S.push_back(i * h);
        for (int i = 0; i < p - 1; ++i) S.push_back(L);
        return greville(p - 2, S);
    }
    return greville(p, open_knots(p, ne, L));
}

// Lengths of the FEM grid: mean polyline length of the control-net rows
// (x direction) and columns (y direction); 1 x 1 on the unit square.
// Segment lengths as sqrt(dx^2 + dy^2): control-net coordinates are far from
// the overflow range, and std::hypot's scaling made this loop a third of a
// 256-problem batch's preconditioner set-up.
void net_lengths(const Patch &P, double &Lx, double &Ly)
{
    double sx = 0.0, sy = 0.0;
    auto seg = [](double dx, double dy) { return std::sqrt(dx * dx + dy * dy); };
    for (int j = 0; j < P.n; ++j)
        for (int i = 0; i + 1 < P.m; ++i) {
            const size_t a = (size_t)j * P.m + i;
            sx += seg(P.CP[2 * (a + 1)] - P.CP[2 * a], P.CP[2 * (a + 1) + 1] - P.CP[2 * a + 1]);
        }
    for (int j = 0; j + 1 < P.n; ++j)
        for (int i = 0; i < P.m; ++i) {
            const size_t a = (size_t)j * P.m + i, b = a + P.m;
            sy += seg(P.CP[2 * b] - P.CP[2 * a], P.CP[2 * b + 1] - P.CP[2 * a + 1]);
        }
    Lx = sx / P.n;
    Ly = sy / P.m;
}

}  // namespace iga

#define SOLVE_TRY(call)                                                              \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));          \
            return e_ == cudaErrorMemoryAllocation ? IGA_ERR_NOMEM : IGA_ERR_CUDA;   \
        }                                                                            \
    } while (0)

template <typename T>
static int alloc_prec(PrecState<T> &ps, const iga_plan *pl, const SolverState &S)
{
    if (ps.ready) return IGA_OK;
    const size_t N = (size_t)pl->nfunc;
    std::vector<double> kd, ko, md, mo, ld, lo, nd, no;
    fem_1d(S.gx, kd, ko, md, mo);
    fem_1d(S.gy, ld, lo, nd, no);
    auto up = [&](T **dst, const std::vector<double> &v) -> int {
        std::vector<T> h(v.begin(), v.end());
        SOLVE_TRY(cudaMalloc((void **)dst, sizeof(T) * h.size()));
        SOLVE_TRY(cudaMemcpy(*dst, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
        return IGA_OK;
    };
    int st;
    if ((st = up(&ps.kd, kd)) || (st = up(&ps.ko, ko)) || (st = up(&ps.md, md)) || (st = up(&ps.mo, mo)) ||
        (st = up(&ps.ld, ld)) || (st = up(&ps.lo, lo)) || (st = up(&ps.nd, nd)) || (st = up(&ps.no, no)))
        return st;
    for (T **v : {&ps.x, &ps.r, &ps.z, &ps.tz, &ps.p, &ps.q, &ps.b, &ps.sc, &ps.iz, &ps.ir, &ps.ip, &ps.iq})
        SOLVE_TRY(cudaMalloc((void **)v, sizeof(T) * N));
    ps.ready = true;
    return IGA_OK;
}

static int ensure_state(iga_plan *pl, SolverState **out)
{
    if (pl->solver) {
        *out = pl->solver;
        return IGA_OK;
    }
    SolverState *S = new SolverState();
    pl->solver = S;
    S->device = pl->device;
    SOLVE_TRY(cudaSetDevice(pl->device));
    SOLVE_TRY(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
    SOLVE_TRY(cudaMalloc((void **)&S->s, sizeof(DevScalars)));
    SOLVE_TRY(cudaMemset(S->s, 0, sizeof(DevScalars)));
    SOLVE_TRY(cudaMallocHost((void **)&S->h, sizeof(DevScalars)));
    SOLVE_TRY(cudaMalloc((void **)&S->partials, sizeof(double) * kRedBlocks * 4));
    SOLVE_TRY(cudaMalloc((void **)&S->counter, sizeof(unsigned)));
    SOLVE_TRY(cudaMemset(S->counter, 0, sizeof(unsigned)));
    SOLVE_TRY(cudaMalloc((void **)&S->r64, sizeof(double) * pl->nfunc));
    SOLVE_TRY(cudaMalloc((void **)&S->q64, sizeof(double) * pl->nfunc));
    double Lx, Ly;
    net_lengths(pl->patch, Lx, Ly);
    S->gx = fem_nodes_1d(pl->p, pl->nex, Lx);
    S->gy = fem_nodes_1d(pl->p, pl->ney, Ly);
    *out = S;
    return IGA_OK;
}

template <typename T>
static void free_prec(PrecState<T> &ps)
{
    T *bufs[] = {ps.kd, ps.ko, ps.md, ps.mo, ps.ld, ps.lo, ps.nd, ps.no, ps.x, ps.r, ps.z, ps.tz, ps.p,
                 ps.q, ps.b, ps.sc, ps.iz, ps.ir, ps.ip, ps.iq, ps.Vx, ps.lx, ps.W1, ps.W2, ps.Dv, ps.Lf};
    for (T *v : bufs)
        if (v) cudaFree(v);
    if (ps.chunk) cudaGraphExecDestroy(ps.chunk);
    if (ps.loop) cudaGraphExecDestroy(ps.loop);
    ps = PrecState<T>{};
}

void iga_solver_release(iga_plan *pl)
{
    SolverState *S = pl->solver;
    if (!S) return;
    cudaSetDevice(S->device);
    free_prec(S->d);
    free_prec(S->f);
    for (void *v : {(void *)S->s, (void *)S->partials, (void *)S->counter, (void *)S->r64, (void *)S->q64,
                    (void *)S->ks64, (void *)S->ks32})
        if (v) cudaFree(v);
    if (S->h) cudaFreeHost(S->h);
    if (S->stream) cudaStreamDestroy(S->stream);
    delete S;
    pl->solver = nullptr;
}

template <typename T>
static FemCoef<T> coef_of(const PrecState<T> &ps, const iga_plan *pl)
{
    FemCoef<T> c = ps.coef();
    c.m = pl->m;
    c.n = pl->n;
    return c;
}

template <typename T>
static InnerCG<T> inner_of(PrecState<T> &ps, const iga_plan *pl, SolverState *S)
{
    InnerCG<T> a;
    a.z = ps.iz;
    a.r = ps.ir;
    a.p = ps.ip;
    a.q = ps.iq;
    a.rhs = nullptr;
    a.c = coef_of(ps, pl);
    a.s = S->s;
    a.partials = S->partials;
    a.counter = S->counter;
    return a;
}

// One captured graph of kChunk inner iterations (3 kernels each, no-ops once done).
template <typename T>
static int inner_chunk_graph(PrecState<T> &ps, const iga_plan *pl, SolverState *S)
{
    if (ps.chunk) return IGA_OK;
    InnerCG<T> a = inner_of(ps, pl, S);
    cudaGraph_t g;
    SOLVE_TRY(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < kChunk; ++k) {
        icg_q_kernel<T><<<kRedBlocks, kThreads, 0, S->stream>>>(a);
        icg_update_kernel<T><<<kRedBlocks, kThreads, 0, S->stream>>>(a);
        icg_p_kernel<T><<<kRedBlocks, kThreads, 0, S->stream>>>(a);
    }
    SOLVE_TRY(cudaStreamEndCapture(S->stream, &g));
    SOLVE_TRY(cudaGraphInstantiate(&ps.chunk, g, 0));
    cudaGraphDestroy(g);
    return IGA_OK;
}

namespace iga {
void interior_pencil(const std::vector<double> &g, std::vector<double> &Kd, std::vector<double> &Ko,
                            std::vector<double> &Md, std::vector<double> &Mo)
{
    std::vector<double> kd, ko, md, mo;
    fem_1d(g, kd, ko, md, mo);
    const int n = (int)g.size() - 2;
    Kd.assign(kd.begin() + 1, kd.begin() + 1 + n);
    Md.assign(md.begin() + 1, md.begin() + 1 + n);
    Ko.assign(ko.begin() + 1, ko.begin() + 1 + n);
    Mo.assign(mo.begin() + 1, mo.begin() + 1 + n);
}
}  // namespace iga

// Eigenpairs of the x pencil split by parity (pencil_fold): even modes
// 0 .. fe-1 then odd modes, each a half vector. v . r = u . (r[i] + r[nx-1-i])_i
// (the middle entry taken once) for an even mode and u . (r[i] - r[nx-1-i])_i
// for an odd one, which halves the flops of both transforms (the even-odd
// decomposition of spectral and fast-diagonalisation methods). Eigenpairs
// computed on the device (bisection, inverse iteration).
static int fold_eig(const std::vector<double> &Kd, const std::vector<double> &Ko, const std::vector<double> &Md,
                    const std::vector<double> &Mo, SolverState *S)
{
    const int n = (int)Kd.size(), fo = n / 2, fe = n - fo;
    std::vector<double> hk[2][4];
    std::vector<PencilRef> refs(2);
    for (int parity = 0; parity < 2; ++parity) {
        pencil_fold(n, Kd.data(), Ko.data(), Md.data(), Mo.data(), parity, hk[parity][0], hk[parity][1],
                    hk[parity][2], hk[parity][3]);
        refs[parity] = PencilRef{parity == 0 ? fe : fo, hk[parity][0].data(), hk[parity][1].data(),
                                 hk[parity][2].data(), hk[parity][3].data()};
    }
    std::vector<std::vector<double>> lam, vec;
    int st = pencil_eig_device(S->device, refs, lam, &vec);
    if (st) return st;
    S->fold = true;
    S->fe = fe;
    S->fo = fo;
    S->lamx.assign(n, 0.0);
    S->Vx.assign((size_t)fe * fe + (size_t)fo * fo, 0.0);
    for (int parity = 0; parity < 2; ++parity) {
        const int h = refs[parity].n;
        if (h == 0) continue;
        double *L = S->lamx.data() + (parity == 0 ? 0 : fe);
        double *V = S->Vx.data() + (parity == 0 ? 0 : (size_t)fe * fe);
        std::copy(lam[parity].begin(), lam[parity].end(), L);
        const double sc = 1.0 / std::sqrt(2.0);
        for (size_t i = 0; i < (size_t)h * h; ++i) V[i] = sc * vec[parity][i];
    }
    return IGA_OK;
}

// The x pencil's eigenpairs and, for every x mode a, the LDL^T factors of the
// y system lx[a] My + Ky on the free nodes, built once per plan on the host.
static int fd_setup(PrecState<double> &, const iga_plan *pl, SolverState *S)
{
    if (S->fd_host) return IGA_OK;
    std::vector<double> Kd, Ko, Md, Mo;
    interior_pencil(S->gx, Kd, Ko, Md, Mo);
    const int nx = (int)Kd.size();
    if (pl->pc_split && pencil_centrosymmetric(nx, Kd.data(), Ko.data(), Md.data(), Mo.data())) {
        const int st = fold_eig(Kd, Ko, Md, Mo, S);
        if (st) return st;
    } else {
        S->fold = false;
        std::vector<std::vector<double>> lam, vec;
        const int st = pencil_eig_device(S->device, {PencilRef{nx, Kd.data(), Ko.data(), Md.data(), Mo.data()}}, lam, &vec);
        if (st) return st;
        S->lamx = lam[0];
        S->Vx = vec[0];
    }
    interior_pencil(S->gy, Kd, Ko, Md, Mo);
    const int ny = (int)Kd.size();
    S->Dv.assign((size_t)nx * ny, 0.0);
    S->Lf.assign((size_t)nx * ny, 0.0);
    for (int a = 0; a < nx; ++a) {
        const double lam = S->lamx[a];
        double cprev = 0.0, eprev = 0.0;   // e_{b-1} / d_{b-1} and e_{b-1}
        for (int b = 0; b < ny; ++b) {
            const double den = lam * Md[b] + Kd[b] - eprev * cprev;
            const double e = b + 1 < ny ? lam * Mo[b] + Ko[b] : 0.0;
            S->Dv[(size_t)a * ny + b] = 1.0 / den;
            S->Lf[(size_t)a * ny + b] = cprev;
            cprev = e / den;
            eprev = e;
        }
    }
    S->fd_host = true;
    return IGA_OK;
}

static int prepare_gemms(PrecState<double> &) { return IGA_OK; }
static int prepare_gemms(PrecState<float> &ps)
{
    const int nxp = ps.nxp, nyp = ps.nyp;
    int st = gemm_tf32_prepare(ps.g1, GemmOperand{ps.Vx, nxp, false}, GemmOperand{ps.W2, nxp, false}, ps.W1, nyp, nxp,
                               nyp, nxp, nxp, nyp, GemmSplit{ps.kb, false});
    if (st) return st;
    ps.g1.const_op = 1;   // Vx
    st = gemm_tf32_prepare(ps.g2, GemmOperand{ps.W1, nyp, true}, GemmOperand{ps.Vx, nxp, true}, ps.W2, nxp, nyp, nxp,
                           nxp, nyp, nxp, GemmSplit{ps.kb, true});
    ps.g2.const_op = 2;   // Vx
    return st;
}

template <typename T>
static int fd_upload(PrecState<T> &ps, const iga_plan *pl, SolverState *S)
{
    if (ps.Vx) return IGA_OK;
    PrecState<double> dummy;
    if (const int st0 = fd_setup(dummy, pl, S)) return st0;
    const int nx = pl->m - 2, ny = pl->n - 2;
    // multiples of 16: aligned rows for the GEMMs and 16-byte moves; the
    // DGEMMs do no more flops than they must (2112 -> 2064 at 2048^2: FP64
    // PCG 114 -> 111 ms; TF32 GEMMs inside the solver's graph unchanged).
    // With the parity split the x index runs over the even block (fe values,
    // padded to kb) and then the odd block (fo values, padded).
    const int fe = S->fold ? S->fe : nx, fo = S->fold ? S->fo : 0;
    const int kb = (fe + 15) / 16 * 16, kob = (fo + 15) / 16 * 16;
    const int nxp = S->fold ? kb + kob : kb, nyp = (ny + 15) / 16 * 16;
    ps.nxp = nxp;
    ps.nyp = nyp;
    ps.kb = S->fold ? kb : 0;
    ps.fe = fe;
    ps.fo = fo;
    ps.nmodes = S->fold ? nxp : nx;
    // device row of host mode a (even modes, then odd ones from row kb)
    auto row_of = [&](int a) { return a < fe ? a : kb + (a - fe); };
    // zero-padded eigenvector matrix, block diagonal with the split: row
    // row_of(a) holds mode a's (half) vector from column 0 (even) or kb (odd)
    auto up_mat = [&](T **dst) -> int {
        std::vector<T> h((size_t)nxp * nxp, T(0));
        for (int a = 0; a < fe; ++a)
            for (int i = 0; i < fe; ++i) h[(size_t)a * nxp + i] = (T)S->Vx[(size_t)a * fe + i];
        const double *Vo = S->Vx.data() + (size_t)fe * fe;
        for (int a = 0; a < fo; ++a)
            for (int i = 0; i < fo; ++i) h[(size_t)(kb + a) * nxp + kb + i] = (T)Vo[(size_t)a * fo + i];
        SOLVE_TRY(cudaMalloc((void **)dst, sizeof(T) * h.size()));
        SOLVE_TRY(cudaMemcpy(*dst, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
        return IGA_OK;
    };
    // padded eigenvalues 1 keep the scaling finite
    auto up_vec = [&](T **dst, const std::vector<double> &v, int np) -> int {
        std::vector<T> h(np, T(1));
        for (size_t i = 0; i < v.size(); ++i) h[row_of((int)i)] = (T)v[i];
        SOLVE_TRY(cudaMalloc((void **)dst, sizeof(T) * h.size()));
        SOLVE_TRY(cudaMemcpy(*dst, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
        return IGA_OK;
    };
    // y factors in the layout of Wt: element (b, row_of(a)) at b + row_of(a) nyp
    // (padded modes: zero factors, so their solves return zeros)
    auto up_fac = [&](T **dst, const std::vector<double> &F) -> int {
        std::vector<T> h((size_t)nxp * nyp, T(0));
        for (int a = 0; a < nx; ++a)
            for (int b = 0; b < ny; ++b) h[(size_t)row_of(a) * nyp + b] = (T)F[(size_t)a * ny + b];
        SOLVE_TRY(cudaMalloc((void **)dst, sizeof(T) * h.size()));
        SOLVE_TRY(cudaMemcpy(*dst, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
        return IGA_OK;
    };
    int st;
    if ((st = up_mat(&ps.Vx)) || (st = up_vec(&ps.lx, S->lamx, nxp)) || (st = up_fac(&ps.Dv, S->Dv)) ||
        (st = up_fac(&ps.Lf, S->Lf)))
        return st;
    ps.tri_w = tri_warps(nyp, sizeof(T), ps.tri_smem);
    SOLVE_TRY(cudaDeviceGetAttribute(&ps.nsm, cudaDevAttrMultiProcessorCount, pl->device));
    if (ps.tri_w)
        SOLVE_TRY(cudaFuncSetAttribute(fd_tri_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)ps.tri_smem));
    SOLVE_TRY(cudaMalloc((void **)&ps.W1, sizeof(T) * (size_t)nxp * nyp));
    SOLVE_TRY(cudaMalloc((void **)&ps.W2, sizeof(T) * (size_t)nxp * nyp));
    return prepare_gemms(ps);
}

// The transforms' GEMMs in the row-major views of the work matrices:
//   W1[a][b] = sum_k Vx[a][k] W2[b][k]   (both operands K-major),
//   W2[b][i] = sum_a W1[a][b] Vx[a][i]   (both operands MN-major),
// with Vx[a][k] = component k of eigenvector a (ld nxp), W1 [nxp][nyp],
// W2 [nyp][nxp]. With the parity split, W2's columns (the GEMMs' k for the
// first, their n for the second) are the even folds then the odd folds, and
// Vx is block diagonal at kb (even modes' half vectors, odd modes' half
// vectors): each output tile runs over its own block's k range only, half
// the flops of the full transforms. FP32: tcgen05 TF32 tiles fed by tensor maps built here once
// (the preconditioner only has to be a close SPD approximation of K_fem^-1;
// the flexible PCG and the FP64 refinement absorb the difference); FP64:
// DMMA tiles.
static int transform_gemm(PrecState<double> &ps, const iga_plan *, int which, cudaStream_t s,
                          const GemmScatter &sc = GemmScatter())
{
    const int nxp = ps.nxp, nyp = ps.nyp;
    if (which == 1)
        return gemm_f64_launch(GemmOperand{ps.Vx, nxp, false}, GemmOperand{ps.W2, nxp, false}, ps.W1, nyp, nxp, nyp,
                               nxp, nxp, nyp, s, GemmScatter(), GemmSplit{ps.kb, false});
    return gemm_f64_launch(GemmOperand{ps.W1, nyp, true}, GemmOperand{ps.Vx, nxp, true}, ps.W2, nxp, nyp, nxp, nxp, nyp,
                           nxp, s, sc, GemmSplit{ps.kb, true});
}

static int transform_gemm(PrecState<float> &ps, const iga_plan *pl, int which, cudaStream_t s,
                          const GemmScatter &sc = GemmScatter())
{
    return gemm_tf32_launch(which == 1 ? ps.g1 : ps.g2, s, pl->d_err, sc);
}

// z = K_fem^-1 r on the free nodes (R, Z: the interior blocks of r, z,
// zero-padded to multiples of 16 so the GEMMs run with aligned leading
// dimensions). With Kx V = Mx V diag(lx) (V Mx-orthonormal), K_fem =
// Kx (x) My + Mx (x) Ky becomes, mode by mode in x, the tridiagonal y system
// lx[a] My + Ky: Wt = R^T Vx (so that each mode's y values are contiguous),
// column a of Wt solved along y, Z = Vx Wt^T. Two GEMMs and one pass of
// tridiagonal solves (the fast diagonalisation in both directions would take
// four GEMMs). With the parity split the gather folds r (r[i] +- r[nx-1-i]),
// the GEMMs work on the two half blocks, and the unfold kernel forms z.
// V is the vectors' type; an FP32 transform of FP64 vectors (T = float,
// V = double) passes sc, the device scalars whose rr scales the data.
template <typename T, typename V>
static int fd_apply(PrecState<T> &ps, const iga_plan *pl, SolverState *S, const V *r, V *z, const DevScalars *sc)
{
    const int m = pl->m, n = pl->n, nx = m - 2, ny = n - 2;
    if (nx <= 0 || ny <= 0) {   // no free nodes: the ring is everything
        SOLVE_TRY(launch_k(boundary_copy_kernel<V>, dim3(kRedBlocks), dim3(kThreads), 0, S->stream, z, r, m, n));
        return IGA_OK;
    }
    const int nxp = ps.nxp, nyp = ps.nyp;
    int seg = (ny + 31) / 32;
    seg |= 1;   // odd: conflict-free shared-memory rows
    constexpr int VN = Pk<T>::n;
    SOLVE_TRY(launch_k(fd_gather_kernel<T, V>, grid2d(nxp / VN, nyp, ps.nsm), dim3(128), 0, S->stream, r, ps.W2, z, m, n, nx, ny,
                       nxp, nyp, ps.kb, ps.fo, sc));
    int e = transform_gemm(ps, pl, 1, S->stream);
    if (e == IGA_OK) {
        if (ps.tri_w) {
            // one mode per warp as long as the modes reach every SM, else the most
            // warps per CTA that shared memory allows (warps then loop over modes)
            const int nm = ps.nmodes;
            const int w = std::max(1, std::min(ps.tri_w, (nm + ps.nsm - 1) / ps.nsm));
            const int grid = std::min((nm + w - 1) / w, ps.nsm);
            const size_t smem = ps.tri_smem / ps.tri_w * w;
            SOLVE_TRY(launch_k(fd_tri_kernel<T, true>, dim3(grid), dim3(w * 32), smem, S->stream, ps.W1,
                               (const T *)ps.Lf, (const T *)ps.Dv, nm, ny, nyp, seg, S->s));
        } else {
            SOLVE_TRY(launch_k(fd_tri_kernel<T, false>, dim3((ps.nmodes + 7) / 8), dim3(256), 0, S->stream, ps.W1,
                               (const T *)ps.Lf, (const T *)ps.Dv, ps.nmodes, ny, nyp, seg, S->s));
        }
        if (ps.kb > 0) {
            // parity split: the second GEMM writes both halves' products, the
            // unfold kernel combines them into z's interior
            e = transform_gemm(ps, pl, 2, S->stream);
            if (e == IGA_OK)
                SOLVE_TRY(launch_k(fd_unfold_kernel<T, V>, grid2d(ps.fe, ny, ps.nsm), dim3(128), 0, S->stream,
                                   (const T *)ps.W2, z, m, nx, ny, nxp, ps.kb, ps.fe, ps.fo,
                                   sc ? &sc->rr : (const double *)nullptr));
        } else {
            // the second GEMM's epilogue writes z's interior itself
            GemmScatter gs;
            gs.out = z;
            gs.f64 = std::is_same<V, double>::value;
            gs.ld = m;
            gs.rows = ny;
            gs.cols = nx;
            gs.rr = sc ? &sc->rr : nullptr;
            e = transform_gemm(ps, pl, 2, S->stream, gs);
        }
    }
    if (e != IGA_OK) {
        set_error("GEMM launch failed in the FEM preconditioner: " + last_error());
        return e;
    }
    return IGA_OK;
}

template <typename T>
static int pc_apply_core(PrecState<T> &ps, const iga_plan *pl, SolverState *S, const iga_solve_opts &o, const T *r,
                         T *z, double pc_rtol, int64_t &pc_iters);

static const double *kscale(SolverState *S, double *) { return S->ks64; }
static const float *kscale(SolverState *S, float *) { return S->ks32; }

// Scaling vector of the current kappa (null when the plan has none).
static int update_kscale(const iga_plan *pl, SolverState *S)
{
    if (!pl->kappa_dev || S->kappa_version == pl->kappa_version) return IGA_OK;
    if (!S->ks64) {
        SOLVE_TRY(cudaMalloc((void **)&S->ks64, sizeof(double) * pl->nfunc));
        SOLVE_TRY(cudaMalloc((void **)&S->ks32, sizeof(float) * pl->nfunc));
    }
    kappa_scale_kernel<<<kRedBlocks, kThreads, 0, S->stream>>>(pl->kappa_dev, S->ks64, S->ks32, pl->grid);
    S->kappa_version = pl->kappa_version;
    SOLVE_TRY(cudaGetLastError());
    return IGA_OK;
}

// z = M^-1 r for FP64 vectors with the preconditioner evaluated in FP32
// (IGA_MIXED_PC): the input divided by ||r|| into FP32 (inside the
// transform's gather for the exact inverse), the FP32 preconditioner, the
// output multiplied back into FP64. The outer flexible PCG absorbs the FP32
// (TF32 GEMM) rounding of the preconditioner.
static int pc_apply_fp32(const iga_plan *pl, SolverState *S, const iga_solve_opts &o, const double *r, double *z,
                         double pc_rtol, int64_t &pc_iters)
{
    const long long N = pl->nfunc;
    PrecState<float> &f = S->f;
    int st;
    const double *rin = r;
    if (pl->kappa_dev) {
        if ((st = update_kscale(pl, S))) return st;
        mul_kernel<double><<<kRedBlocks, kThreads, 0, S->stream>>>(S->d.sc, r, S->ks64, N);
        rin = S->d.sc;
    }
    if (o.pc == IGA_PC_FEM_EXACT) {
        if ((st = fd_upload(f, pl, S))) return st;
        if ((st = fd_apply<float, double>(f, pl, S, rin, z, S->s))) return st;
    } else {
        SOLVE_TRY(launch_k(to_fp32_kernel, dim3(kRedBlocks), dim3(kThreads), 0, S->stream, rin, f.sc, N,
                           (const DevScalars *)S->s));
        if ((st = pc_apply_core<float>(f, pl, S, o, f.sc, f.tz, pc_rtol, pc_iters))) return st;
        SOLVE_TRY(launch_k(from_fp32_kernel, dim3(kRedBlocks), dim3(kThreads), 0, S->stream, (const float *)f.tz, z, N,
                           (const DevScalars *)S->s));
    }
    if (pl->kappa_dev)
        SOLVE_TRY(launch_k(mul_kernel<double>, dim3(kRedBlocks), dim3(kThreads), 0, S->stream, z, (const double *)z,
                           (const double *)S->ks64, N));
    return IGA_OK;
}

// z = M^-1 r for the configured preconditioner; with a coefficient kappa,
// z = S M^-1 (S r) with the local scaling S.
template <typename T>
static int pc_apply(PrecState<T> &ps, const iga_plan *pl, SolverState *S, const iga_solve_opts &o, const T *r, T *z,
                    double pc_rtol, int64_t &pc_iters)
{
    const long long N = pl->nfunc;
    if constexpr (std::is_same<T, double>::value) {
        if (o.precision == IGA_MIXED_PC && o.pc != IGA_PC_NONE) return pc_apply_fp32(pl, S, o, r, z, pc_rtol, pc_iters);
    }
    if (o.pc == IGA_PC_NONE || !pl->kappa_dev) return pc_apply_core(ps, pl, S, o, r, z, pc_rtol, pc_iters);
    int st;
    if ((st = update_kscale(pl, S))) return st;
    const T *sv = kscale(S, (T *)nullptr);
    SOLVE_TRY(launch_k(mul_kernel<T>, dim3(kRedBlocks), dim3(kThreads), 0, S->stream, ps.sc, r, sv, N));
    if ((st = pc_apply_core(ps, pl, S, o, ps.sc, z, pc_rtol, pc_iters))) return st;
    SOLVE_TRY(launch_k(mul_kernel<T>, dim3(kRedBlocks), dim3(kThreads), 0, S->stream, z, (const T *)z, sv, N));
    return IGA_OK;
}

template <typename T>
static int pc_apply_core(PrecState<T> &ps, const iga_plan *pl, SolverState *S, const iga_solve_opts &o, const T *r,
                         T *z, double pc_rtol, int64_t &pc_iters)
{
    const long long N = pl->nfunc;
    if (o.pc == IGA_PC_NONE) {
        SOLVE_TRY(launch_k(copy_kernel<T>, dim3(kRedBlocks), dim3(kThreads), 0, S->stream, z, r, N));
        return IGA_OK;
    }
    int st;
    if (o.pc == IGA_PC_FEM_EXACT) {
        if ((st = fd_upload(ps, pl, S))) return st;
        return fd_apply<T, T>(ps, pl, S, r, z, nullptr);
    }
    if ((st = inner_chunk_graph(ps, pl, S))) return st;
    InnerCG<T> a = inner_of(ps, pl, S);
    icg_init_kernel<T><<<kRedBlocks, kThreads, 0, S->stream>>>(a, r, pc_rtol, o.pc_max_it);
    // Keep one chunk in flight ahead of the completion check.
    SOLVE_TRY(cudaGraphLaunch(ps.chunk, S->stream));
    int launched = 1;
    for (;;) {
        SOLVE_TRY(cudaMemcpyAsync(S->h, S->s, sizeof(DevScalars), cudaMemcpyDeviceToHost, S->stream));
        cudaEvent_t ev;
        SOLVE_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        SOLVE_TRY(cudaEventRecord(ev, S->stream));
        if ((long long)launched * kChunk < (long long)o.pc_max_it + kChunk) {
            SOLVE_TRY(cudaGraphLaunch(ps.chunk, S->stream));
            ++launched;
        }
        SOLVE_TRY(cudaEventSynchronize(ev));
        cudaEventDestroy(ev);
        if (S->h->idone) break;
        if ((long long)launched * kChunk >= (long long)o.pc_max_it + 2 * kChunk) break;
    }
    SOLVE_TRY(cudaStreamSynchronize(S->stream));
    pc_iters += S->h->iiters;
    if (S->h->ibreak) return IGA_ERR_BREAKDOWN;
    copy_kernel<T><<<kRedBlocks, kThreads, 0, S->stream>>>(z, ps.iz, N);
    return IGA_OK;
}

static int sync_scalars(SolverState *S)
{
    SOLVE_TRY(cudaMemcpyAsync(S->h, S->s, sizeof(DevScalars), cudaMemcpyDeviceToHost, S->stream));
    SOLVE_TRY(cudaStreamSynchronize(S->stream));
    return IGA_OK;
}

// Flexible PCG on K x = b in precision T, from the current x; stops when the
// recurrence residual satisfies ||r|| <= rtol ||b_ref||. Returns iterations.
template <typename T>
static int pcg(iga_plan *pl, SolverState *S, PrecState<T> &ps, const iga_solve_opts &o, const T *b, T *x, double rtol,
               double bnorm, double pc_rtol, int prec, int &its, int64_t &pc_iters)
{
    const long long N = pl->nfunc;
    const cudaStream_t s = S->stream;
    int st;
    // r = b - K x, rr = r.r
    if ((st = iga_apply_internal_sb(pl, prec, x, ps.q, s, IGA_SIGN_SPD, IGA_BC_IDENTITY))) return st;
    sub_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(b, ps.q, ps.r, N, S->s, S->partials, S->counter);
    if ((st = sync_scalars(S))) return st;
    if (std::sqrt(S->h->rr) <= rtol * bnorm) return IGA_OK;
    if ((st = pc_apply(ps, pl, S, o, ps.r, ps.z, pc_rtol, pc_iters))) return st;
    dot_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(ps.r, ps.z, N, &S->s->rz, S->partials, S->counter);
    pcg_p_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(ps.p, ps.z, N, S->s, 1);
    cudaMemsetAsync(&S->s->breakdown, 0, sizeof(int), s);
    for (int it = 0; it < o.max_it; ++it) {
        if ((st = iga_apply_internal_sb(pl, prec, ps.p, ps.q, s, IGA_SIGN_SPD, IGA_BC_IDENTITY))) return st;
        pcg_pq_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(ps.p, ps.q, N, S->s, S->partials, S->counter);
        pcg_xr_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(x, ps.r, ps.p, ps.q, ps.z, N, S->s, S->partials,
                                                         S->counter);
        ++its;
        if ((st = sync_scalars(S))) return st;
        if (S->h->breakdown) return IGA_ERR_BREAKDOWN;
        if (!std::isfinite(S->h->rr)) return IGA_ERR_NONFINITE;
        if (std::sqrt(S->h->rr) <= rtol * bnorm) return IGA_OK;
        if ((st = pc_apply(ps, pl, S, o, ps.r, ps.z, pc_rtol, pc_iters))) return st;
        pcg_beta_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(ps.r, ps.z, N, S->s, S->partials, S->counter);
        pcg_p_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(ps.p, ps.z, N, S->s, 0);
    }
    return IGA_ERR_NOT_CONVERGED;
}

// Builds the device-side loop for the current preconditioner choice: body =
// q = K p; alpha; x += alpha p, r -= alpha q, r.z_old (+ loop condition);
// z = M^-1 r; beta; p = z + beta p, on the fixed buffers of ps.
template <typename T>
static int build_loop(iga_plan *pl, SolverState *S, PrecState<T> &ps, const iga_solve_opts &o, int prec)
{
    const int scaled = pl->kappa_dev ? 1 : 0;
    if (ps.loop_pc == o.pc && ps.loop_scaled == scaled && ps.loop_prec == o.precision && (ps.loop || ps.loop_failed))
        return ps.loop ? IGA_OK : IGA_ERR_UNSUPPORTED;
    if (ps.loop) {
        cudaGraphExecDestroy(ps.loop);
        ps.loop = nullptr;
    }
    const long long N = pl->nfunc;
    const cudaStream_t s = S->stream;
    cudaGraph_t g;
    SOLVE_TRY(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    SOLVE_TRY(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    SOLVE_TRY(cudaGraphAddNode(&node, g, nullptr, 0, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    SOLVE_TRY(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    int64_t dummy = 0;
    // Programmatic dependencies between the body's kernels (the inner-CG
    // preconditioner runs child graphs and keeps ordinary edges).
    pdl_capture() = o.pc != IGA_PC_FEM_CG;
    int st = iga_apply_internal_sb(pl, prec, ps.p, ps.q, s, IGA_SIGN_SPD, IGA_BC_IDENTITY);
    auto launched = [&](cudaError_t e) {
        if (e != cudaSuccess && !st) {
            set_error(std::string("PCG loop launch: ") + cudaGetErrorString(e));
            st = IGA_ERR_CUDA;
        }
    };
    if (!st) {
        launched(launch_k(pcg_pq_kernel<T>, dim3(kRedBlocks), dim3(kThreads), 0, s, (const T *)ps.p, (const T *)ps.q,
                          N, S->s, S->partials, S->counter));
        launched(launch_k(pcg_xr_cond_kernel<T>, dim3(kRedBlocks), dim3(kThreads), 0, s, ps.x, ps.r, (const T *)ps.p,
                          (const T *)ps.q, (const T *)ps.z, N, S->s, S->partials, S->counter, h));
        if (!st) st = pc_apply(ps, pl, S, o, ps.r, ps.z, o.pc_rtol, dummy);
    }
    if (!st) {
        launched(launch_k(pcg_beta_kernel<T>, dim3(kRedBlocks), dim3(kThreads), 0, s, (const T *)ps.r,
                          (const T *)ps.z, N, S->s, S->partials, S->counter));
        launched(launch_k(pcg_p_kernel<T>, dim3(kRedBlocks), dim3(kThreads), 0, s, ps.p, (const T *)ps.z, N,
                          (const DevScalars *)S->s, 0));
    }
    pdl_capture() = false;
    cudaGraph_t captured = body;
    const cudaError_t ce = cudaStreamEndCapture(s, &captured);
    if (st || ce != cudaSuccess) {
        cudaGraphDestroy(g);
        if (!st) set_error(std::string("PCG loop capture: ") + cudaGetErrorString(ce));
        return st ? st : IGA_ERR_CUDA;
    }
    cudaGraphInstantiateParams ip = {};
    const cudaError_t ie = cudaGraphInstantiateWithParams(&ps.loop, g, &ip);
    if (ie != cudaSuccess) {
        cudaGraphNodeType t = cudaGraphNodeTypeEmpty;
        if (ip.errNode_out) cudaGraphNodeGetType(ip.errNode_out, &t);
        set_error(std::string("PCG loop instantiation: ") + cudaGetErrorString(ie) + " (result " +
                  std::to_string((int)ip.result_out) + ", node type " + std::to_string((int)t) + ")");
        cudaGetLastError();
        cudaGraphDestroy(g);
        ps.loop = nullptr;
        ps.loop_pc = o.pc;
        ps.loop_scaled = scaled;
        ps.loop_prec = o.precision;
        ps.loop_failed = true;
        return IGA_ERR_UNSUPPORTED;
    }
    cudaGraphDestroy(g);
    ps.loop_failed = false;
    ps.loop_pc = o.pc;
    ps.loop_scaled = scaled;
    ps.loop_prec = o.precision;
    return IGA_OK;
}

// Flexible PCG whose iterations run on the device: one graph launch per solve.
// x_zero: x is known to be zero and b nonzero (a refinement sweep on the
// normalised residual): r = b without the operator and no host check before
// the loop.
template <typename T>
static int pcg_graph(iga_plan *pl, SolverState *S, PrecState<T> &ps, const iga_solve_opts &o, const T *b, T *x,
                     double rtol, double bnorm, int prec, int &its, bool x_zero = false)
{
    const long long N = pl->nfunc;
    const cudaStream_t s = S->stream;
    int st;
    if ((st = update_kscale(pl, S))) return st;
    if (o.pc == IGA_PC_FEM_EXACT) {   // device set-up before any capture
        if (std::is_same<T, double>::value && o.precision == IGA_MIXED_PC) st = fd_upload(S->f, pl, S);
        else st = fd_upload(ps, pl, S);
        if (st) return st;
    }
    if (b != ps.b) copy_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(ps.b, b, N);
    if (x != ps.x) copy_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(ps.x, x, N);
    if (x_zero) {
        copy_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(ps.r, ps.b, N);
        dot_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(ps.r, ps.r, N, &S->s->rr, S->partials, S->counter);
    } else {
        if ((st = iga_apply_internal_sb(pl, prec, ps.x, ps.q, s, IGA_SIGN_SPD, IGA_BC_IDENTITY))) return st;
        sub_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(ps.b, ps.q, ps.r, N, S->s, S->partials, S->counter);
        if ((st = sync_scalars(S))) return st;
        if (std::sqrt(S->h->rr) <= rtol * bnorm) return IGA_OK;
    }
    int64_t dummy = 0;
    if ((st = pc_apply(ps, pl, S, o, ps.r, ps.z, o.pc_rtol, dummy))) return st;
    dot_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(ps.r, ps.z, N, &S->s->rz, S->partials, S->counter);
    pcg_p_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(ps.p, ps.z, N, S->s, 1);
    st = pl->solver_graph ? build_loop(pl, S, ps, o, prec) : IGA_ERR_UNSUPPORTED;
    if (st == IGA_ERR_UNSUPPORTED) {   // e.g. a library kernel not allowed in a conditional body, or the host loop asked for
        int64_t pcits = 0;
        st = pcg<T>(pl, S, ps, o, ps.b, ps.x, rtol, bnorm, o.pc_rtol, prec, its, pcits);
        if (x != ps.x) copy_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(x, ps.x, N);
        return st;
    }
    if (st) return st;
    loop_init_kernel<<<1, 1, 0, s>>>(S->s, rtol * rtol * bnorm * bnorm, o.max_it);
    SOLVE_TRY(cudaGraphLaunch(ps.loop, s));
    if (x != ps.x) copy_kernel<T><<<kRedBlocks, kThreads, 0, s>>>(x, ps.x, N);
    if ((st = sync_scalars(S))) return st;
    its += S->h->it;
    if (S->h->breakdown) return IGA_ERR_BREAKDOWN;
    if (!std::isfinite(S->h->rr)) return IGA_ERR_NONFINITE;
    return std::sqrt(S->h->rr) <= rtol * bnorm ? IGA_OK : IGA_ERR_NOT_CONVERGED;
}

// ||b - K x|| (FP64 operator), into S->h->rr and S->h->bb.
static int true_residual(iga_plan *pl, SolverState *S, const double *b, const double *x)
{
    int st;
    if ((st = iga_apply_internal_sb(pl, IGA_FP64, x, S->q64, S->stream, IGA_SIGN_SPD, IGA_BC_IDENTITY))) return st;
    residual_kernel<<<kRedBlocks, kThreads, 0, S->stream>>>(b, S->q64, S->r64, pl->nfunc, S->s, S->partials,
                                                          S->counter);
    return sync_scalars(S);
}

extern "C" {

void iga_solve_opts_default(iga_solve_opts *o)
{
    if (!o) return;
    o->precision = IGA_FP64;
    o->pc = IGA_PC_FEM_CG;
    o->rtol = 1e-10;
    o->max_it = 10000;
    o->pc_rtol = 1e-10;
    o->pc_max_it = 10000;
    o->sweep_rtol = 1e-3;
    o->max_sweeps = 10;
    o->x0_nonzero = 0;
}

int iga_fem_nodes(const iga_plan *pl, double *gx, double *gy)
{
    if (!pl || !gx || !gy) return IGA_ERR_ARG;
    double Lx, Ly;
    net_lengths(pl->patch, Lx, Ly);
    const std::vector<double> a = fem_nodes_1d(pl->p, pl->nex, Lx), b = fem_nodes_1d(pl->p, pl->ney, Ly);
    std::memcpy(gx, a.data(), a.size() * sizeof(double));
    std::memcpy(gy, b.data(), b.size() * sizeof(double));
    return IGA_OK;
}

int iga_fem_nodes_1d(int p, int ne, double L, double *g)
{
    if (!g || p < 1 || p > 5 || ne < 1 || !(L > 0.0)) return IGA_ERR_ARG;
    const std::vector<double> a = fem_nodes_1d(p, ne, L);
    std::memcpy(g, a.data(), a.size() * sizeof(double));
    return IGA_OK;
}

int iga_pc_apply(iga_plan *pl, int pc, int prec, const void *r, void *z, double pc_rtol, int pc_max_it,
                 void *stream)
{
    if (!pl || !r || !z || (prec != IGA_FP64 && prec != IGA_FP32)) return IGA_ERR_ARG;
    if (pc != IGA_PC_NONE && pc != IGA_PC_FEM_CG && pc != IGA_PC_FEM_EXACT) return IGA_ERR_ARG;
    SolverState *S;
    int st;
    if ((st = ensure_state(pl, &S))) return st;
    cudaEvent_t ev;
    SOLVE_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    SOLVE_TRY(cudaEventRecord(ev, (cudaStream_t)stream));
    SOLVE_TRY(cudaStreamWaitEvent(S->stream, ev, 0));
    iga_solve_opts o;
    iga_solve_opts_default(&o);
    o.pc = pc;
    o.pc_max_it = pc_max_it;
    int64_t its = 0;
    if (prec == IGA_FP64) {
        if ((st = alloc_prec(S->d, pl, *S))) return st;
        st = pc_apply<double>(S->d, pl, S, o, (const double *)r, (double *)z, pc_rtol, its);
    } else {
        if ((st = alloc_prec(S->f, pl, *S))) return st;
        st = pc_apply<float>(S->f, pl, S, o, (const float *)r, (float *)z, pc_rtol, its);
    }
    SOLVE_TRY(cudaEventRecord(ev, S->stream));
    SOLVE_TRY(cudaStreamWaitEvent((cudaStream_t)stream, ev, 0));
    cudaEventDestroy(ev);
    return st;
}

int iga_plan_set_pc_split(iga_plan *pl, int enable)
{
    if (!pl || (enable != 0 && enable != 1)) return IGA_ERR_ARG;
    if (pl->solver) {
        cudaSetDevice(pl->device);
        cudaDeviceSynchronize();
        iga_solver_release(pl);
    }
    pl->pc_split = enable != 0;
    return IGA_OK;
}

int iga_plan_set_solver_graph(iga_plan *pl, int enable)
{
    if (!pl || (enable != 0 && enable != 1)) return IGA_ERR_ARG;
    pl->solver_graph = enable != 0;
    return IGA_OK;
}

int iga_fem_apply(iga_plan *pl, int prec, const void *x, void *y, void *stream)
{
    if (!pl || !x || !y) return IGA_ERR_ARG;
    SolverState *S;
    int st;
    if ((st = ensure_state(pl, &S))) return st;
    if (prec == IGA_FP64) {
        if ((st = alloc_prec(S->d, pl, *S))) return st;
        fem_apply_kernel<double><<<kRedBlocks, kThreads, 0, (cudaStream_t)stream>>>(
            (const double *)x, (double *)y, coef_of(S->d, pl));
    } else if (prec == IGA_FP32) {
        if ((st = alloc_prec(S->f, pl, *S))) return st;
        fem_apply_kernel<float><<<kRedBlocks, kThreads, 0, (cudaStream_t)stream>>>((const float *)x, (float *)y,
                                                                                 coef_of(S->f, pl));
    } else {
        return IGA_ERR_ARG;
    }
    SOLVE_TRY(cudaGetLastError());
    return IGA_OK;
}

int iga_fem_assemble_csr(iga_plan *pl, int sign, int32_t *rowptr, int32_t *col, double *val, int64_t *nnz,
                         void *stream)
{
    if (!pl || (sign != 1 && sign != -1)) return IGA_ERR_ARG;
    const int m = pl->m, n = pl->n;
    // Row lengths: 1 on the boundary, (free neighbours in x) * (free neighbours in y) inside.
    auto cnt = [](int i, int mm) { return 1 + (i - 1 >= 1) + (i + 1 <= mm - 2); };
    std::vector<int32_t> rp((size_t)m * n + 1);
    long long acc = 0;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            rp[(size_t)j * m + i] = (int32_t)acc;
            const bool b = i == 0 || j == 0 || i == m - 1 || j == n - 1;
            acc += b ? 1 : cnt(i, m) * cnt(j, n);
        }
    rp[(size_t)m * n] = (int32_t)acc;
    if (acc > INT32_MAX) return IGA_ERR_UNSUPPORTED;
    if (nnz) *nnz = acc;
    if (!rowptr && !col && !val) return IGA_OK;
    if (!rowptr || !col || !val) return IGA_ERR_ARG;
    SolverState *S;
    int st;
    if ((st = ensure_state(pl, &S))) return st;
    if ((st = alloc_prec(S->d, pl, *S))) return st;
    cudaStream_t s = (cudaStream_t)stream;
    SOLVE_TRY(cudaMemcpyAsync(rowptr, rp.data(), rp.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    fem_csr_kernel<<<kRedBlocks, kThreads, 0, s>>>(rowptr, col, val, coef_of(S->d, pl), (double)sign);
    SOLVE_TRY(cudaStreamSynchronize(s));
    return IGA_OK;
}

int iga_solve(iga_plan *pl, const double *b, double *x, const iga_solve_opts *o_in, iga_solve_stats *stats,
              void *stream)
{
    if (!pl || !b || !x) return IGA_ERR_ARG;
    iga_solve_opts o;
    iga_solve_opts_default(&o);
    if (o_in) o = *o_in;
    if (o.pc != IGA_PC_NONE && o.pc != IGA_PC_FEM_CG && o.pc != IGA_PC_FEM_EXACT) {
        set_error("unknown preconditioner");
        return IGA_ERR_ARG;
    }
    if (!pl->op64.ready) {
        set_error("iga_solve needs the FP64 operator (plan precision IGA_FP64 or IGA_MIXED)");
        return IGA_ERR_ARG;
    }
    if (o.precision != IGA_FP64 && o.precision != IGA_MIXED && o.precision != IGA_MIXED_PC) {
        set_error("iga_solve precision is IGA_FP64, IGA_MIXED or IGA_MIXED_PC");
        return IGA_ERR_ARG;
    }
    if (o.precision == IGA_MIXED && !pl->op32.ready) {
        set_error("IGA_MIXED solves need a plan created with precision IGA_MIXED");
        return IGA_ERR_ARG;
    }
    SolverState *S;
    int st;
    if ((st = ensure_state(pl, &S))) return st;
    SOLVE_TRY(cudaSetDevice(pl->device));
    const auto t0 = std::chrono::steady_clock::now();
    // Order the solve after the caller's stream and the caller's stream after the solve.
    cudaEvent_t ev;
    SOLVE_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    SOLVE_TRY(cudaEventRecord(ev, (cudaStream_t)stream));
    SOLVE_TRY(cudaStreamWaitEvent(S->stream, ev, 0));
    const long long N = pl->nfunc;
    iga_solve_stats stt{};
    SOLVE_TRY(cudaMemsetAsync(&S->s->err, 0, sizeof(int), S->stream));
    if (!o.x0_nonzero) zero_kernel<double><<<kRedBlocks, kThreads, 0, S->stream>>>(x, N);
    if ((st = true_residual(pl, S, b, x))) return st;
    if (!std::isfinite(S->h->bb) || !std::isfinite(S->h->rr)) {
        cudaEventDestroy(ev);
        if (stats) {
            *stats = iga_solve_stats{};
            stats->status = IGA_ERR_NONFINITE;
            stats->relres = NAN;
        }
        set_error("non-finite value in b or in the initial residual");
        return IGA_ERR_NONFINITE;
    }
    const double bnorm = std::sqrt(S->h->bb);
    double rel = bnorm > 0 ? std::sqrt(S->h->rr) / bnorm : 0.0;
    int result = IGA_OK;
    if (o.precision != IGA_MIXED) {
        if ((st = alloc_prec(S->d, pl, *S))) return st;
        if (o.precision == IGA_MIXED_PC && o.pc != IGA_PC_NONE && (st = alloc_prec(S->f, pl, *S))) return st;
        // Restart from the true residual until it meets rtol (recurrence drift).
        for (int restart = 0; restart < 4 && rel > o.rtol; ++restart) {
            st = o.pc == IGA_PC_FEM_CG
                     ? pcg<double>(pl, S, S->d, o, b, x, o.rtol, bnorm, o.pc_rtol, IGA_FP64, stt.iterations,
                                   stt.pc_iterations)
                     : pcg_graph<double>(pl, S, S->d, o, b, x, o.rtol, bnorm, IGA_FP64, stt.iterations);
            if (st && st != IGA_ERR_NOT_CONVERGED) {
                result = st;
                break;
            }
            if ((st = true_residual(pl, S, b, x))) return st;
            rel = std::sqrt(S->h->rr) / bnorm;
            if (!std::isfinite(rel)) {
                result = IGA_ERR_NONFINITE;
                break;
            }
        }
    } else {
        if ((st = alloc_prec(S->f, pl, *S))) return st;
        for (int sw = 0; sw < o.max_sweeps && rel > o.rtol; ++sw) {
            // rhs of the sweep: r64 / ||r64|| in FP32; correction d solves K d = r / ||r||.
            const double scale = std::sqrt(S->h->rr);
            // A sweep asks for sweep_rtol, or for less when less is left to do:
            // a fifth of the reduction that would reach rtol (margin for the
            // FP32 recurrence residual drifting from the FP64 one).
            const double need = o.rtol * bnorm / scale;
            const double srtol = std::max(o.sweep_rtol, std::min(0.2 * need, 0.5));
            scale_down_kernel<<<kRedBlocks, kThreads, 0, S->stream>>>(S->r64, S->f.b, N, S->s);
            zero_kernel<float><<<kRedBlocks, kThreads, 0, S->stream>>>(S->f.x, N);
            st = o.pc == IGA_PC_FEM_CG
                     ? pcg<float>(pl, S, S->f, o, S->f.b, S->f.x, srtol, 1.0, o.pc_rtol, IGA_FP32, stt.iterations,
                                  stt.pc_iterations)
                     : pcg_graph<float>(pl, S, S->f, o, S->f.b, S->f.x, srtol, 1.0, IGA_FP32, stt.iterations, true);
            if (st && st != IGA_ERR_NOT_CONVERGED) {
                result = st;
                break;
            }
            refine_update_kernel<<<kRedBlocks, kThreads, 0, S->stream>>>(x, S->f.x, N, scale);
            ++stt.sweeps;
            if ((st = true_residual(pl, S, b, x))) return st;
            rel = std::sqrt(S->h->rr) / bnorm;
            if (!std::isfinite(rel)) {
                result = IGA_ERR_NONFINITE;
                break;
            }
        }
    }
    SOLVE_TRY(cudaEventRecord(ev, S->stream));
    SOLVE_TRY(cudaStreamWaitEvent((cudaStream_t)stream, ev, 0));
    SOLVE_TRY(cudaStreamSynchronize(S->stream));
    cudaEventDestroy(ev);
    stt.relres = rel;
    if (S->h->err) {   // host copy current as of the last true residual
        set_error("a bounded device wait gave up in the preconditioner");
        result = IGA_ERR_TIMEOUT;
    }
    if (result == IGA_OK && !(rel <= o.rtol)) result = IGA_ERR_NOT_CONVERGED;
    stt.status = result;
    stt.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (stats) *stats = stt;
    return result;
}

int iga_spectrum_estimate(iga_plan *pl, int pc, int steps, uint64_t seed, double *lam_min, double *lam_max,
                          int *steps_done)
{
    if (!pl || !lam_min || !lam_max || steps < 1) return IGA_ERR_ARG;
    if (pc != IGA_PC_NONE && pc != IGA_PC_FEM_CG && pc != IGA_PC_FEM_EXACT) return IGA_ERR_ARG;
    if (!pl->op64.ready) {
        set_error("iga_spectrum_estimate needs the FP64 operator");
        return IGA_ERR_ARG;
    }
    SolverState *S;
    int st;
    if ((st = ensure_state(pl, &S))) return st;
    SOLVE_TRY(cudaSetDevice(pl->device));
    if ((st = alloc_prec(S->d, pl, *S))) return st;
    PrecState<double> &ps = S->d;
    const long long N = pl->nfunc;
    const cudaStream_t s = S->stream;
    iga_solve_opts o;
    iga_solve_opts_default(&o);
    o.pc = pc;
    o.pc_rtol = 1e-13;
    // seeded random start vector, zero on the boundary ring (the Krylov space
    // stays on the free control points: identity rows and identity PC rows)
    std::vector<double> h((size_t)N);
    std::mt19937_64 gen(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    for (int j = 0; j < pl->n; ++j)
        for (int i = 0; i < pl->m; ++i)
            h[(size_t)j * pl->m + i] = (i == 0 || j == 0 || i == pl->m - 1 || j == pl->n - 1) ? 0.0 : nd(gen);
    SOLVE_TRY(cudaMemcpyAsync(ps.r, h.data(), sizeof(double) * N, cudaMemcpyHostToDevice, s));
    zero_kernel<double><<<kRedBlocks, kThreads, 0, s>>>(ps.x, N);
    int64_t pcits = 0;
    if ((st = pc_apply(ps, pl, S, o, ps.r, ps.z, o.pc_rtol, pcits))) return st;
    dot_kernel<double><<<kRedBlocks, kThreads, 0, s>>>(ps.r, ps.z, N, &S->s->rz, S->partials, S->counter);
    pcg_p_kernel<double><<<kRedBlocks, kThreads, 0, s>>>(ps.p, ps.z, N, S->s, 1);
    SOLVE_TRY(cudaMemsetAsync(&S->s->breakdown, 0, sizeof(int), s));
    if ((st = sync_scalars(S))) return st;
    const double rr0 = S->h->rz;
    std::vector<double> alpha, beta;
    for (int k = 0; k < steps; ++k) {
        const double rz_old = S->h->rz;
        if ((st = iga_apply_internal_sb(pl, IGA_FP64, ps.p, ps.q, s, IGA_SIGN_SPD, IGA_BC_IDENTITY))) return st;
        pcg_pq_kernel<double><<<kRedBlocks, kThreads, 0, s>>>(ps.p, ps.q, N, S->s, S->partials, S->counter);
        pcg_xr_kernel<double><<<kRedBlocks, kThreads, 0, s>>>(ps.x, ps.r, ps.p, ps.q, ps.z, N, S->s, S->partials,
                                                             S->counter);
        if ((st = pc_apply(ps, pl, S, o, ps.r, ps.z, o.pc_rtol, pcits))) return st;
        dot_kernel<double><<<kRedBlocks, kThreads, 0, s>>>(ps.r, ps.z, N, &S->s->rz, S->partials, S->counter);
        if ((st = sync_scalars(S))) return st;
        if (S->h->breakdown || !(S->h->alpha > 0.0)) break;
        alpha.push_back(S->h->alpha);
        const double rz_new = S->h->rz;
        if (!(rz_new > 1e-28 * rr0)) break;   // the Krylov space is exhausted
        beta.push_back(rz_new / rz_old);
        S->h->beta = beta.back();
        SOLVE_TRY(cudaMemcpyAsync(&S->s->beta, &S->h->beta, sizeof(double), cudaMemcpyHostToDevice, s));
        pcg_p_kernel<double><<<kRedBlocks, kThreads, 0, s>>>(ps.p, ps.z, N, S->s, 0);
    }
    const int K = (int)alpha.size();
    if (K < 1) {
        set_error("iga_spectrum_estimate: no Lanczos step completed");
        return IGA_ERR_BREAKDOWN;
    }
    // Lanczos matrix of the PCG coefficients: T_kk = 1/a_k + b_{k-1}/a_{k-1},
    // T_k,k+1 = sqrt(b_k) / a_k (M^-1 K in the M-inner product)
    std::vector<double> Td(K), To(K, 0.0), Md(K, 1.0), Mo(K, 0.0), lam(K), V((size_t)K * K);
    for (int k = 0; k < K; ++k) {
        Td[k] = 1.0 / alpha[k] + (k > 0 ? beta[k - 1] / alpha[k - 1] : 0.0);
        if (k + 1 < K) To[k] = -std::sqrt(beta[k]) / alpha[k];
    }
    pencil_eig(K, Td.data(), To.data(), Md.data(), Mo.data(), lam.data(), V.data());
    *lam_min = lam[0];
    *lam_max = lam[K - 1];
    if (steps_done) *steps_done = K;
    return IGA_OK;
}

}  // extern "C"
