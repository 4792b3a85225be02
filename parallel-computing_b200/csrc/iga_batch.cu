// Batched solves (include/iga_batch.h): many independent single-patch
// Poisson problems of uneven size and degree, advanced together.
//
// Layout: every batch vector is the concatenation of the problems' vectors.
// Work lists cover the whole batch in each launch:
//   - operator: one CTA per (problem, column strip, block of W row strips),
//     one launch per degree present (the degrees' launches run concurrently),
//     then one seam launch for all problems;
//   - vector updates and reductions: fixed chunks of kChunkLen entries, never
//     crossing a problem; each problem's dot products are summed in chunk
//     order by its last chunk (deterministic, no atomics on values);
//   - preconditioner: 64 x 64 output tiles of four GEMM stages per problem
//     (exact FEM inverse by fast diagonalisation).
// Per-problem scalars live on the device; a problem that has converged is
// marked inactive and every later launch skips its items. The PCG iteration
// is the body of a conditional WHILE node; mixed precision nests the FP32
// PCG loop inside a WHILE loop over FP64 refinement sweeps, so a batch solve
// is one graph launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <atomic>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "../../include/iga_batch.h"
#include "iga_apply.cuh"
#include "iga_fastdiag.hpp"
#include "iga_fem.hpp"
#include "iga_plan.hpp"
#include "iga_tune.hpp"
#include "iga_umma.cuh"

namespace iga {

constexpr int kBT = 256;          // threads of the vector / reduction kernels
constexpr int kChunkLen = 2048;   // entries per reduction chunk
constexpr int kTile = 64;         // preconditioner GEMM output tile (kTile x kTile)
constexpr int kTK = 16;           // GEMM k-step

// Per-problem solver scalars.
struct BScal {
    double alpha, beta, rz, rr, rzo, tol2, bb, scale, relres;
    int it, itot, status, sweeps;
};

struct BCfg {
    double rtol, sweep_rtol2;
    int maxit, max_sweeps;
};

struct BDev {
    const int4 *chunks;   // (problem, start in problem, length, -)
    const int *c0, *nc;   // first chunk and chunk count of each problem
    const long long *off; // vector offset of each problem
    double *partials;     // [chunk][4]
    unsigned *counters;   // per problem
    BScal *sc;
    const BCfg *cfg;
};

// ------------------------------------------------------------ reductions
// Sums K values over the chunks of problem pr; the problem's last chunk to
// finish adds the chunk partials in chunk order and returns true (thread 0
// holds the totals). Chunk c of the launch is blockIdx.x.
template <int K>
__device__ bool chunk_reduce(double (&v)[K], int pr, const BDev &d, double (&tot)[K])
{
    __shared__ double sh[K][kBT / 32];
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
            for (int w = 0; w < kBT / 32; ++w) s += sh[k][w];
            d.partials[(size_t)blockIdx.x * 4 + k] = s;
        }
        __threadfence();
        const unsigned t = atomicAdd(&d.counters[pr], 1u);
        last = (t == (unsigned)d.nc[pr] - 1u);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    const int first = d.c0[pr], cnt = d.nc[pr];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (int b = threadIdx.x; b < cnt; b += kBT) s += ((volatile double *)d.partials)[(size_t)(first + b) * 4 + k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) sh[k][wid] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = 0.0;
            for (int w = 0; w < kBT / 32; ++w) s += sh[k][w];
            tot[k] = s;
        }
        d.counters[pr] = 0u;
    }
    return true;
}

// ------------------------------------------------------------ vector kernels
// FP64 PCG start: r = b - q (q = K x), rr, bb; tol2 = rtol^2 bb.
__global__ void __launch_bounds__(kBT) bk_init64(BDev d, const int *__restrict__ act64, int *__restrict__ act,
                                                 const double *__restrict__ b, const double *__restrict__ q,
                                                 double *__restrict__ r)
{
    const int4 ck = d.chunks[blockIdx.x];
    const int pr = ck.x;
    if (!act64[pr]) return;
    const long long base = d.off[pr] + ck.y;
    double v[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < ck.z; i += kBT) {
        const long long t = base + i;
        const double rv = b[t] - q[t];
        r[t] = rv;
        v[0] += rv * rv;
        v[1] += b[t] * b[t];
    }
    double tot[2];
    if (chunk_reduce<2>(v, pr, d, tot) && threadIdx.x == 0) {
        BScal &S = d.sc[pr];
        S.rr = tot[0];
        S.bb = tot[1];
        S.tol2 = d.cfg->rtol * d.cfg->rtol * tot[1];
        S.it = 0;
        const bool fin = isfinite(tot[0]) && isfinite(tot[1]);
        if (!fin) S.status = IGA_ERR_NONFINITE;
        act[pr] = (fin && tot[0] > S.tol2) ? 1 : 0;
    }
}

// FP64 true residual r64 = b - q64 after a PCG run or a refinement sweep.
// mode 0: plain FP64 solve (act64 stays set while relres > rtol, for a
// restart); mode 1: after a mixed sweep (counts it); mode 2: before the first
// sweep. act64 cleared once relres <= rtol, on failure, or out of sweeps.
__global__ void __launch_bounds__(kBT) bk_res64(BDev d, int *__restrict__ act64, const double *__restrict__ b,
                                                const double *__restrict__ q, double *__restrict__ r, int mode)
{
    const int4 ck = d.chunks[blockIdx.x];
    const int pr = ck.x;
    if (!act64[pr]) return;
    const long long base = d.off[pr] + ck.y;
    double v[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < ck.z; i += kBT) {
        const long long t = base + i;
        const double rv = b[t] - q[t];
        r[t] = rv;
        v[0] += rv * rv;
        v[1] += b[t] * b[t];
    }
    double tot[2];
    if (chunk_reduce<2>(v, pr, d, tot) && threadIdx.x == 0) {
        BScal &S = d.sc[pr];
        S.bb = tot[1];
        S.scale = sqrt(tot[0]);
        S.relres = tot[1] > 0.0 ? sqrt(tot[0] / tot[1]) : sqrt(tot[0]);
        S.itot += S.it;
        S.it = 0;
        if (mode == 1) S.sweeps += 1;
        const bool fin = isfinite(S.relres);
        if (!fin) S.status = IGA_ERR_NONFINITE;
        bool go = fin && S.status == 0 && S.relres > d.cfg->rtol;
        if (mode != 0) go = go && S.sweeps < d.cfg->max_sweeps;
        act64[pr] = go ? 1 : 0;
    }
}

// Mixed sweep start: r32 = r64 / ||r64||, x32 = 0, rr; tol2 = t^2 rr with t =
// sweep_rtol, or less reduction when less is left: a fifth of what would
// reach rtol (margin for the FP32 recurrence residual's drift).
__global__ void __launch_bounds__(kBT) bk_sweep_init(BDev d, const int *__restrict__ act64, int *__restrict__ act,
                                                     const double *__restrict__ r64, float *__restrict__ r32,
                                                     float *__restrict__ x32)
{
    const int4 ck = d.chunks[blockIdx.x];
    const int pr = ck.x;
    if (!act64[pr]) return;
    const long long base = d.off[pr] + ck.y;
    const double sc = d.sc[pr].scale;
    const double inv = sc > 0.0 ? 1.0 / sc : 0.0;
    double v[1] = {0.0};
    for (int i = threadIdx.x; i < ck.z; i += kBT) {
        const long long t = base + i;
        const float rv = (float)(r64[t] * inv);
        r32[t] = rv;
        x32[t] = 0.0f;
        v[0] += (double)rv * (double)rv;
    }
    double tot[1];
    if (chunk_reduce<1>(v, pr, d, tot) && threadIdx.x == 0) {
        BScal &S = d.sc[pr];
        S.rr = tot[0];
        const double need = sc > 0.0 ? d.cfg->rtol * sqrt(S.bb) / sc : 0.0;
        const double t = fmax(sqrt(d.cfg->sweep_rtol2), fmin(0.2 * need, 0.5));
        S.tol2 = t * t * tot[0];
        S.it = 0;
        act[pr] = (isfinite(tot[0]) && tot[0] > S.tol2) ? 1 : 0;
    }
}

// rz = r.z and the first direction p = z.
template <typename T>
__global__ void __launch_bounds__(kBT) bk_rz_p(BDev d, const int *__restrict__ act, const T *__restrict__ r,
                                               const T *__restrict__ z, T *__restrict__ p)
{
    const int4 ck = d.chunks[blockIdx.x];
    const int pr = ck.x;
    if (!act[pr]) return;
    const long long base = d.off[pr] + ck.y;
    double v[1] = {0.0};
    for (int i = threadIdx.x; i < ck.z; i += kBT) {
        const long long t = base + i;
        const T zv = z[t];
        p[t] = zv;
        v[0] += (double)r[t] * (double)zv;
    }
    double tot[1];
    if (chunk_reduce<1>(v, pr, d, tot) && threadIdx.x == 0) d.sc[pr].rz = tot[0];
}

// alpha = rz / p.q (breakdown when p.q <= 0 or not finite).
template <typename T>
__global__ void __launch_bounds__(kBT) bk_pq(BDev d, int *__restrict__ act, const T *__restrict__ p,
                                             const T *__restrict__ q)
{
    const int4 ck = d.chunks[blockIdx.x];
    const int pr = ck.x;
    if (!act[pr]) return;
    const long long base = d.off[pr] + ck.y;
    double v[1] = {0.0};
    for (int i = threadIdx.x; i < ck.z; i += kBT) {
        const long long t = base + i;
        v[0] += (double)p[t] * (double)q[t];
    }
    double tot[1];
    if (chunk_reduce<1>(v, pr, d, tot) && threadIdx.x == 0) {
        BScal &S = d.sc[pr];
        if (!(tot[0] > 0.0) || !isfinite(tot[0])) {
            S.status = isfinite(tot[0]) ? IGA_ERR_BREAKDOWN : IGA_ERR_NONFINITE;
            S.alpha = 0.0;
            act[pr] = 0;
        } else {
            S.alpha = S.rz / tot[0];
        }
    }
}

// x += alpha p, r -= alpha q; rr = r.r and rzo = r.z_old (z not yet replaced);
// counts the iteration and deactivates the problem when rr <= tol2.
template <typename T>
__global__ void __launch_bounds__(kBT) bk_xr(BDev d, int *__restrict__ act, T *__restrict__ x, T *__restrict__ r,
                                             const T *__restrict__ p, const T *__restrict__ q,
                                             const T *__restrict__ z)
{
    const int4 ck = d.chunks[blockIdx.x];
    const int pr = ck.x;
    if (!act[pr]) return;
    const long long base = d.off[pr] + ck.y;
    const T al = (T)d.sc[pr].alpha;
    double v[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < ck.z; i += kBT) {
        const long long t = base + i;
        x[t] += al * p[t];
        const T rv = r[t] - al * q[t];
        r[t] = rv;
        v[0] += (double)rv * (double)rv;
        v[1] += (double)rv * (double)z[t];
    }
    double tot[2];
    if (chunk_reduce<2>(v, pr, d, tot) && threadIdx.x == 0) {
        BScal &S = d.sc[pr];
        S.rr = tot[0];
        S.rzo = tot[1];
        S.it += 1;
        const bool fin = isfinite(tot[0]);
        if (!fin) S.status = IGA_ERR_NONFINITE;
        act[pr] = (fin && tot[0] > S.tol2 && S.it < d.cfg->maxit) ? 1 : 0;
    }
}

// Flexible (Polak-Ribiere) beta = (r.z - r.z_old) / rz_old; rz = r.z.
template <typename T>
__global__ void __launch_bounds__(kBT) bk_beta(BDev d, const int *__restrict__ act, const T *__restrict__ r,
                                               const T *__restrict__ z)
{
    const int4 ck = d.chunks[blockIdx.x];
    const int pr = ck.x;
    if (!act[pr]) return;
    const long long base = d.off[pr] + ck.y;
    double v[1] = {0.0};
    for (int i = threadIdx.x; i < ck.z; i += kBT) {
        const long long t = base + i;
        v[0] += (double)r[t] * (double)z[t];
    }
    double tot[1];
    if (chunk_reduce<1>(v, pr, d, tot) && threadIdx.x == 0) {
        BScal &S = d.sc[pr];
        S.beta = (tot[0] - S.rzo) / S.rz;
        S.rz = tot[0];
    }
}

template <typename T>
__global__ void __launch_bounds__(kBT) bk_p(BDev d, const int *__restrict__ act, T *__restrict__ p,
                                            const T *__restrict__ z)
{
    const int4 ck = d.chunks[blockIdx.x];
    const int pr = ck.x;
    if (!act[pr]) return;
    const long long base = d.off[pr] + ck.y;
    const T be = (T)d.sc[pr].beta;
    for (int i = threadIdx.x; i < ck.z; i += kBT) {
        const long long t = base + i;
        p[t] = z[t] + be * p[t];
    }
}

template <typename T>
__global__ void __launch_bounds__(kBT) bk_copy(BDev d, const int *__restrict__ act, const T *__restrict__ src,
                                               T *__restrict__ dst)
{
    const int4 ck = d.chunks[blockIdx.x];
    const int pr = ck.x;
    if (!act[pr]) return;
    const long long base = d.off[pr] + ck.y;
    for (int i = threadIdx.x; i < ck.z; i += kBT) dst[base + i] = src[base + i];
}

// Refinement update x64 += ||r64|| * d32 of every problem still refining.
__global__ void __launch_bounds__(kBT) bk_refine(BDev d, const int *__restrict__ act64, double *__restrict__ x,
                                                 const float *__restrict__ d32)
{
    const int4 ck = d.chunks[blockIdx.x];
    const int pr = ck.x;
    if (!act64[pr]) return;
    const long long base = d.off[pr] + ck.y;
    const double sc = d.sc[pr].scale;
    for (int i = threadIdx.x; i < ck.z; i += kBT) x[base + i] += sc * (double)d32[base + i];
}

// Loop condition: does any problem remain active?
__global__ void __launch_bounds__(kBT) bk_cond(const int *__restrict__ act, int n, cudaGraphConditionalHandle h)
{
    int any = 0;
    for (int i = threadIdx.x; i < n; i += kBT) any |= act[i];
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

// ------------------------------------------------------------ exact FEM inverse, batched
// z = K_fem^-1 r on the free nodes of every problem (R, Z the interior blocks
// of r, z: column-major nx x ny, rows = x), z = r on the boundary ring. With
// Kx Vx = Mx Vx diag(lx), K_fem = Kx (x) My + Mx (x) Ky becomes the tridiagonal
// y system lx[a] My + Ky for every x mode a:
//   stage 1: W1 = Vx^T R                     (GEMM tiles of all active problems)
//   rows:    row a of W1 solved along y      (one thread per (problem, a))
//   stage 3: Z = Vx W1, scattered into z     (GEMM tiles)
template <typename T>
struct FdProb {
    const T *Vx, *lx;      // x eigenvectors (column-major, ld nx) and eigenvalues
    const T *VxT;          // the transpose of Vx (column-major), for the tcgen05 tiles
    const T *Vxp, *VxTp;   // FP32: Vx and VxT with columns padded to ldv (a multiple of 4): 16-byte rows
    int ldv;
    const T *Dv, *Cf;      // LDL^T factors of the y systems: 1 / pivot, upper off-diagonal; [b][a], ld nx
    const double *yc;      // free y nodes' pencil Kd | Ko | Md | Mo (ny each)
    T *W1;                 // nx * ny work matrix
    long long off;         // vector offset of the problem
    int m, n, nx, ny;
};

// Row solves of the y systems: forward y_b = Dv_b w_b + beta_b y_{b-1},
// beta_b = -e_{b-1} Dv_b, backward x_b = y_b - C_b x_{b+1}, e_b = lx[a] Mo_b +
// Ko_b. A block takes 32 consecutive x modes (threadIdx.x, coalesced rows) and
// cuts y into kRowSeg segments (threadIdx.y): each thread solves its segment
// in registers with a zero carry-in, the segments' affine carry maps
// (c -> end + prod c) are composed through shared memory, and each thread
// adds its carry times the running coefficient product. One read of W, Dv, C
// and one write of W. rows = (problem, first x mode) per block.
constexpr int kRowSeg = 16;                // segments per row
constexpr int kRowLen = 17;                // rows per segment: ny <= kRowSeg * kRowLen (patches up to 272 free nodes)

template <typename T>
__global__ void __launch_bounds__(32 * kRowSeg, sizeof(T) == 4 ? 2 : 1) fd_rows_kernel(const FdProb<T> *__restrict__ fps,
                                                              const int2 *__restrict__ rows,
                                                              const int *__restrict__ act)
{
    using R = T;   // segment arithmetic in the preconditioner's precision (registers: 2 blocks per SM in FP32)
    __shared__ R mE[kRowSeg][32], mP[kRowSeg][32];
    const int2 rw = rows[blockIdx.x];
    if (!act[rw.x]) return;
    const FdProb<T> &f = fps[rw.x];
    const int nx = f.nx, ny = f.ny;
    const int a = rw.y + threadIdx.x, sg = threadIdx.y;
    const int seglen = (ny + kRowSeg - 1) / kRowSeg;   // <= kRowLen
    const int b0 = sg * seglen, len = max(0, min(seglen, ny - b0));
    const bool live = a < nx;
    const R lam = live ? f.lx[a] : R(0);
    const double *yc = f.yc;
    T *W = f.W1;
    R w[kRowLen], c[kRowLen];
#pragma unroll
    for (int k = 0; k < kRowLen; ++k) {
        const bool in = live && k < len;
        w[k] = in ? W[a + (size_t)(b0 + k) * nx] : R(0);
        c[k] = in ? f.Dv[a + (size_t)(b0 + k) * nx] : R(0);   // Dv now, C later
    }
    // forward, zero carry-in; c[k] becomes beta_k
    R y = 0, pr = 1;
#pragma unroll
    for (int k = 0; k < kRowLen; ++k) {
        if (k < len) {
            const int b = b0 + k;
            const R beta = b == 0 ? R(0) : -(lam * (R)yc[3 * ny + b - 1] + (R)yc[ny + b - 1]) * c[k];
            y = c[k] * w[k] + beta * y;
            pr *= beta;
            w[k] = y;
            c[k] = beta;
        }
    }
    mE[sg][threadIdx.x] = y;
    mP[sg][threadIdx.x] = pr;
    __syncthreads();
    R cin = 0;
    for (int s2 = 0; s2 < sg; ++s2) cin = mE[s2][threadIdx.x] + mP[s2][threadIdx.x] * cin;
    R r = 1;
#pragma unroll
    for (int k = 0; k < kRowLen; ++k) {
        if (k < len) {
            r *= c[k];
            w[k] += r * cin;
        }
    }
    __syncthreads();   // carry maps read; the backward pass reuses them
#pragma unroll
    for (int k = 0; k < kRowLen; ++k) c[k] = (live && k < len) ? f.Cf[a + (size_t)(b0 + k) * nx] : R(0);
    R x = 0, q = 1;
#pragma unroll
    for (int k = kRowLen - 1; k >= 0; --k) {
        if (k < len) {
            x = w[k] - c[k] * x;
            q *= -c[k];
            w[k] = x;
        }
    }
    mE[sg][threadIdx.x] = x;
    mP[sg][threadIdx.x] = q;
    __syncthreads();
    cin = 0;
    for (int s2 = kRowSeg - 1; s2 > sg; --s2) cin = mE[s2][threadIdx.x] + mP[s2][threadIdx.x] * cin;
    r = 1;
#pragma unroll
    for (int k = kRowLen - 1; k >= 0; --k) {
        if (k < len) {
            r *= -c[k];
            if (live) W[a + (size_t)(b0 + k) * nx] = (T)(w[k] + r * cin);
        }
    }
}

// Tensor-core tiles: FP64 through DMMA (mma.sync m16n8k8, FP64 accumulate),
// FP32 through TF32 MMA (mma.sync m16n8k8, operands rounded to TF32 once when
// staged, FP32 accumulate): the FP32 preconditioner only has to be a close
// SPD approximation of K_fem^-1 (the flexible PCG and the FP64 refinement
// absorb the difference).
// FP64: D (16 x 8) += A (16 x 8) B (8 x 8); fragments (g = lane / 4, t = lane % 4)
// a = A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4]; b = B[t][g], B[t+4][g];
// d = D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1] (the layout of the FP32 tile).
__device__ __forceinline__ void mma_tile(double (&d)[4], const double (&a)[4], const double (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

__device__ __forceinline__ void mma_tile(float (&d)[4], const float (&a)[4], const float (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(__float_as_uint(a[0])), "r"(__float_as_uint(a[1])), "r"(__float_as_uint(a[2])),
          "r"(__float_as_uint(a[3])), "r"(__float_as_uint(b[0])), "r"(__float_as_uint(b[1])));
}

__device__ __forceinline__ double to_operand(double v) { return v; }
__device__ __forceinline__ float to_operand(float v)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return __uint_as_float(r);
}

// 64 x 64 output tile of one problem per CTA of 4 warps (2 x 2 warp tiles of
// 32 x 32). Operands contiguous along k in memory are staged as [row][k]
// (ld 20), the others as [k][row] (ld 72): both make the fragment loads of a
// warp conflict-free. Row / column blocks entirely outside the problem skip
// their MMAs.
template <typename T, int STAGE>
__global__ void __launch_bounds__(128) fd_gemm_kernel(const FdProb<T> *__restrict__ fps, const int4 *__restrict__ tiles,
                                                      const int *__restrict__ act, const T *__restrict__ rb,
                                                      T *__restrict__ zb)
{
    static_assert(STAGE == 1 || STAGE == 3, "stages 1 (W1 = Vx^T R) and 3 (Z = Vx W1)");
    constexpr bool A_KF = STAGE == 1;   // A contiguous along k: staged [a][k]
    constexpr bool B_KF = true;         // B contiguous along k: staged [b][k]
    constexpr int LKF = 20, LRF = 72;
    constexpr int SA = A_KF ? kTile * LKF : kTK * LRF;
    constexpr int SB = B_KF ? kTile * LKF : kTK * LRF;
    __shared__ __align__(16) T As[2][SA];
    __shared__ __align__(16) T Bs[2][SB];
    const int4 tl = tiles[blockIdx.x];
    if (!act[tl.x]) return;
    const FdProb<T> &f = fps[tl.x];
    const int nx = f.nx, ny = f.ny, m = f.m;
    const int K = nx;
    const int a0 = tl.y * kTile, b0 = tl.z * kTile;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int wm = (w & 1) * 32, wn = (w >> 1) * 32;
    const T *r = rb + f.off;
    T *z = zb + f.off;

    if (STAGE == 1 && tl.y == 0 && tl.z == 0) {   // boundary ring: identity rows of K_fem
        const int n = f.n;
        const int nb = 2 * m + 2 * (n - 2);
        for (int u = tid; u < nb; u += 128) {
            int idx;
            if (u < m) idx = u;
            else if (u < 2 * m) idx = (n - 1) * m + (u - m);
            else {
                const int v = u - 2 * m;
                idx = (1 + v / 2) * m + ((v & 1) ? (m - 1) : 0);
            }
            z[idx] = r[idx];
        }
    }

    auto ldA = [&](int a, int k) -> T {
        if (a >= nx || k >= K) return T(0);
        if (STAGE == 1) return f.Vx[(size_t)a * nx + k];          // Vx^T
        return f.Vx[(size_t)k * nx + a];                          // Vx (stage 3)
    };
    auto ldB = [&](int k, int b) -> T {
        if (k >= K || b >= ny) return T(0);
        if (STAGE == 1) return r[(size_t)(b + 1) * m + (k + 1)];   // R
        return f.W1[(size_t)b * nx + k];                          // W1 after the row solves (stage 3)
    };
    // element (row, k) of this thread's i-th fetch, coalesced along the contiguous index
    auto coord = [&](bool kf, int i, int &row, int &k) {
        if (kf) {
            k = tid & 15;
            row = (tid >> 4) + 8 * i;
        } else {
            row = tid & 63;
            k = (tid >> 6) + 2 * i;
        }
    };
    T ra[8], rbv[8];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            int row, k;
            coord(A_KF, i, row, k);
            ra[i] = ldA(a0 + row, k0 + k);
            coord(B_KF, i, row, k);
            rbv[i] = ldB(k0 + k, b0 + row);
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            int row, k;
            coord(A_KF, i, row, k);
            As[buf][A_KF ? row * LKF + k : k * LRF + row] = to_operand(ra[i]);
            coord(B_KF, i, row, k);
            Bs[buf][B_KF ? row * LKF + k : k * LRF + row] = to_operand(rbv[i]);
        }
    };
    auto Aat = [&](int buf, int row, int k) -> T { return As[buf][A_KF ? row * LKF + k : k * LRF + row]; };
    auto Bat = [&](int buf, int k, int col) -> T { return Bs[buf][B_KF ? col * LKF + k : k * LRF + col]; };

    constexpr int MB = 2;      // row blocks of 16 rows in the warp tile (m16n8k8 in both precisions)
    constexpr int RB = 16;
    constexpr int NACC = 4;
    T acc[MB][4][NACC];
#pragma unroll
    for (int i = 0; i < MB; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int c = 0; c < NACC; ++c) acc[i][j][c] = T(0);
    bool rv[MB], cv[4];
#pragma unroll
    for (int i = 0; i < MB; ++i) rv[i] = a0 + wm + i * RB < nx;
#pragma unroll
    for (int j = 0; j < 4; ++j) cv[j] = b0 + wn + j * 8 < ny;

    const int nk = (K + kTK - 1) / kTK;
    fetch(0);
    stash(0);
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < nk) fetch((kt + 1) * kTK);
#pragma unroll
        for (int kk = 0; kk < kTK; kk += 8) {   // m16n8k8: FP64 DMMA or TF32
                T av[2][4], bv[4][2];
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const int r0 = wm + i * 16 + g;
                    av[i][0] = Aat(buf, r0, kk + t4);
                    av[i][1] = Aat(buf, r0 + 8, kk + t4);
                    av[i][2] = Aat(buf, r0, kk + t4 + 4);
                    av[i][3] = Aat(buf, r0 + 8, kk + t4 + 4);
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    bv[j][0] = Bat(buf, kk + t4, wn + j * 8 + g);
                    bv[j][1] = Bat(buf, kk + t4 + 4, wn + j * 8 + g);
                }
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (rv[i] && cv[j]) mma_tile(acc[i][j], av[i], bv[j]);
            }
        if (kt + 1 < nk) stash(buf ^ 1);
        __syncthreads();
    }
    // accumulator element c of block (i, j): row i*RB + g (+8 for c >= 2),
    // column j*8 + 2 t4 + (c & 1)
#pragma unroll
    for (int i = 0; i < MB; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int c = 0; c < NACC; ++c) {
                const int a = a0 + wm + i * RB + g + (c >> 1) * 8;
                const int b = b0 + wn + j * 8 + 2 * t4 + (c & 1);
                if (a >= nx || b >= ny) continue;
                const T v = acc[i][j][c];
                if (STAGE == 1) f.W1[(size_t)b * nx + a] = v;
                else z[(size_t)(b + 1) * m + (a + 1)] = v;
            }
}

// FP32 preconditioner tiles on the 5th-generation tensor cores (tcgen05,
// kind::tf32): C[a + b ldc] = sum_k A[a lda + k] B[b ldb + k] for a 128 x 64
// output tile of one problem, the FP32 accumulator in TMEM.
//   stage 1: A rows = Vx columns (Vx^T), B rows = R^T (r + m + 1, ld m), C = W1
//   stage 3: A rows = VxT columns (Vx),   B rows = W1^T (ld nx),        C = z + m + 1 (ld m)
// All 128 threads stage 32-wide K slices (rounded to TF32) into two shared
// memory buffers in the no-swizzle K-major layout; thread 0 issues four
// 128 x 64 x 8 MMAs per slice and commits them to the buffer's mbarrier,
// which the threads wait on (bounded) before refilling that buffer. The
// epilogue reads the accumulator with tcgen05.ld (warp w: rows 32w .. 32w+31).
constexpr int kUM = 128, kUN = 64, kUK = 32;
constexpr int kALbo = (kUM / 8) * 128 + 16;   // K-chunk stride of an A buffer (+16 B: conflict-free stores)
constexpr int kBLbo = (kUN / 8) * 128 + 16;
constexpr int kAStage = 8 * kALbo, kBStage = 8 * kBLbo;   // 8 chunks of 4 values = 32 k
constexpr int kUmmaSmem = 2 * (kAStage + kBStage) + 64;

template <int STAGE>
__global__ void __launch_bounds__(128) fd_umma_kernel(const FdProb<float> *__restrict__ fps,
                                                      const int4 *__restrict__ tiles, const int *__restrict__ act,
                                                      const float *__restrict__ rb, float *__restrict__ zb,
                                                      int *__restrict__ err)
{
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + 2 * (kAStage + kBStage));
    uint32_t *tbase = reinterpret_cast<uint32_t *>(bars + 2);
    const int4 tl = tiles[blockIdx.x];
    if (!act[tl.x]) return;
    const FdProb<float> &f = fps[tl.x];
    const int nx = f.nx, ny = f.ny, m = f.m, K = nx;
    const int a0 = tl.y * kUM, b0 = tl.z * kUN;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const float *A, *Bm;
    float *C;
    int lda, ldb, ldc;
    if (STAGE == 1) {
        A = f.Vxp; lda = f.ldv; Bm = rb + f.off + m + 1; ldb = m; C = f.W1; ldc = nx;
    } else {
        A = f.VxTp; lda = f.ldv; Bm = f.W1; ldb = nx; C = zb + f.off + m + 1; ldc = m;
    }
    if (STAGE == 1 && tl.y == 0 && tl.z == 0) {   // boundary ring: identity rows of K_fem
        const float *r = rb + f.off;
        float *z = zb + f.off;
        const int n = f.n, nb = 2 * m + 2 * (n - 2);
        for (int u = tid; u < nb; u += 128) {
            int idx;
            if (u < m) idx = u;
            else if (u < 2 * m) idx = (n - 1) * m + (u - m);
            else {
                const int v = u - 2 * m;
                idx = (1 + v / 2) * m + ((v & 1) ? (m - 1) : 0);
            }
            z[idx] = r[idx];
        }
    }
    if (warp == 0) {
        umma::alloc(tbase, kUN);
        umma::relinquish();
    }
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tbase;

    // A (rows padded to lda, a multiple of 4, zero past K): thread t moves the
    // 16-byte K chunk t % 8 of rows t / 8 + 16 i; B: thread (warp, lane) moves
    // k = lane of rows warp + 4 i. Two register sets: slice kt + 2 is loaded
    // while slice kt + 1 goes from the other set into shared memory, so a
    // slice's global loads have a whole iteration to land.
    struct Regs {
        float4 a[kUM / 16];
        float b[kUN / 4];
    };
    Regs R0, R1;
    auto fetch = [&](int kt, Regs &rg) {
        const int k0 = kt * kUK, k = k0 + lane;
        const bool kin = k < K;
        const int kc = k0 + 4 * (tid & 7);
#pragma unroll
        for (int i = 0; i < kUM / 16; ++i) {
            const int a = a0 + (tid >> 3) + 16 * i;
            rg.a[i] = (kc < K && a < nx) ? *reinterpret_cast<const float4 *>(A + (size_t)a * lda + kc)
                                         : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < kUN / 4; ++i) {
            const int b = b0 + warp + 4 * i;
            rg.b[i] = (kin && b < ny) ? Bm[(size_t)b * ldb + k] : 0.0f;
        }
    };
    auto stash = [&](int buf, const Regs &rg) {
        unsigned char *Ab = sm + buf * kAStage, *Bb = sm + 2 * kAStage + buf * kBStage;
        const int ch = lane >> 2, w4 = (lane & 3) * 4;
#pragma unroll
        for (int i = 0; i < kUM / 16; ++i) {
            const int r = (tid >> 3) + 16 * i;
            const float4 v = make_float4(to_operand(rg.a[i].x), to_operand(rg.a[i].y), to_operand(rg.a[i].z),
                                         to_operand(rg.a[i].w));
            *reinterpret_cast<float4 *>(Ab + (tid & 7) * kALbo + (r >> 3) * 128 + (r & 7) * 16) = v;
        }
#pragma unroll
        for (int i = 0; i < kUN / 4; ++i) {
            const int r = warp + 4 * i;
            *reinterpret_cast<float *>(Bb + ch * kBLbo + (r >> 3) * 128 + (r & 7) * 16 + w4) = to_operand(rg.b[i]);
        }
    };
    constexpr uint32_t IDESC = umma::idesc_tf32<kUM, kUN>();
    const int nk = (K + kUK - 1) / kUK;
    fetch(0, R0);
    if (nk > 1) fetch(1, R1);
    stash(0, R0);
    fence_proxy_async_smem();
    __syncthreads();
    bool failed = false;
    int last = -1;   // last slice whose MMAs were issued
    // one iteration: MMAs of slice kt; loads of slice kt + 2 into the set that
    // held slice kt (`cur`); slice kt + 1 from the other set (`nxt`) into the
    // buffer freed by slice kt - 1
    auto step = [&](int kt, Regs &cur, Regs &nxt) -> bool {
        const int buf = kt & 1;
        if (tid == 0) {
            umma::fence_after_sync();
            const unsigned char *Ab = sm + buf * kAStage, *Bb = sm + 2 * kAStage + buf * kBStage;
#pragma unroll
            for (int j = 0; j < kUK / 8; ++j)
                umma::mma_tf32(tmem, umma::smem_desc(Ab + 2 * j * kALbo, kALbo, 128),
                               umma::smem_desc(Bb + 2 * j * kBLbo, kBLbo, 128), IDESC, (kt > 0 || j > 0) ? 1u : 0u);
            umma::commit(&bars[buf]);
        }
        last = kt;
        if (kt + 2 < nk) fetch(kt + 2, cur);
        if (kt + 1 < nk) {
            bool ok = true;
            if (kt >= 1) ok = mbar_wait_bounded(&bars[(kt - 1) & 1], ((kt - 1) >> 1) & 1);   // buffer reused
            if (__syncthreads_or(!ok)) return false;
            stash((kt + 1) & 1, nxt);
            fence_proxy_async_smem();
        }
        __syncthreads();
        return true;
    };
    for (int kt = 0; kt < nk; ++kt) {
        const bool ok = (kt & 1) ? step(kt, R1, R0) : step(kt, R0, R1);
        if (!ok) {
            failed = true;
            break;
        }
    }
    // all MMAs done: the last commit tracks every earlier MMA of thread 0
    const bool ok = mbar_wait_bounded(&bars[last & 1], (last >> 1) & 1);
    failed = __syncthreads_or(failed || !ok);
    if (failed) {
        if (tid == 0) atomicExch(err, 8 /* IGA_ERR_TIMEOUT */);
        mbar_wait_bounded(&bars[last & 1], (last >> 1) & 1);
    } else {
        umma::fence_after_sync();
        const int a = a0 + 32 * warp + lane;
#pragma unroll
        for (int c0 = 0; c0 < kUN; c0 += 16) {
            float v[16];
            umma::ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
            umma::wait_ld();
            if (a < nx) {
#pragma unroll
                for (int c = 0; c < 16; ++c) {
                    const int b = b0 + c0 + c;
                    if (b < ny) C[a + (size_t)b * ldc] = v[c];
                }
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::dealloc(tmem, kUN);
}

// ------------------------------------------------------------ host state
template <typename T>
struct BVec {
    T *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *b = nullptr;
    ApplyParams<T> *prm = nullptr;   // per problem (x, y passed separately)
    FdProb<T> *fd = nullptr;
    T *W1 = nullptr, *Dv = nullptr, *Cf = nullptr;
    std::vector<T *> basis;          // eigenvectors / eigenvalues per distinct 1-D grid
};

struct BGroup {
    int P = 0;
    int W[2] = {0, 0};            // warps per CTA: [0] FP64, [1] FP32
    int4 *items[2] = {nullptr, nullptr};
    int nitems[2] = {0, 0};
};

}  // namespace iga

using namespace iga;

struct iga_batch {
    int count = 0, precision = IGA_FP64, device = 0;
    std::vector<iga_plan *> plans;
    PlanArena arena;   // device memory of the plans' tables and geometry
    std::vector<long long> off;   // count + 1
    long long ntot = 0;
    std::vector<BGroup> groups;
    int nchunks = 0, ntiles = 0, nrows = 0, ntiles_tc = 0;
    int4 *chunks = nullptr, *tiles = nullptr, *tiles_tc = nullptr;
    int *d_err = nullptr;   // device error flag of the tcgen05 tiles (bounded waits)
    int2 *rows = nullptr;
    std::vector<double *> ycoef;     // y pencils of the distinct 1-D grids
    int *c0 = nullptr, *nc = nullptr;
    long long *d_off = nullptr;
    double *partials = nullptr;
    unsigned *counters = nullptr;
    BScal *sc = nullptr;
    BCfg *cfg = nullptr, *h_cfg = nullptr;
    BScal *h_sc = nullptr;
    int *act = nullptr, *act64 = nullptr, *ones = nullptr;
    BVec<double> v64;
    BVec<float> v32;
    bool fd_ready = false;
    cudaStream_t s[3] = {nullptr, nullptr, nullptr}, aux[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_pc = -1;
    bool graph_nested = true;   // mixed: sweeps inside the graph (else host loop over sweep graphs)
    BDev dev() const
    {
        BDev d;
        d.chunks = chunks;
        d.c0 = c0;
        d.nc = nc;
        d.off = d_off;
        d.partials = partials;
        d.counters = counters;
        d.sc = sc;
        d.cfg = cfg;
        return d;
    }
};

#define BT_TRY(call)                                                                 \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));          \
            return e_ == cudaErrorMemoryAllocation ? IGA_ERR_NOMEM : IGA_ERR_CUDA;   \
        }                                                                            \
    } while (0)

namespace {

template <typename T>
int bmalloc(T **p, size_t n)
{
    BT_TRY(cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(n, 1)));
    return IGA_OK;
}

template <typename T>
int bupload(T **p, const std::vector<T> &h)
{
    int st;
    if ((st = bmalloc(p, h.size()))) return st;
    if (!h.empty()) BT_TRY(cudaMemcpy(*p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return IGA_OK;
}

int prec_index(int prec) { return prec == IGA_FP32 ? 1 : 0; }

// Built-in rows per strip when the table has no entry: short strips for
// small patches (more CTAs), longer ones for large patches (fewer seams).
int default_rows(int p, int ney)
{
    int ty = ney <= 64 ? 16 : (ney <= 160 ? 24 : 32);
    return std::max(ty, p);
}

template <int P, typename T>
int set_attr_pt(int W)
{
    constexpr int NST = apply_stages<P, T>();
    const size_t smem = apply_smem_bytes<P, T, 0, NST>(W);
    BT_TRY(cudaFuncSetAttribute(apply_batch_kernel<P, T, NST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return IGA_OK;
}

template <typename T>
int set_attr(int P, int W)
{
    switch (P) {
    case 1: return set_attr_pt<1, T>(W);
    case 2: return set_attr_pt<2, T>(W);
    case 3: return set_attr_pt<3, T>(W);
    case 4: return set_attr_pt<4, T>(W);
    case 5: return set_attr_pt<5, T>(W);
    default: return IGA_ERR_UNSUPPORTED;
    }
}

template <int P, typename T>
void launch_group_pt(const iga_batch *B, const BGroup &G, const ApplyParams<T> *prm, const int *act, const T *x, T *y,
                     cudaStream_t s)
{
    constexpr int NST = apply_stages<P, T>();
    const int pi = sizeof(T) == 8 ? 0 : 1;
    const int W = G.W[pi];
    if (G.nitems[pi] == 0) return;
    const size_t smem = apply_smem_bytes<P, T, 0, NST>(W);
    apply_batch_kernel<P, T, NST><<<G.nitems[pi], dim3(32, W), smem, s>>>(prm, G.items[pi], act, B->d_off, x, y);
}

template <typename T>
void launch_group(const iga_batch *B, const BGroup &G, const ApplyParams<T> *prm, const int *act, const T *x, T *y,
                  cudaStream_t s)
{
    switch (G.P) {
    case 1: launch_group_pt<1, T>(B, G, prm, act, x, y, s); break;
    case 2: launch_group_pt<2, T>(B, G, prm, act, x, y, s); break;
    case 3: launch_group_pt<3, T>(B, G, prm, act, x, y, s); break;
    case 4: launch_group_pt<4, T>(B, G, prm, act, x, y, s); break;
    case 5: launch_group_pt<5, T>(B, G, prm, act, x, y, s); break;
    default: break;
    }
}

template <typename T>
BVec<T> &vecs(iga_batch *B);
template <>
BVec<double> &vecs<double>(iga_batch *B) { return B->v64; }
template <>
BVec<float> &vecs<float>(iga_batch *B) { return B->v32; }

// y = K x for the problems with act set. The first group runs on s, the
// others on aux (forked from and joined back into s), then the seams.
template <typename T>
int batch_apply(iga_batch *B, const T *x, T *y, const int *act, cudaStream_t s, cudaStream_t aux)
{
    const ApplyParams<T> *prm = vecs<T>(B).prm;
    const bool fork = B->groups.size() > 1 && aux;
    if (fork) {
        BT_TRY(cudaEventRecord(B->fork, s));
        BT_TRY(cudaStreamWaitEvent(aux, B->fork, 0));
    }
    for (size_t gi = 0; gi < B->groups.size(); ++gi)
        launch_group<T>(B, B->groups[gi], prm, act, x, y, (fork && gi > 0) ? aux : s);
    if (fork) {
        BT_TRY(cudaEventRecord(B->join, aux));
        BT_TRY(cudaStreamWaitEvent(s, B->join, 0));
    }
    seam_fixup_batch_kernel<T><<<dim3(16, B->count), 256, 0, s>>>(prm, act, B->d_off, x, y);
    BT_TRY(cudaGetLastError());
    return IGA_OK;
}

template <typename T>
int batch_pc(iga_batch *B, int pc, const T *r, T *z, const int *act, cudaStream_t s)
{
    const BDev d = B->dev();
    if (pc == IGA_PC_NONE) {
        bk_copy<T><<<B->nchunks, kBT, 0, s>>>(d, act, r, z);
    } else {
        const FdProb<T> *fd = vecs<T>(B).fd;
        if constexpr (sizeof(T) == 4) {   // TF32 tiles on tcgen05
            fd_umma_kernel<1><<<B->ntiles_tc, 128, kUmmaSmem, s>>>(fd, B->tiles_tc, act, r, z, B->d_err);
            fd_rows_kernel<T><<<B->nrows, dim3(32, kRowSeg), 0, s>>>(fd, B->rows, act);
            fd_umma_kernel<3><<<B->ntiles_tc, 128, kUmmaSmem, s>>>(fd, B->tiles_tc, act, r, z, B->d_err);
        } else {                          // FP64 tiles on DMMA
            fd_gemm_kernel<T, 1><<<B->ntiles, 128, 0, s>>>(fd, B->tiles, act, r, z);
            fd_rows_kernel<T><<<B->nrows, dim3(32, kRowSeg), 0, s>>>(fd, B->rows, act);
            fd_gemm_kernel<T, 3><<<B->ntiles, 128, 0, s>>>(fd, B->tiles, act, r, z);
        }
    }
    BT_TRY(cudaGetLastError());
    return IGA_OK;
}

// z = M^-1 r, rz, p = z for the active problems.
template <typename T>
int pcg_start(iga_batch *B, int pc, cudaStream_t s)
{
    BVec<T> &v = vecs<T>(B);
    int st;
    if ((st = batch_pc<T>(B, pc, v.r, v.z, B->act, s))) return st;
    bk_rz_p<T><<<B->nchunks, kBT, 0, s>>>(B->dev(), B->act, v.r, v.z, v.p);
    BT_TRY(cudaGetLastError());
    return IGA_OK;
}

// One flexible PCG iteration of every active problem, then the loop condition.
template <typename T>
int pcg_iteration(iga_batch *B, int pc, cudaStream_t s, cudaStream_t aux, cudaGraphConditionalHandle h)
{
    BVec<T> &v = vecs<T>(B);
    const BDev d = B->dev();
    int st;
    if ((st = batch_apply<T>(B, v.p, v.q, B->act, s, aux))) return st;
    bk_pq<T><<<B->nchunks, kBT, 0, s>>>(d, B->act, v.p, v.q);
    bk_xr<T><<<B->nchunks, kBT, 0, s>>>(d, B->act, v.x, v.r, v.p, v.q, v.z);
    if ((st = batch_pc<T>(B, pc, v.r, v.z, B->act, s))) return st;
    bk_beta<T><<<B->nchunks, kBT, 0, s>>>(d, B->act, v.r, v.z);
    bk_p<T><<<B->nchunks, kBT, 0, s>>>(d, B->act, v.p, v.z);
    bk_cond<<<1, kBT, 0, s>>>(B->act, B->count, h);
    BT_TRY(cudaGetLastError());
    return IGA_OK;
}

// Adds a conditional WHILE node at the current capture position of s and
// starts capturing its body on bs. The condition is set explicitly by a
// kernel just before the node (any of flags[0..n) set): a handle's default
// value is only applied when the top-level graph is launched, not when an
// enclosing loop body runs again.
int begin_while(cudaStream_t s, cudaStream_t bs, const int *flags, int n, cudaGraphNode_t *node,
                cudaGraphConditionalHandle *h)
{
    cudaStreamCaptureStatus cs;
    cudaGraph_t g;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    BT_TRY(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) {
        set_error("begin_while: stream is not capturing");
        return IGA_ERR_CUDA;
    }
    BT_TRY(cudaGraphConditionalHandleCreate(h, g, 0, 0));
    bk_cond<<<1, kBT, 0, s>>>(flags, n, *h);
    BT_TRY(cudaGetLastError());
    BT_TRY(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = *h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    BT_TRY(cudaGraphAddNode(node, g, deps, nd, &np));
    BT_TRY(cudaStreamUpdateCaptureDependencies(s, node, 1, cudaStreamSetCaptureDependencies));
    BT_TRY(cudaStreamBeginCaptureToGraph(bs, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeRelaxed));
    return IGA_OK;
}

int end_while(cudaStream_t bs)
{
    cudaGraph_t body = nullptr;
    BT_TRY(cudaStreamEndCapture(bs, &body));
    return IGA_OK;
}

// One mixed-precision refinement sweep on stream s (FP32 PCG loop on s2).
int sweep_body(iga_batch *B, int pc, cudaStream_t s, cudaStream_t aux, cudaStream_t s2, cudaStream_t aux2)
{
    const BDev d = B->dev();
    int st;
    bk_sweep_init<<<B->nchunks, kBT, 0, s>>>(d, B->act64, B->act, B->v64.r, B->v32.r, B->v32.x);
    if ((st = pcg_start<float>(B, pc, s))) return st;
    cudaGraphNode_t node;
    cudaGraphConditionalHandle h;
    if ((st = begin_while(s, s2, B->act, B->count, &node, &h))) return st;
    st = pcg_iteration<float>(B, pc, s2, aux2, h);
    const int st2 = end_while(s2);
    if (st || st2) return st ? st : st2;
    bk_refine<<<B->nchunks, kBT, 0, s>>>(d, B->act64, B->v64.x, B->v32.x);
    if ((st = batch_apply<double>(B, B->v64.x, B->v64.q, B->act64, s, aux))) return st;
    bk_res64<<<B->nchunks, kBT, 0, s>>>(d, B->act64, B->v64.b, B->v64.q, B->v64.r, 1);
    BT_TRY(cudaGetLastError());
    return IGA_OK;
}

int instantiate(cudaGraph_t g, cudaGraphExec_t *out)
{
    cudaGraphInstantiateParams ip = {};
    const cudaError_t e = cudaGraphInstantiateWithParams(out, g, &ip);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        set_error(std::string("batch graph instantiation: ") + cudaGetErrorString(e) + " (result " +
                  std::to_string((int)ip.result_out) + ")");
        return IGA_ERR_UNSUPPORTED;
    }
    return IGA_OK;
}

// Captures the solve graph for preconditioner pc.
//   FP64:  K x; r = b - Kx; z = M^-1 r; p = z; WHILE { PCG iteration }; K x; true residual.
//   MIXED: K x; true residual; WHILE { sweep: r32 = r/||r||; FP32 PCG start;
//          WHILE { FP32 PCG iteration }; x += ||r|| d; K x; true residual }.
// nested = false (MIXED only): the graph is one sweep, driven by a host loop.
int build_graph(iga_batch *B, int pc, bool nested)
{
    if (B->graph) {
        cudaGraphExecDestroy(B->graph);
        B->graph = nullptr;
    }
    cudaStream_t s = B->s[0], a0 = B->aux[0];
    const BDev d = B->dev();
    BT_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    int st = IGA_OK;
    cudaGraphNode_t node;
    cudaGraphConditionalHandle h;
    if (B->precision == IGA_FP64) {
        st = batch_apply<double>(B, B->v64.x, B->v64.q, B->act64, s, a0);
        if (!st) {
            bk_init64<<<B->nchunks, kBT, 0, s>>>(d, B->act64, B->act, B->v64.b, B->v64.q, B->v64.r);
            st = pcg_start<double>(B, pc, s);
        }
        if (!st) st = begin_while(s, B->s[1], B->act, B->count, &node, &h);
        if (!st) {
            st = pcg_iteration<double>(B, pc, B->s[1], B->aux[1], h);
            const int st2 = end_while(B->s[1]);
            if (!st) st = st2;
        }
        if (!st) st = batch_apply<double>(B, B->v64.x, B->v64.q, B->act64, s, a0);
        if (!st) bk_res64<<<B->nchunks, kBT, 0, s>>>(d, B->act64, B->v64.b, B->v64.q, B->v64.r, 0);
    } else if (nested) {
        st = batch_apply<double>(B, B->v64.x, B->v64.q, B->act64, s, a0);
        if (!st) {
            bk_res64<<<B->nchunks, kBT, 0, s>>>(d, B->act64, B->v64.b, B->v64.q, B->v64.r, 2);
            st = begin_while(s, B->s[1], B->act64, B->count, &node, &h);
        }
        if (!st) {
            st = sweep_body(B, pc, B->s[1], B->aux[1], B->s[2], B->aux[2]);
            if (!st) bk_cond<<<1, kBT, 0, B->s[1]>>>(B->act64, B->count, h);
            const int st2 = end_while(B->s[1]);
            if (!st) st = st2;
        }
    } else {
        st = sweep_body(B, pc, s, a0, B->s[1], B->aux[1]);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (st || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (!st) set_error(std::string("batch graph capture: ") + cudaGetErrorString(ce));
        return st ? st : IGA_ERR_CUDA;
    }
    st = instantiate(g, &B->graph);
    cudaGraphDestroy(g);
    if (!st) B->graph_pc = pc;
    return st;
}

// LDL^T factors of the y systems lx[a] My + Ky, one thread per (problem =
// blockIdx.y, x mode a): Dv_b = 1 / d_b and Cf_b = e_b / d_b along y (layout
// [b][a], ld nx), from the FP64 eigenvalues; f32 (optional) gets FP32 copies.
__global__ void fd_ldl_kernel(const FdProb<double> *__restrict__ f64, const FdProb<float> *__restrict__ f32)
{
    const int i = blockIdx.y;
    const FdProb<double> &f = f64[i];
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= f.nx) return;
    const int nx = f.nx, ny = f.ny;
    const double *Kd = f.yc, *Ko = Kd + ny, *Md = Kd + 2 * ny, *Mo = Kd + 3 * ny;
    double *Dv = const_cast<double *>(f.Dv), *Cf = const_cast<double *>(f.Cf);
    float *Dv32 = f32 ? const_cast<float *>(f32[i].Dv) : nullptr, *Cf32 = f32 ? const_cast<float *>(f32[i].Cf) : nullptr;
    const double lam = f.lx[a];
    double cprev = 0.0, eprev = 0.0;
    for (int b = 0; b < ny; ++b) {
        const double den = lam * Md[b] + Kd[b] - eprev * cprev;
        const double e = b + 1 < ny ? lam * Mo[b] + Ko[b] : 0.0;
        const double dv = 1.0 / den, cf = e / den;
        const size_t at = (size_t)b * nx + a;
        Dv[at] = dv;
        Cf[at] = cf;
        if (Dv32) {
            Dv32[at] = (float)dv;
            Cf32[at] = (float)cf;
        }
        cprev = cf;
        eprev = e;
    }
}

// One distinct grid's eigenpairs on the device: mode a < fe from the even
// half (half vectors at U + ue, hn_e long), the others from the odd half
// (U + uo, hn_o long; uo < 0: a pencil that was not split, fe = n), scaled
// by sc; mirrored entries v[n-1-i] = +-u[i]; lam: the n eigenvalues in the
// same mode order. Outputs: V (component i of mode a at a n + i) and its
// transpose VT, FP64 and, when V32 is set, FP32 with 16-byte padded copies
// (row length ldp).
struct BasisDev {
    int n, fe, hn_e, hn_o, ldp;
    long long ue, uo, lo;
    double sc;
    double *V, *VT, *L;
    float *V32, *VT32, *Vp32, *VTp32, *L32;
};

__global__ void basis_build_kernel(const BasisDev *__restrict__ bs, const double *__restrict__ U,
                                   const double *__restrict__ lam)
{
    const BasisDev b = bs[blockIdx.y];
    const int n = b.n;
    const long long nn = (long long)n * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn; t += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(t / n), i = (int)(t - (long long)a * n);
        const bool even = a < b.fe;
        const int hn = even ? b.hn_e : b.hn_o;
        const double *u = U + (even ? b.ue + (long long)a * hn : b.uo + (long long)(a - b.fe) * hn);
        double v;
        if (b.uo < 0 && even) {
            v = u[i];
        } else if (i < hn) {
            v = b.sc * u[i];
        } else {
            const int im = n - 1 - i;
            v = (im < hn && im != i) ? (even ? b.sc : -b.sc) * u[im] : 0.0;
        }
        b.V[t] = v;
        b.VT[(long long)i * n + a] = v;
        if (b.V32) {
            b.V32[t] = (float)v;
            b.VT32[(long long)i * n + a] = (float)v;
            b.Vp32[(long long)a * b.ldp + i] = (float)v;
            b.VTp32[(long long)i * b.ldp + a] = (float)v;
        }
        if (i == 0) {
            b.L[a] = lam[b.lo + a];
            if (b.L32) b.L32[a] = (float)lam[b.lo + a];
        }
    }
}

__global__ void gather_flags_kernel(int *const *__restrict__ flags, int n, int *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = *flags[i];
}

// Eigenpairs of the FEM pencils of every distinct 1-D grid, uploaded in T.
int setup_fd(iga_batch *B)
{
    if (B->fd_ready) return IGA_OK;
    struct Basis {
        int n = 0;   // free nodes of the grid
    };
    std::map<std::vector<double>, int> index;
    std::vector<std::vector<double>> grids;
    std::vector<int> bx(B->count), by(B->count);
    // Net lengths summed over different numbers of segments differ in the last
    // bits for patches of the same extent; rounded to 14 significant digits,
    // equal grids are found equal and share one eigen-decomposition (the 256
    // benchmark problems have 30 distinct grids).
    auto snap = [](double L) {
        if (!(L > 0.0) || !std::isfinite(L)) return L;
        const double e = std::pow(10.0, std::floor(std::log10(L)) - 13);
        return std::round(L / e) * e;
    };
    // net lengths of every problem (the heavy part of the grid index), threaded
    const unsigned nthr = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), 16u));
    std::vector<double> hLx(B->count), hLy(B->count);
    {
        std::vector<std::thread> th;
        for (unsigned w = 0; w < nthr; ++w)
            th.emplace_back([&, w]() {
                for (int i = (int)w; i < B->count; i += (int)nthr) net_lengths(B->plans[i]->patch, hLx[i], hLy[i]);
            });
        for (auto &t : th) t.join();
    }
    for (int i = 0; i < B->count; ++i) {
        const iga_plan *pl = B->plans[i];
        const double Lx = snap(hLx[i]), Ly = snap(hLy[i]);
        for (int dir = 0; dir < 2; ++dir) {
            std::vector<double> g = dir == 0 ? fem_nodes_1d(pl->p, pl->nex, Lx) : fem_nodes_1d(pl->p, pl->ney, Ly);
            auto it = index.find(g);
            int id;
            if (it == index.end()) {
                id = (int)grids.size();
                index.emplace(g, id);
                grids.push_back(std::move(g));
            } else {
                id = it->second;
            }
            (dir == 0 ? bx : by)[i] = id;
        }
    }
    // Eigenpairs of every distinct grid's pencil: split by parity (the FEM
    // nodes are symmetric about the middle: two half-size pencils), the
    // eigenpairs of all of them on the device (one thread per eigenpair),
    // expanded there to full vectors (even modes first, then odd ones).
    std::vector<Basis> bases(grids.size());
    std::vector<std::vector<double>> pencils(grids.size());   // Kd | Ko | Md | Mo of the free nodes
    struct Half {
        int grid, parity;   // parity -1: the whole pencil (not centrosymmetric)
        std::vector<double> kd, ko, md, mo;
    };
    std::vector<Half> halves;
    for (size_t k = 0; k < grids.size(); ++k) {
        std::vector<double> Kd, Ko, Md, Mo;
        interior_pencil(grids[k], Kd, Ko, Md, Mo);
        const int n = (int)Kd.size();
        bases[k].n = n;
        for (const std::vector<double> *v : {&Kd, &Ko, &Md, &Mo}) pencils[k].insert(pencils[k].end(), v->begin(), v->end());
        if (n == 0) continue;
        if (pencil_centrosymmetric(n, Kd.data(), Ko.data(), Md.data(), Mo.data())) {
            for (int parity = 0; parity < 2; ++parity) {
                Half h;
                h.grid = (int)k;
                h.parity = parity;
                pencil_fold(n, Kd.data(), Ko.data(), Md.data(), Mo.data(), parity, h.kd, h.ko, h.md, h.mo);
                if (!h.kd.empty()) halves.push_back(std::move(h));
            }
        } else {
            halves.push_back(Half{(int)k, -1, Kd, Ko, Md, Mo});
        }
    }
    std::vector<PencilRef> refs;
    for (const Half &h : halves) refs.push_back(PencilRef{(int)h.kd.size(), h.kd.data(), h.ko.data(), h.md.data(), h.mo.data()});
    std::vector<std::vector<double>> hlam;
    double *dU = nullptr;            // the half vectors, left on the device
    std::vector<long long> voff;     // offset of each half's block in dU
    {
        const int st = pencil_eig_device(B->device, refs, hlam, nullptr, &dU, &voff);
        if (st) return st;
    }
    // the half vectors stay on the device where they were computed (plus the
    // eigenvalues, uploaded in mode order); the device expands them into every
    // grid's full eigenvector matrix, its transpose and (MIXED) the FP32
    // copies, in one buffer per precision
    std::vector<long long> lo_of(grids.size(), -1), ue_of(grids.size(), -1), uo_of(grids.size(), -1);
    std::vector<int> hne(grids.size(), 0), hno(grids.size(), 0), fe_of(grids.size(), 0);
    std::vector<char> split(grids.size(), 0);
    std::vector<double> hL(0);
    for (size_t r = 0; r < halves.size(); ++r) {
        const Half &h = halves[r];
        const int hn = (int)h.kd.size();
        if (h.parity <= 0) {   // even half or whole pencil: first in mode order
            ue_of[h.grid] = voff[r];
            hne[h.grid] = hn;
            fe_of[h.grid] = hn;
            split[h.grid] = h.parity == 0;
        } else {
            uo_of[h.grid] = voff[r];
            hno[h.grid] = hn;
        }
    }
    // eigenvalues in mode order per grid: even half, then odd half
    for (size_t k = 0; k < grids.size(); ++k) {
        lo_of[k] = (long long)hL.size();
        for (int parity = 0; parity < 2; ++parity)
            for (size_t r = 0; r < halves.size(); ++r)
                if (halves[r].grid == (int)k && (halves[r].parity == parity || (parity == 0 && halves[r].parity < 0)))
                    hL.insert(hL.end(), hlam[r].begin(), hlam[r].end());
    }
    double *dL = nullptr;
    {
        int st;
        if ((st = bupload(&dL, hL))) {
            cudaFree(dU);
            return st;
        }
    }
    const bool mixed = B->precision == IGA_MIXED;
    // every sub-array starts on a 16-byte boundary (the FP32 padded copies
    // move as 16-byte words)
    auto al4 = [](size_t x) { return (x + 3) / 4 * 4; };
    size_t tot64 = 0, tot32 = 0;
    for (const Basis &bb : bases) {
        const size_t n = (size_t)bb.n, ldp = al4(n);
        tot64 += 2 * al4(n * n) + al4(n);
        if (mixed) tot32 += 2 * al4(n * n) + 2 * n * ldp + al4(n);
    }
    double *b64 = nullptr;
    float *b32 = nullptr;
    {
        int st;
        if ((st = bmalloc(&b64, tot64))) return st;
        B->v64.basis.push_back(b64);
        if (mixed) {
            if ((st = bmalloc(&b32, tot32))) return st;
            BT_TRY(cudaMemset(b32, 0, sizeof(float) * tot32));   // the padding columns
            B->v32.basis.push_back(b32);
        }
    }
    std::vector<BasisDev> bd(grids.size());
    std::vector<double *> V64(grids.size()), VT64(grids.size()), L64(grids.size());
    std::vector<float *> V32(grids.size(), nullptr), VT32(grids.size(), nullptr), Vp32(grids.size(), nullptr),
        VTp32(grids.size(), nullptr), L32(grids.size(), nullptr);
    {
        size_t o64 = 0, o32 = 0;
        for (size_t k = 0; k < grids.size(); ++k) {
            const int n = bases[k].n;
            const size_t nn = (size_t)n * n, ldp = al4((size_t)n);
            V64[k] = b64 + o64;
            VT64[k] = V64[k] + al4(nn);
            L64[k] = VT64[k] + al4(nn);
            o64 += 2 * al4(nn) + al4(n);
            if (mixed) {
                V32[k] = b32 + o32;
                VT32[k] = V32[k] + al4(nn);
                Vp32[k] = VT32[k] + al4(nn);
                VTp32[k] = Vp32[k] + (size_t)n * ldp;
                L32[k] = VTp32[k] + (size_t)n * ldp;
                o32 += 2 * al4(nn) + 2 * (size_t)n * ldp + al4(n);
            }
            BasisDev &d = bd[k];
            d.n = n;
            d.fe = split[k] ? fe_of[k] : n;
            d.hn_e = hne[k];
            d.hn_o = hno[k];
            d.ldp = (int)ldp;
            d.ue = ue_of[k] < 0 ? 0 : ue_of[k];
            d.uo = split[k] ? uo_of[k] : -1;
            d.lo = lo_of[k];
            d.sc = split[k] ? 1.0 / std::sqrt(2.0) : 1.0;
            d.V = V64[k];
            d.VT = VT64[k];
            d.L = L64[k];
            d.V32 = V32[k];
            d.VT32 = VT32[k];
            d.Vp32 = Vp32[k];
            d.VTp32 = VTp32[k];
            d.L32 = L32[k];
        }
        BasisDev *dbd = nullptr;
        int st;
        if ((st = bupload(&dbd, bd))) return st;
        int nmax = 1;
        for (const Basis &bb : bases) nmax = std::max(nmax, bb.n);
        const long long nn = (long long)nmax * nmax;
        const dim3 grid((unsigned)std::max(1LL, std::min((nn + 255) / 256, 256LL)), (unsigned)grids.size());
        basis_build_kernel<<<grid, 256>>>(dbd, dU, dL);
        const cudaError_t ke = cudaGetLastError();
        cudaDeviceSynchronize();
        cudaFree(dbd);
        cudaFree(dU);
        cudaFree(dL);
        if (ke != cudaSuccess) {
            set_error(std::string("basis_build_kernel: ") + cudaGetErrorString(ke));
            return IGA_ERR_CUDA;
        }
    }
    // y pencils of the grids (double, shared by both precisions)
    for (size_t k = 0; k < grids.size(); ++k) {
        double *d = nullptr;
        int st;
        if ((st = bupload(&d, pencils[k]))) return st;
        B->ycoef.push_back(d);
    }
    auto upload_prec = [&](auto tag) -> int {
        using T = decltype(tag);
        BVec<T> &v = vecs<T>(B);
        const bool f64 = sizeof(T) == 8;
        auto pick = [&](double *d, float *f) { return f64 ? (T *)(void *)d : (T *)(void *)f; };
        std::vector<FdProb<T>> fp(B->count);
        size_t wtot = 0;
        for (int i = 0; i < B->count; ++i) wtot += (size_t)(B->plans[i]->m - 2) * (B->plans[i]->n - 2);
        int st;
        if ((st = bmalloc(&v.W1, wtot)) || (st = bmalloc(&v.Dv, wtot)) || (st = bmalloc(&v.Cf, wtot))) return st;
        size_t wo = 0;
        for (int i = 0; i < B->count; ++i) {
            const iga_plan *pl = B->plans[i];
            FdProb<T> &f = fp[i];
            f.Vx = pick(V64[bx[i]], V32[bx[i]]);
            f.VxT = pick(VT64[bx[i]], VT32[bx[i]]);
            f.Vxp = f64 ? nullptr : pick(nullptr, Vp32[bx[i]]);
            f.VxTp = f64 ? nullptr : pick(nullptr, VTp32[bx[i]]);
            f.ldv = (bases[bx[i]].n + 3) / 4 * 4;
            f.lx = pick(L64[bx[i]], L32[bx[i]]);
            f.yc = B->ycoef[by[i]];
            f.W1 = v.W1 + wo;
            f.Dv = v.Dv + wo;
            f.Cf = v.Cf + wo;
            f.off = B->off[i];
            f.m = pl->m;
            f.n = pl->n;
            f.nx = pl->m - 2;
            f.ny = pl->n - 2;
            wo += (size_t)f.nx * f.ny;
        }
        return bupload(&v.fd, fp);
    };
    int st;
    if ((st = upload_prec(double{}))) return st;
    if (B->precision == IGA_MIXED && (st = upload_prec(float{}))) return st;
    // LDL^T factors of lx[a] My + Ky for every problem and x mode, on the
    // device from the FP64 eigenvalues (both precisions' copies)
    {
        int maxnx = 1;
        for (int i = 0; i < B->count; ++i) maxnx = std::max(maxnx, B->plans[i]->m - 2);
        const dim3 grid((unsigned)((maxnx + 127) / 128), (unsigned)B->count);
        fd_ldl_kernel<<<grid, 128>>>(B->v64.fd, B->precision == IGA_MIXED ? B->v32.fd : nullptr);
        BT_TRY(cudaGetLastError());
    }
    // GEMM tiles, largest contraction first
    std::vector<std::pair<int, int4>> tl;
    for (int i = 0; i < B->count; ++i) {
        const int nx = B->plans[i]->m - 2, ny = B->plans[i]->n - 2;
        if (nx <= 0 || ny <= 0) continue;
        for (int a = 0; a < (nx + kTile - 1) / kTile; ++a)
            for (int b = 0; b < (ny + kTile - 1) / kTile; ++b) tl.push_back({nx + ny, make_int4(i, a, b, 0)});
    }
    std::stable_sort(tl.begin(), tl.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
    std::vector<int4> tiles;
    for (auto &t : tl) tiles.push_back(t.second);
    if (tiles.empty()) tiles.push_back(make_int4(0, 0, 0, 0));   // never active: nx or ny is 0
    B->ntiles = (int)tl.size();
    // row-solve blocks: (problem, first x mode) for every 32 modes
    std::vector<int2> rows;
    for (int i = 0; i < B->count; ++i) {
        const int nx = B->plans[i]->m - 2, ny = B->plans[i]->n - 2;
        if (nx <= 0 || ny <= 0) continue;
        for (int a0 = 0; a0 < nx; a0 += 32) rows.push_back(make_int2(i, a0));
    }
    B->nrows = (int)rows.size();
    if (rows.empty()) rows.push_back(make_int2(0, 0));
    if ((st = bupload(&B->rows, rows))) return st;
    // 128 x 64 tiles of the tcgen05 path (FP32)
    if (B->precision == IGA_MIXED) {
        std::vector<std::pair<int, int4>> tt;
        for (int i = 0; i < B->count; ++i) {
            const int nx = B->plans[i]->m - 2, ny = B->plans[i]->n - 2;
            if (nx <= 0 || ny <= 0) continue;
            for (int a = 0; a < (nx + kUM - 1) / kUM; ++a)
                for (int b = 0; b < (ny + kUN - 1) / kUN; ++b) tt.push_back({nx, make_int4(i, a, b, 0)});
        }
        std::stable_sort(tt.begin(), tt.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
        std::vector<int4> tc;
        for (auto &t : tt) tc.push_back(t.second);
        B->ntiles_tc = (int)tc.size();
        if (tc.empty()) tc.push_back(make_int4(0, 0, 0, 0));
        if ((st = bupload(&B->tiles_tc, tc))) return st;
        BT_TRY(cudaFuncSetAttribute(fd_umma_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kUmmaSmem));
        BT_TRY(cudaFuncSetAttribute(fd_umma_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kUmmaSmem));
    }
    if ((st = bupload(&B->tiles, tiles))) return st;
    B->fd_ready = true;
    return IGA_OK;
}

template <typename T>
int setup_params(iga_batch *B)
{
    std::vector<ApplyParams<T>> prm(B->count);
    for (int i = 0; i < B->count; ++i) {
        const iga_plan *pl = B->plans[i];
        const OperatorData &op = sizeof(T) == 8 ? pl->op64 : pl->op32;
        ApplyParams<T> &a = prm[i];
        a.x = nullptr;
        a.y = nullptr;
        a.G = (const T *)op.G;
        a.tabX = (const T *)op.tabX;
        a.tabY = (const T *)op.tabY;
        a.CP = (const T *)op.CP;
        a.wq = (const T *)op.wq;
        a.kappa = nullptr;
        a.frame = (T *)op.frame;
        a.g = op.grid;
        a.sign = T(1);
        a.bc = IGA_BC_IDENTITY;
        a.err = pl->d_err;
    }
    return bupload(&vecs<T>(B).prm, prm);
}

// Work items of every degree group for warps-per-CTA W (per precision).
int setup_items(iga_batch *B, int pi)
{
    for (BGroup &G : B->groups) {
        if (G.items[pi]) {
            cudaFree(G.items[pi]);
            G.items[pi] = nullptr;
        }
        const int W = G.W[pi];
        // the kernels deal strips to warps unless their tables are in shared
        // memory (apply_txshared: FP64 p >= 4 with precomputed G)
        const bool flat = pi == 1 || G.P <= 3;
        std::vector<int4> items;
        for (int i = 0; i < B->count; ++i) {
            const iga_plan *pl = B->plans[i];
            if (pl->p != G.P) continue;
            const StripGrid &g = (pi ? pl->op32 : pl->op64).grid;
            if (flat) {   // one item per strip (warp)
                for (int gx = 0; gx < g.NSX; ++gx)
                    for (int gy = 0; gy < g.NSY; ++gy) items.push_back(make_int4(i, gx, gy, 0));
            } else {      // one item per CTA: W strips of a column
                for (int gyb = 0; gyb < (g.NSY + W - 1) / W; ++gyb)
                    for (int gx = 0; gx < g.NSX; ++gx) items.push_back(make_int4(i, gx, gyb, 0));
            }
        }
        if (flat)
            while (items.size() % W) items.push_back(make_int4(-1, 0, 0, 0));   // whole CTAs
        G.nitems[pi] = (int)(flat ? items.size() / W : items.size());         // CTAs
        int st;
        if ((st = bupload(&G.items[pi], items))) return st;
        const int prec = pi ? IGA_FP32 : IGA_FP64;
        if ((st = pi ? set_attr<float>(G.P, warps_for(G.P, prec, 0)) : set_attr<double>(G.P, warps_for(G.P, prec, 0))))
            return st;
    }
    return IGA_OK;
}

void free_vecs_common(BVec<double> &v)
{
    for (void *p : {(void *)v.x, (void *)v.r, (void *)v.z, (void *)v.p, (void *)v.q, (void *)v.b, (void *)v.prm,
                    (void *)v.fd, (void *)v.W1, (void *)v.Dv, (void *)v.Cf})
        if (p) cudaFree(p);
    for (double *p : v.basis) cudaFree(p);
}
void free_vecs_common(BVec<float> &v)
{
    for (void *p : {(void *)v.x, (void *)v.r, (void *)v.z, (void *)v.p, (void *)v.q, (void *)v.b, (void *)v.prm,
                    (void *)v.fd, (void *)v.W1, (void *)v.Dv, (void *)v.Cf})
        if (p) cudaFree(p);
    for (float *p : v.basis) cudaFree(p);
}

// Batch without solver data when solver = false (the autotuner's timing runs).
// rows[i] > 0 overrides problem i's rows per strip; warps[p] > 0 the warps of degree p.
int create_batch(const iga_mesh_desc *meshes, int count, int precision, int device, const TuneTable &tt,
                 const int *rows, const int *warps_over, bool solver, iga_batch **out)
{
    *out = nullptr;
    if (!meshes || count <= 0 || (precision != IGA_FP64 && precision != IGA_MIXED)) {
        set_error("iga_batch_create: need count > 0 meshes and precision IGA_FP64 or IGA_MIXED");
        return IGA_ERR_ARG;
    }
    iga_batch *B = new iga_batch();
    B->count = count;
    B->precision = precision;
    B->device = device;
    auto fail = [&](int st) {
        iga_batch_destroy(B);
        return st;
    };
    BT_TRY(cudaSetDevice(device));
    B->off.assign(count + 1, 0);
    const int tprec = precision == IGA_MIXED ? IGA_MIXED : IGA_FP64;
    for (int i = 0; i < count; ++i) {
        if (meshes[i].nElemX + meshes[i].p < 3 || meshes[i].nElemY + meshes[i].q < 3) {
            set_error("iga_batch_create: every patch needs an interior control point in each direction");
            return fail(IGA_ERR_UNSUPPORTED);
        }
        if (meshes[i].nElemY + meshes[i].q - 2 > kRowSeg * kRowLen) {
            set_error("iga_batch_create: problem " + std::to_string(i) + " has more than " +
                      std::to_string(kRowSeg * kRowLen) + " free control points in y (batches hold small patches)");
            return fail(IGA_ERR_UNSUPPORTED);
        }
        if (meshes[i].kappa) {
            set_error("iga_batch_create: coefficient kappa is not supported in batches");
            return fail(IGA_ERR_UNSUPPORTED);
        }
    }
    // The plans are built by host threads (mesh tables, strip layout: host
    // work), all from the batch's arena in deferred mode: their host data is
    // staged and sent in one copy after the last plan, their geometry set-up
    // launched after that.
    B->arena.defer = true;
    std::vector<iga_plan *> built(count, nullptr);
    std::vector<int> status(count, IGA_OK);
    std::vector<std::string> message(count);
    {
        // host threads building plans: one core is left to the arena's copy thread
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const unsigned nthr = hw > 2 ? std::min(hw - 1, 16u) : 1u;
        std::atomic<int> next{0};
        auto work = [&]() {
            cudaSetDevice(device);
            plan_arena() = &B->arena;
            for (int i; (i = next.fetch_add(1)) < count;) {
                iga_opts o;
                iga_opts_default(&o);
                o.precision = precision;
                o.geometry = IGA_GEOM_PRECOMPUTED;
                o.sign = IGA_SIGN_SPD;
                o.bc = IGA_BC_IDENTITY;
                o.device = device;
                int ty = rows && rows[i] > 0 ? rows[i] : tune_rows(tt, meshes[i].p, tprec, meshes[i].nElemY);
                if (ty <= 0) ty = default_rows(meshes[i].p, meshes[i].nElemY);
                o.rows_per_strip = std::max(ty, std::max(1, meshes[i].p));
                status[i] = iga_plan_create(&meshes[i], &o, &built[i]);
                if (status[i]) message[i] = last_error();
            }
            plan_arena() = nullptr;
        };
        std::vector<std::thread> th;
        for (unsigned w = 1; w < nthr; ++w) th.emplace_back(work);
        work();
        for (auto &t : th) t.join();
    }
    for (int i = 0; i < count; ++i)
        if (built[i]) B->plans.push_back(built[i]);
    for (int i = 0; i < count; ++i)
        if (status[i]) {
            set_error("iga_batch_create: problem " + std::to_string(i) + ": " + message[i]);
            return fail(status[i]);
        }
    for (int i = 0; i < count; ++i) B->off[i + 1] = B->off[i] + B->plans[i]->nfunc;
    BT_TRY(B->arena.flush());   // the plans' tables and control points, then their geometry set-up
    B->arena.defer = false;
    B->ntot = B->off[count];
    // degree groups
    for (int i = 0; i < count; ++i) {
        const int P = B->plans[i]->p;
        bool found = false;
        for (auto &G : B->groups) found = found || G.P == P;
        if (!found) {
            BGroup G;
            G.P = P;
            for (int pi = 0; pi < 2; ++pi) {
                const int prec = pi ? IGA_FP32 : IGA_FP64;
                const int cap = warps_for(P, prec, 0);
                int w = warps_over && warps_over[P] > 0 ? warps_over[P] : tune_warps(tt, P, pi ? IGA_MIXED : IGA_FP64);
                if (w <= 0) w = cap;
                G.W[pi] = std::min(std::max(w, 1), cap);
            }
            B->groups.push_back(G);
        }
    }
    std::sort(B->groups.begin(), B->groups.end(), [](const BGroup &a, const BGroup &b) { return a.P > b.P; });
    int st;
    if ((st = setup_items(B, 0))) return fail(st);
    if (precision == IGA_MIXED && (st = setup_items(B, 1))) return fail(st);
    // chunks
    std::vector<int4> ch;
    std::vector<int> c0(count), nc(count);
    for (int i = 0; i < count; ++i) {
        const long long N = B->off[i + 1] - B->off[i];
        c0[i] = (int)ch.size();
        for (long long s0 = 0; s0 < N; s0 += kChunkLen)
            ch.push_back(make_int4(i, (int)s0, (int)std::min<long long>(kChunkLen, N - s0), (int)(ch.size() - c0[i])));
        nc[i] = (int)ch.size() - c0[i];
    }
    B->nchunks = (int)ch.size();
    if ((st = bupload(&B->chunks, ch)) || (st = bupload(&B->c0, c0)) || (st = bupload(&B->nc, nc)) ||
        (st = bupload(&B->d_off, B->off)))
        return fail(st);
    if ((st = bmalloc(&B->d_err, 1))) return fail(st);
    BT_TRY(cudaMemset(B->d_err, 0, sizeof(int)));
    if ((st = bmalloc(&B->partials, (size_t)B->nchunks * 4)) || (st = bmalloc(&B->counters, count)) ||
        (st = bmalloc(&B->sc, count)) || (st = bmalloc(&B->cfg, 1)) || (st = bmalloc(&B->act, count)) ||
        (st = bmalloc(&B->act64, count)))
        return fail(st);
    BT_TRY(cudaMemset(B->counters, 0, sizeof(unsigned) * count));
    BT_TRY(cudaMemset(B->sc, 0, sizeof(BScal) * count));
    if ((st = bupload(&B->ones, std::vector<int>(count, 1)))) return fail(st);
    BT_TRY(cudaMallocHost((void **)&B->h_cfg, sizeof(BCfg)));
    BT_TRY(cudaMallocHost((void **)&B->h_sc, sizeof(BScal) * count));
    for (int k = 0; k < 3; ++k) {
        BT_TRY(cudaStreamCreateWithFlags(&B->s[k], cudaStreamNonBlocking));
        BT_TRY(cudaStreamCreateWithFlags(&B->aux[k], cudaStreamNonBlocking));
    }
    BT_TRY(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming));
    BT_TRY(cudaEventCreateWithFlags(&B->join, cudaEventDisableTiming));
    if ((st = setup_params<double>(B))) return fail(st);
    if (precision == IGA_MIXED && (st = setup_params<float>(B))) return fail(st);
    const size_t N = (size_t)B->ntot;
    BVec<double> &v = B->v64;
    if ((st = bmalloc(&v.x, N)) || (st = bmalloc(&v.q, N))) return fail(st);
    if (solver) {
        if ((st = bmalloc(&v.r, N)) || (st = bmalloc(&v.z, N)) || (st = bmalloc(&v.p, N)) || (st = bmalloc(&v.b, N)))
            return fail(st);
        if (precision == IGA_MIXED) {
            BVec<float> &f = B->v32;
            if ((st = bmalloc(&f.x, N)) || (st = bmalloc(&f.r, N)) || (st = bmalloc(&f.z, N)) ||
                (st = bmalloc(&f.p, N)) || (st = bmalloc(&f.q, N)))
                return fail(st);
        }
        if ((st = setup_fd(B))) return fail(st);
    } else if (precision == IGA_MIXED) {
        if ((st = bmalloc(&B->v32.x, N)) || (st = bmalloc(&B->v32.q, N))) return fail(st);
    }
    // the plans' geometry set-up ran without a synchronisation each: check
    // their flags now, gathered by one kernel
    {
        std::vector<int *> flags(count);
        for (int i = 0; i < count; ++i) flags[i] = B->plans[i]->d_err;
        int **dflags = nullptr;
        int *dout = nullptr;
        if ((st = bupload(&dflags, flags)) || (st = bmalloc(&dout, count))) return fail(st);
        gather_flags_kernel<<<(count + 255) / 256, 256>>>(dflags, count, dout);
        std::vector<int> herr(count, 0);
        const cudaError_t e = cudaMemcpy(herr.data(), dout, sizeof(int) * count, cudaMemcpyDeviceToHost);
        cudaFree(dflags);
        cudaFree(dout);
        BT_TRY(e);
        for (int i = 0; i < count; ++i)
            if (herr[i]) {
                set_error("iga_batch_create: problem " + std::to_string(i) +
                          ": geometry has a non-positive Jacobian determinant");
                return fail(IGA_ERR_ARG);
            }
    }
    *out = B;
    return IGA_OK;
}

// Median time (us) of `reps` batched applies in precision pi after warm-up.
int time_apply(iga_batch *B, int pi, int reps, double &us)
{
    cudaStream_t s = B->s[0];
    cudaEvent_t e0, e1;
    BT_TRY(cudaEventCreate(&e0));
    BT_TRY(cudaEventCreate(&e1));
    if (pi == 0) BT_TRY(cudaMemsetAsync(B->v64.x, 0, sizeof(double) * B->ntot, s));
    else BT_TRY(cudaMemsetAsync(B->v32.x, 0, sizeof(float) * B->ntot, s));
    std::vector<float> t;
    int st = IGA_OK;
    for (int k = 0; k < reps + 3 && !st; ++k) {
        BT_TRY(cudaEventRecord(e0, s));
        st = pi == 0 ? batch_apply<double>(B, B->v64.x, B->v64.q, B->ones, s, B->aux[0])
                     : batch_apply<float>(B, B->v32.x, B->v32.q, B->ones, s, B->aux[0]);
        BT_TRY(cudaEventRecord(e1, s));
        BT_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        BT_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (k >= 3) t.push_back(ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    std::sort(t.begin(), t.end());
    us = 1000.0 * t[t.size() / 2];
    return IGA_OK;
}

}  // namespace

extern "C" {

void iga_batch_opts_default(iga_batch_opts *o)
{
    if (!o) return;
    o->precision = IGA_FP64;
    o->device = 0;
    o->tune_file = nullptr;
}

int iga_batch_create(const iga_mesh_desc *meshes, int count, const iga_batch_opts *opts_in, iga_batch **out)
{
    if (!out) return IGA_ERR_ARG;
    iga_batch_opts o;
    iga_batch_opts_default(&o);
    if (opts_in) o = *opts_in;
    TuneTable tt;
    if (o.tune_file) {
        std::string err;
        if (!tune_read(o.tune_file, tt, err)) {
            set_error(err);
            return IGA_ERR_ARG;
        }
    }
    return create_batch(meshes, count, o.precision, o.device, tt, nullptr, nullptr, true, out);
}

int iga_batch_destroy(iga_batch *B)
{
    if (!B) return IGA_OK;
    cudaSetDevice(B->device);
    B->arena.stop_copier();   // its queued copies read the plans' control points
    cudaDeviceSynchronize();
    if (B->graph) cudaGraphExecDestroy(B->graph);
    for (iga_plan *pl : B->plans) iga_plan_destroy(pl);
    B->plans.clear();
    B->arena.release();
    for (BGroup &G : B->groups)
        for (int pi = 0; pi < 2; ++pi)
            if (G.items[pi]) cudaFree(G.items[pi]);
    for (double *p : B->ycoef) cudaFree(p);
    for (void *p : {(void *)B->chunks, (void *)B->tiles, (void *)B->tiles_tc, (void *)B->d_err, (void *)B->rows, (void *)B->c0, (void *)B->nc, (void *)B->d_off,
                    (void *)B->partials, (void *)B->counters, (void *)B->sc, (void *)B->cfg, (void *)B->act,
                    (void *)B->act64, (void *)B->ones})
        if (p) cudaFree(p);
    free_vecs_common(B->v64);
    free_vecs_common(B->v32);
    if (B->h_cfg) cudaFreeHost(B->h_cfg);
    if (B->h_sc) cudaFreeHost(B->h_sc);
    for (int k = 0; k < 3; ++k) {
        if (B->s[k]) cudaStreamDestroy(B->s[k]);
        if (B->aux[k]) cudaStreamDestroy(B->aux[k]);
    }
    if (B->fork) cudaEventDestroy(B->fork);
    if (B->join) cudaEventDestroy(B->join);
    delete B;
    return IGA_OK;
}

int iga_batch_offsets(const iga_batch *B, int64_t *offsets)
{
    if (!B || !offsets) return IGA_ERR_ARG;
    for (int i = 0; i <= B->count; ++i) offsets[i] = B->off[i];
    return IGA_OK;
}

iga_plan *iga_batch_plan(iga_batch *B, int i)
{
    if (!B || i < 0 || i >= B->count) return nullptr;
    return B->plans[i];
}

int iga_batch_shape(const iga_batch *B, int i, int precision, int *rows, int *warps)
{
    if (!B || i < 0 || i >= B->count || !rows || !warps) return IGA_ERR_ARG;
    const int pi = prec_index(precision);
    const iga_plan *pl = B->plans[i];
    *rows = (pi ? pl->op32 : pl->op64).grid.TY;
    *warps = 0;
    for (const BGroup &G : B->groups)
        if (G.P == B->plans[i]->p) *warps = G.W[pi];
    return IGA_OK;
}

int iga_batch_apply(iga_batch *B, int precision, const void *x, void *y, void *stream)
{
    if (!B || !x || !y) return IGA_ERR_ARG;
    if (precision == IGA_FP32 && B->precision != IGA_MIXED) {
        set_error("iga_batch_apply: FP32 needs a MIXED batch");
        return IGA_ERR_ARG;
    }
    if (precision != IGA_FP64 && precision != IGA_FP32) return IGA_ERR_ARG;
    BT_TRY(cudaSetDevice(B->device));
    cudaStream_t s = (cudaStream_t)stream;
    return precision == IGA_FP64 ? batch_apply<double>(B, (const double *)x, (double *)y, B->ones, s, nullptr)
                                 : batch_apply<float>(B, (const float *)x, (float *)y, B->ones, s, nullptr);
}

int iga_batch_pc_apply(iga_batch *B, int pc, int precision, const void *r, void *z, void *stream)
{
    if (!B || !r || !z) return IGA_ERR_ARG;
    if (pc != IGA_PC_NONE && pc != IGA_PC_FEM_EXACT) {
        set_error("iga_batch_pc_apply: batches support IGA_PC_FEM_EXACT and IGA_PC_NONE");
        return IGA_ERR_UNSUPPORTED;
    }
    if ((precision != IGA_FP64 && precision != IGA_FP32) || (precision == IGA_FP32 && B->precision != IGA_MIXED))
        return IGA_ERR_ARG;
    BT_TRY(cudaSetDevice(B->device));
    cudaStream_t s = (cudaStream_t)stream;
    return precision == IGA_FP64 ? batch_pc<double>(B, pc, (const double *)r, (double *)z, B->ones, s)
                                 : batch_pc<float>(B, pc, (const float *)r, (float *)z, B->ones, s);
}

int iga_batch_solve(iga_batch *B, const double *b, double *x, const iga_solve_opts *o_in, iga_batch_stats *stats,
                    int *iterations, double *relres, void *stream)
{
    if (!B || !b || !x) return IGA_ERR_ARG;
    iga_solve_opts o;
    iga_solve_opts_default(&o);
    o.pc = IGA_PC_FEM_EXACT;
    if (o_in) o = *o_in;
    if (o.pc != IGA_PC_FEM_EXACT && o.pc != IGA_PC_NONE) {
        set_error("iga_batch_solve: batches support IGA_PC_FEM_EXACT and IGA_PC_NONE");
        return IGA_ERR_UNSUPPORTED;
    }
    if (!(o.rtol > 0.0) || o.max_it <= 0 || (B->precision == IGA_MIXED && (!(o.sweep_rtol > 0.0) || o.max_sweeps <= 0)))
        return IGA_ERR_ARG;
    const auto t0 = std::chrono::steady_clock::now();
    BT_TRY(cudaSetDevice(B->device));
    cudaStream_t s = B->s[0];
    cudaEvent_t ev;
    BT_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    BT_TRY(cudaEventRecord(ev, (cudaStream_t)stream));
    BT_TRY(cudaStreamWaitEvent(s, ev, 0));
    const size_t N = (size_t)B->ntot;
    B->h_cfg->rtol = o.rtol;
    B->h_cfg->sweep_rtol2 = o.sweep_rtol * o.sweep_rtol;
    B->h_cfg->maxit = o.max_it;
    B->h_cfg->max_sweeps = o.max_sweeps;
    BT_TRY(cudaMemcpyAsync(B->cfg, B->h_cfg, sizeof(BCfg), cudaMemcpyHostToDevice, s));
    BT_TRY(cudaMemcpyAsync(B->v64.b, b, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    if (o.x0_nonzero) BT_TRY(cudaMemcpyAsync(B->v64.x, x, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    else BT_TRY(cudaMemsetAsync(B->v64.x, 0, sizeof(double) * N, s));
    BT_TRY(cudaMemsetAsync(B->sc, 0, sizeof(BScal) * B->count, s));
    BT_TRY(cudaMemcpyAsync(B->act64, B->ones, sizeof(int) * B->count, cudaMemcpyDeviceToDevice, s));
    BT_TRY(cudaMemsetAsync(B->act, 0, sizeof(int) * B->count, s));
    int st = IGA_OK;
    if (!B->graph || B->graph_pc != o.pc) {
        st = build_graph(B, o.pc, B->precision == IGA_MIXED && B->graph_nested);
        if (st == IGA_ERR_UNSUPPORTED && B->precision == IGA_MIXED && B->graph_nested) {
            B->graph_nested = false;   // nested loops not instantiable: host loop over sweep graphs
            st = build_graph(B, o.pc, false);
        }
        if (st) {
            cudaEventDestroy(ev);
            return st;
        }
    }
    auto any_active = [&](bool &any) -> int {
        BT_TRY(cudaMemcpyAsync(B->h_sc, B->sc, sizeof(BScal) * B->count, cudaMemcpyDeviceToHost, s));
        std::vector<int> a(B->count);
        BT_TRY(cudaMemcpyAsync(a.data(), B->act64, sizeof(int) * B->count, cudaMemcpyDeviceToHost, s));
        BT_TRY(cudaStreamSynchronize(s));
        any = false;
        for (int v : a) any = any || v;
        return IGA_OK;
    };
    bool any = false;
    if (B->precision == IGA_FP64) {
        // Restart from the true residual while a problem misses rtol (recurrence drift).
        for (int restart = 0; restart < 4; ++restart) {
            BT_TRY(cudaGraphLaunch(B->graph, s));
            if ((st = any_active(any))) break;
            if (!any) break;
        }
    } else if (B->graph_nested) {
        BT_TRY(cudaGraphLaunch(B->graph, s));
        st = any_active(any);
    } else {
        // initial residual, then one graph launch per sweep
        if (!(st = batch_apply<double>(B, B->v64.x, B->v64.q, B->act64, s, B->aux[0]))) {
            bk_res64<<<B->nchunks, kBT, 0, s>>>(B->dev(), B->act64, B->v64.b, B->v64.q, B->v64.r, 2);
            st = any_active(any);
        }
        for (int sw = 0; !st && any && sw < o.max_sweeps; ++sw) {
            BT_TRY(cudaGraphLaunch(B->graph, s));
            st = any_active(any);
        }
    }
    BT_TRY(cudaMemcpyAsync(x, B->v64.x, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    BT_TRY(cudaEventRecord(ev, s));
    BT_TRY(cudaStreamWaitEvent((cudaStream_t)stream, ev, 0));
    BT_TRY(cudaStreamSynchronize(s));
    cudaEventDestroy(ev);
    if (st) return st;
    int herr = 0;
    BT_TRY(cudaMemcpy(&herr, B->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) {
        BT_TRY(cudaMemset(B->d_err, 0, sizeof(int)));
        set_error("iga_batch_solve: a bounded device wait gave up (tensor-core preconditioner tiles)");
        return IGA_ERR_TIMEOUT;
    }
    iga_batch_stats S{};
    int result = IGA_OK;
    for (int i = 0; i < B->count; ++i) {
        const BScal &c = B->h_sc[i];
        const bool ok = c.status == 0 && c.relres <= o.rtol;
        S.converged += ok;
        if (!ok && result == IGA_OK) result = c.status ? c.status : IGA_ERR_NOT_CONVERGED;
        S.max_iterations = std::max(S.max_iterations, c.itot);
        S.total_iterations += c.itot;
        S.max_sweeps = std::max(S.max_sweeps, c.sweeps);
        S.max_relres = std::max(S.max_relres, std::isfinite(c.relres) ? c.relres : INFINITY);
        if (iterations) iterations[i] = c.itot;
        if (relres) relres[i] = c.relres;
    }
    S.status = result;
    S.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (stats) *stats = S;
    return result;
}

int iga_tune_lookup(const char *tune_file, int p, int precision, int nElemX, int nElemY, int *rows, int *warps)
{
    (void)nElemX;
    if (!tune_file || !rows || !warps) return IGA_ERR_ARG;
    TuneTable tt;
    std::string err;
    if (!tune_read(tune_file, tt, err)) {
        set_error(err);
        return IGA_ERR_ARG;
    }
    const int prec = precision == IGA_MIXED ? IGA_MIXED : IGA_FP64;
    *rows = tune_rows(tt, p, prec, nElemY);
    *warps = tune_warps(tt, p, prec);
    return IGA_OK;
}

int iga_batch_autotune(const iga_mesh_desc *meshes, int count, int precision, int device, const char *tune_file)
{
    if (!meshes || count <= 0 || !tune_file || (precision != IGA_FP64 && precision != IGA_MIXED)) return IGA_ERR_ARG;
    TuneTable tt;
    std::string err;
    if (!tune_read(tune_file, tt, err)) {
        set_error(err);
        return IGA_ERR_ARG;
    }
    BT_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    BT_TRY(cudaGetDeviceProperties(&prop, device));
    tt.device = prop.name;
    tt.sm_count = prop.multiProcessorCount;
    const int pi = precision == IGA_MIXED ? 1 : 0;
    const int kprec = precision == IGA_MIXED ? IGA_MIXED : IGA_FP64;
    std::vector<int> degrees;
    for (int i = 0; i < count; ++i)
        if (std::find(degrees.begin(), degrees.end(), meshes[i].p) == degrees.end()) degrees.push_back(meshes[i].p);
    for (int P : degrees) {
        // 1) rows per strip, per size bucket, at the largest warps per CTA
        std::map<int, std::vector<int>> buckets;
        for (int i = 0; i < count; ++i)
            if (meshes[i].p == P) buckets[tune_bucket(meshes[i].nElemY)].push_back(i);
        std::vector<int> rows_of(count, 0);
        for (auto &kv : buckets) {
            std::vector<iga_mesh_desc> sub;
            int maxney = 0;
            for (int i : kv.second) {
                sub.push_back(meshes[i]);
                maxney = std::max(maxney, meshes[i].nElemY);
            }
            int best = 0;
            double best_us = 1e300;
            for (int ty : {8, 12, 16, 24, 32, 48, 64, 96, 128}) {
                if (ty < P || (ty > maxney && ty != 8 && ty / 2 >= maxney)) continue;
                std::vector<int> r(sub.size(), ty);
                iga_batch *B = nullptr;
                int st = create_batch(sub.data(), (int)sub.size(), precision, device, tt, r.data(), nullptr, false, &B);
                if (st) return st;
                double us = 0.0;
                st = time_apply(B, pi, 10, us);
                iga_batch_destroy(B);
                if (st) return st;
                if (us < best_us) {
                    best_us = us;
                    best = ty;
                }
            }
            tune_set_rows(tt, P, kprec, kv.first, best, best_us);
            for (int i : kv.second) rows_of[i] = best;
        }
        // 2) warps per CTA for the whole degree group at the chosen rows
        std::vector<iga_mesh_desc> sub;
        std::vector<int> r;
        for (int i = 0; i < count; ++i)
            if (meshes[i].p == P) {
                sub.push_back(meshes[i]);
                r.push_back(rows_of[i]);
            }
        const int cap = warps_for(P, pi ? IGA_FP32 : IGA_FP64, 0);
        std::vector<int> cands;
        for (int w : {cap, (3 * cap) / 4, cap / 2, cap / 3, cap / 4, 2, 1})
            if (w >= 1 && std::find(cands.begin(), cands.end(), w) == cands.end()) cands.push_back(w);
        int bestw = cap;
        double best_us = 1e300;
        for (int w : cands) {
            int wo[6] = {0, 0, 0, 0, 0, 0};
            if (P >= 1 && P <= 5) wo[P] = w;
            iga_batch *B = nullptr;
            int st = create_batch(sub.data(), (int)sub.size(), precision, device, tt, r.data(), wo, false, &B);
            if (st) return st;
            double us = 0.0;
            st = time_apply(B, pi, 10, us);
            iga_batch_destroy(B);
            if (st) return st;
            if (us < best_us) {
                best_us = us;
                bestw = w;
            }
        }
        tune_set_warps(tt, P, kprec, bestw, best_us);
    }
    if (!tune_write(tune_file, tt, err)) {
        set_error(err);
        return IGA_ERR_ARG;
    }
    return IGA_OK;
}

}  // extern "C"
