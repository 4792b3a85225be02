// Multi-rank MatMult and flexible PCG over partitioned meshes, one rank per
// GPU, NCCL between the ranks (include/iga_dist.h).
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/iga_dist.h"
#include "iga_plan.hpp"

namespace iga {
namespace {

// ------------------------------------------------------------ NCCL at run time
struct NcclApi {
    void *h = nullptr;
    ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
    ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
    ncclResult_t (*GroupStart)() = nullptr;
    ncclResult_t (*GroupEnd)() = nullptr;
    ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                              cudaStream_t) = nullptr;
    ncclResult_t (*AllGather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
    const char *(*ErrorString)(ncclResult_t) = nullptr;
};

const NcclApi *nccl()
{
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) return;
        bool ok = true;
        auto sym = [&](auto &fn, const char *name) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
            ok = ok && fn;
        };
        sym(api.GetUniqueId, "ncclGetUniqueId");
        sym(api.CommInitRank, "ncclCommInitRank");
        sym(api.CommDestroy, "ncclCommDestroy");
        sym(api.GroupStart, "ncclGroupStart");
        sym(api.GroupEnd, "ncclGroupEnd");
        sym(api.Send, "ncclSend");
        sym(api.Recv, "ncclRecv");
        sym(api.AllReduce, "ncclAllReduce");
        sym(api.AllGather, "ncclAllGather");
        sym(api.ErrorString, "ncclGetErrorString");
        if (ok) api.h = h;
    });
    if (!api.h) set_error("libnccl.so.2 could not be loaded");
    return api.h ? &api : nullptr;
}

#define NCCL_TRY(call)                                                                        \
    do {                                                                                      \
        const ncclResult_t r_ = (call);                                                       \
        if (r_ != ncclSuccess) {                                                              \
            set_error(std::string("NCCL: ") + nc->ErrorString(r_) + " (" #call ")");          \
            return IGA_ERR_CUDA;                                                              \
        }                                                                                     \
    } while (0)

#define DCUDA_TRY(call)                                                                       \
    do {                                                                                      \
        const cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                              \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                    \
            return e_ == cudaErrorMemoryAllocation ? IGA_ERR_NOMEM : IGA_ERR_CUDA;            \
        }                                                                                     \
    } while (0)

// ------------------------------------------------------------ kernels
constexpr int kDB = 256, kDT = 256;   // dot-product grid (fixed: deterministic partials)

struct DistScalars {
    double red[4];                  // all-reduction buffer
    double bb, rr, rz, alpha, beta, tol2;
    int done, breakdown, it, maxit;
};

struct DotPtrs {
    const double *a[3], *b[3];
};

// Block partials of K dot products a[k] . b[k] over n entries.
template <int K>
__global__ void dot_partial_kernel(DotPtrs pp, long long n, double *__restrict__ partials)
{
    const double *const *a = pp.a, *const *b = pp.b;
    double v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] += a[k][i] * b[k][i];
    __shared__ double sh[K][kDT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = v[k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) sh[k][w] = s;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int j = 0; j < kDT / 32; ++j) s += sh[threadIdx.x][j];
        partials[(size_t)threadIdx.x * kDB + blockIdx.x] = s;
    }
}

// out[k] = sum of the block partials of dot k, in block order.
template <int K>
__global__ void dot_final_kernel(const double *__restrict__ partials, double *__restrict__ out)
{
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int j = 0; j < kDB; ++j) s += partials[(size_t)threadIdx.x * kDB + j];
        out[threadIdx.x] = s;
    }
}

__global__ void gather_kernel(double *__restrict__ dst, const double *__restrict__ src, const int *__restrict__ idx,
                              long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[idx[i]];
}

__global__ void scatter_kernel(double *__restrict__ dst, const int *__restrict__ idx, const double *__restrict__ src,
                               long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[idx[i]] = src[i];
}

// dst[idx[i]] += src[i]; indices distinct within one call (one peer).
__global__ void scatter_add_kernel(double *__restrict__ dst, const int *__restrict__ idx,
                                   const double *__restrict__ src, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[idx[i]] += src[i];
}

__global__ void copy_kernel(double *__restrict__ dst, const double *__restrict__ src, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

__global__ void zero_kernel(double *__restrict__ dst, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = 0.0;
}

// r = b - q (the true residual).
__global__ void sub_kernel(double *__restrict__ r, const double *__restrict__ b, const double *__restrict__ q,
                           long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        r[i] = b[i] - q[i];
}

__global__ void init_scalars_kernel(DistScalars *s, double rtol, int maxit)
{
    s->bb = s->red[0];
    s->rr = s->red[1];
    s->rz = s->red[2];
    s->tol2 = rtol * rtol * s->bb;
    s->it = 0;
    s->maxit = maxit;
    s->breakdown = 0;
    s->done = (s->rr <= s->tol2) || !(s->bb > 0.0) || maxit <= 0;
}

__global__ void alpha_kernel(DistScalars *s)
{
    if (s->done) return;
    const double pq = s->red[0];
    if (!(pq > 0.0)) {
        s->breakdown = 1;
        s->done = 1;
        return;
    }
    s->alpha = s->rz / pq;
}

// x += alpha p, r -= alpha q (skipped once the loop is done).
__global__ void xr_kernel(double *__restrict__ x, double *__restrict__ r, const double *__restrict__ p,
                          const double *__restrict__ q, long long n, const DistScalars *__restrict__ s)
{
    if (s->done) return;
    const double a = s->alpha;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        x[i] += a * p[i];
        r[i] -= a * q[i];
    }
}

// Flexible (Polak-Ribiere) beta from red = [r.r, r.z, r.z_old]; convergence test.
__global__ void beta_kernel(DistScalars *s)
{
    if (s->done) return;
    const double rr = s->red[0], rzn = s->red[1], rzo = s->red[2];
    s->it += 1;
    s->beta = (rzn - rzo) / s->rz;
    s->rz = rzn;
    s->rr = rr;
    s->done = !(rr > s->tol2) || s->it >= s->maxit || !(rr == rr) || !(s->beta == s->beta);
}

__global__ void p_kernel(double *__restrict__ p, const double *__restrict__ z, long long n,
                         const DistScalars *__restrict__ s)
{
    if (s->done) return;
    const double be = s->beta;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = z[i] + be * p[i];
}

inline dim3 grid_for(long long n) { return dim3((unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 4 * 148))); }

}  // namespace
}  // namespace iga

using namespace iga;

struct iga_dist {
    iga_part *part = nullptr;
    ncclComm_t comm = nullptr;
    int nranks = 1, rank = 0, device = 0;
    long long nowned = 0, nghost = 0, nblock = 0;
    std::vector<int> recv_count, send_count;      // per peer
    std::vector<long long> recv_off, send_off;    // per peer, offsets into the concatenated lists
    long long nsend = 0;
    int *d_recv_pos = nullptr;   // ghost-list positions, grouped by owner
    int *d_recv_loc = nullptr;   // the same as local-form indices (nowned + position)
    int *d_send_idx = nullptr;   // owned-local indices, grouped by peer
    int *d_pos = nullptr;        // block position of every owned entry
    double *sendbuf = nullptr, *recvbuf = nullptr;
    double *x_local = nullptr, *y_local = nullptr;   // local forms (owned | ghosts)
    double *p_local = nullptr;                       // the search direction in local form
    double *r = nullptr, *z = nullptr, *q = nullptr; // owned vectors
    double *rb = nullptr, *zb = nullptr;             // block vectors of the preconditioner
    double *partials = nullptr;
    DistScalars *s = nullptr, *h_s = nullptr;
    iga_plan *pc_plan = nullptr;   // the sub-patch's plan for the block preconditioner
};

namespace {

// Forward ghost update: src_owned -> ghosts of dst_local (dst_local[:nowned] is the caller's business).
int forward_update(iga_dist *d, const double *src_owned, double *dst_local, cudaStream_t st)
{
    const NcclApi *nc = d->nranks > 1 ? nccl() : nullptr;
    if (d->nranks > 1 && !nc) return IGA_ERR_CUDA;
    if (d->nsend) gather_kernel<<<grid_for(d->nsend), 256, 0, st>>>(d->sendbuf, src_owned, d->d_send_idx, d->nsend);
    if (d->nranks > 1) {
        NCCL_TRY(nc->GroupStart());
        for (int q = 0; q < d->nranks; ++q) {
            if (d->send_count[q]) NCCL_TRY(nc->Send(d->sendbuf + d->send_off[q], d->send_count[q], ncclDouble, q, d->comm, st));
            if (d->recv_count[q]) NCCL_TRY(nc->Recv(d->recvbuf + d->recv_off[q], d->recv_count[q], ncclDouble, q, d->comm, st));
        }
        NCCL_TRY(nc->GroupEnd());
    }
    if (d->nghost) scatter_kernel<<<grid_for(d->nghost), 256, 0, st>>>(dst_local, d->d_recv_loc, d->recvbuf, d->nghost);
    return cudaPeekAtLastError() == cudaSuccess ? IGA_OK : IGA_ERR_CUDA;
}

// Reverse add: y_owned = y_local[:nowned] + the peers' ghost rows, peer by peer in ascending rank order.
int reverse_add(iga_dist *d, const double *y_local, double *y_owned, cudaStream_t st)
{
    const NcclApi *nc = d->nranks > 1 ? nccl() : nullptr;
    if (d->nranks > 1 && !nc) return IGA_ERR_CUDA;
    copy_kernel<<<grid_for(d->nowned), 256, 0, st>>>(y_owned, y_local, d->nowned);
    if (d->nghost) gather_kernel<<<grid_for(d->nghost), 256, 0, st>>>(d->recvbuf, y_local, d->d_recv_loc, d->nghost);
    if (d->nranks > 1) {
        NCCL_TRY(nc->GroupStart());
        for (int q = 0; q < d->nranks; ++q) {
            if (d->recv_count[q]) NCCL_TRY(nc->Send(d->recvbuf + d->recv_off[q], d->recv_count[q], ncclDouble, q, d->comm, st));
            if (d->send_count[q]) NCCL_TRY(nc->Recv(d->sendbuf + d->send_off[q], d->send_count[q], ncclDouble, q, d->comm, st));
        }
        NCCL_TRY(nc->GroupEnd());
    }
    for (int q = 0; q < d->nranks; ++q)
        if (d->send_count[q])
            scatter_add_kernel<<<grid_for(d->send_count[q]), 256, 0, st>>>(y_owned, d->d_send_idx + d->send_off[q],
                                                                          d->sendbuf + d->send_off[q], d->send_count[q]);
    return cudaPeekAtLastError() == cudaSuccess ? IGA_OK : IGA_ERR_CUDA;
}

int dist_matmult(iga_dist *d, const double *x_owned_in_local, double *x_local, double *y_owned, cudaStream_t st)
{
    int e;
    if (x_owned_in_local != x_local) copy_kernel<<<grid_for(d->nowned), 256, 0, st>>>(x_local, x_owned_in_local, d->nowned);
    if ((e = forward_update(d, x_local, x_local, st))) return e;
    if ((e = iga_part_apply(d->part, x_local, d->y_local, st))) return e;
    return reverse_add(d, d->y_local, y_owned, st);
}

// Local dots of K pairs into s->red[first .. first+K-1] (deterministic).
template <int K>
int local_dots(iga_dist *d, const double *const (&a)[K], const double *const (&b)[K], int first, cudaStream_t st)
{
    DotPtrs pp = {};
    for (int k = 0; k < K; ++k) {
        pp.a[k] = a[k];
        pp.b[k] = b[k];
    }
    dot_partial_kernel<K><<<kDB, kDT, 0, st>>>(pp, d->nowned, d->partials);
    dot_final_kernel<K><<<1, 32, 0, st>>>(d->partials, d->s->red + first);
    return cudaPeekAtLastError() == cudaSuccess ? IGA_OK : IGA_ERR_CUDA;
}

int allreduce(iga_dist *d, int k, cudaStream_t st)
{
    if (d->nranks == 1) return IGA_OK;
    const NcclApi *nc = nccl();
    if (!nc) return IGA_ERR_CUDA;
    NCCL_TRY(nc->AllReduce(d->s->red, d->s->red, k, ncclDouble, ncclSum, d->comm, st));
    return IGA_OK;
}

// z = M^-1 r: the exact FEM inverse of the rank's sub-patch on r placed in its block, restricted to the owned entries.
int precond(iga_dist *d, int pc, const double *r, double *z, cudaStream_t st)
{
    if (pc == IGA_PC_NONE) {
        copy_kernel<<<grid_for(d->nowned), 256, 0, st>>>(z, r, d->nowned);
        return cudaPeekAtLastError() == cudaSuccess ? IGA_OK : IGA_ERR_CUDA;
    }
    zero_kernel<<<grid_for(d->nblock), 256, 0, st>>>(d->rb, d->nblock);
    scatter_kernel<<<grid_for(d->nowned), 256, 0, st>>>(d->rb, d->d_pos, r, d->nowned);
    int e = iga_pc_apply(d->pc_plan, IGA_PC_FEM_EXACT, IGA_FP64, d->rb, d->zb, 1e-10, 10000, st);
    if (e) return e;
    gather_kernel<<<grid_for(d->nowned), 256, 0, st>>>(z, d->zb, d->d_pos, d->nowned);
    return cudaPeekAtLastError() == cudaSuccess ? IGA_OK : IGA_ERR_CUDA;
}

}  // namespace

extern "C" {

int iga_dist_unique_id(void *id128)
{
    const NcclApi *nc = nccl();
    if (!nc || !id128) return nc ? IGA_ERR_ARG : IGA_ERR_CUDA;
    ncclUniqueId id;
    NCCL_TRY(nc->GetUniqueId(&id));
    memcpy(id128, &id, sizeof(id));
    return IGA_OK;
}

int iga_dist_comm_create(int nranks, int rank, const void *id128, int device, void **comm)
{
    const NcclApi *nc = nccl();
    if (!nc) return IGA_ERR_CUDA;
    if (!id128 || !comm || nranks < 1 || rank < 0 || rank >= nranks) return IGA_ERR_ARG;
    DCUDA_TRY(cudaSetDevice(device));
    ncclUniqueId id;
    memcpy(&id, id128, sizeof(id));
    ncclComm_t c = nullptr;
    NCCL_TRY(nc->CommInitRank(&c, nranks, id, rank));
    *comm = c;
    return IGA_OK;
}

int iga_dist_comm_destroy(void *comm)
{
    const NcclApi *nc = nccl();
    if (!nc) return IGA_ERR_CUDA;
    if (comm) NCCL_TRY(nc->CommDestroy((ncclComm_t)comm));
    return IGA_OK;
}

int iga_dist_exchange_maps(int nranks, int rank, const int64_t *offsets, const int *ghost_counts, const int64_t *ghosts,
                           int *recv_count, int *recv_pos, int *send_count, int *send_idx, int64_t send_cap,
                           int64_t *nsend)
{
    if (nranks < 1 || rank < 0 || rank >= nranks || !offsets || !ghost_counts || !recv_count || !send_count ||
        !nsend)
        return IGA_ERR_ARG;
    for (int q = 0; q < nranks; ++q)
        if (offsets[q + 1] < offsets[q] || ghost_counts[q] < 0) return IGA_ERR_ARG;
    std::vector<long long> gstart(nranks + 1, 0);
    for (int q = 0; q < nranks; ++q) gstart[q + 1] = gstart[q] + ghost_counts[q];
    auto owner = [&](int64_t g) {
        const int64_t *it = std::upper_bound(offsets, offsets + nranks + 1, g);
        return (int)(it - offsets) - 1;
    };
    // this rank's ghosts grouped by owner (ascending owner, then position)
    std::vector<std::vector<int>> by_owner(nranks);
    for (long long k = 0; k < ghost_counts[rank]; ++k) {
        const int64_t g = ghosts[gstart[rank] + k];
        const int o = owner(g);
        if (o < 0 || o >= nranks || o == rank || g >= offsets[nranks]) {
            set_error("iga_dist_exchange_maps: a ghost outside the other ranks' owned ranges");
            return IGA_ERR_ARG;
        }
        by_owner[o].push_back((int)k);
    }
    long long w = 0;
    for (int q = 0; q < nranks; ++q) {
        recv_count[q] = (int)by_owner[q].size();
        for (int k : by_owner[q]) {
            if (recv_pos) recv_pos[w] = k;
            ++w;
        }
    }
    // entries of this rank that each peer holds as ghosts, in the peer's ghost-list order
    long long ns = 0;
    for (int q = 0; q < nranks; ++q) {
        int c = 0;
        if (q != rank)
            for (long long k = 0; k < ghost_counts[q]; ++k) {
                const int64_t g = ghosts[gstart[q] + k];
                if (g >= offsets[rank] && g < offsets[rank + 1]) {
                    if (send_idx) {
                        if (ns >= send_cap) {
                            set_error("iga_dist_exchange_maps: send_cap too small");
                            return IGA_ERR_ARG;
                        }
                        send_idx[ns] = (int)(g - offsets[rank]);
                    }
                    ++ns;
                    ++c;
                }
            }
        send_count[q] = c;
    }
    *nsend = ns;
    return IGA_OK;
}

int iga_dist_create(iga_part *part, void *comm, int nranks, int rank, int device, iga_dist **out)
{
    if (!part || !out || nranks < 1 || rank < 0 || rank >= nranks || (nranks > 1 && !comm)) return IGA_ERR_ARG;
    *out = nullptr;
    const NcclApi *nc = nranks > 1 ? nccl() : nullptr;
    if (nranks > 1 && !nc) return IGA_ERR_CUDA;
    iga_part_info info;
    int st;
    if ((st = iga_part_get_info(part, &info))) return st;
    if (info.rank != rank) {
        set_error("iga_dist_create: the part's rank differs from the communicator rank");
        return IGA_ERR_ARG;
    }
    iga_opts o;
    iga_opts_default(&o);
    o.sign = IGA_SIGN_SPD;
    o.bc = IGA_BC_IDENTITY;
    o.device = device;
    if ((st = iga_part_build(part, &o))) return st;
    DCUDA_TRY(cudaSetDevice(device));
    iga_dist *d = new iga_dist();
    d->part = part;
    d->comm = (ncclComm_t)comm;
    d->nranks = nranks;
    d->rank = rank;
    d->device = device;
    d->nowned = info.nlocalfunc;
    d->nghost = info.nghost;
    d->nblock = (long long)info.block_m * info.block_n;
    auto fail = [&](int code) {
        iga_dist_destroy(d);
        return code;
    };
    // every rank's owned range and ghost list (all-gathers through NCCL, staged on the device)
    std::vector<int64_t> ghosts_mine(d->nghost);
    if (d->nghost && (st = iga_part_ghosts(part, ghosts_mine.data()))) return fail(st);
    std::vector<int64_t> meta(3 * nranks, 0);   // (owned offset, owned count, ghost count) per rank
    meta[3 * rank] = info.owned_offset;
    meta[3 * rank + 1] = d->nowned;
    meta[3 * rank + 2] = d->nghost;
    cudaStream_t s0 = nullptr;
    DCUDA_TRY(cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking));
    auto gather_all = [&](std::vector<int64_t> &all, const int64_t *mine, size_t count) -> int {
        if (nranks == 1) {
            std::copy(mine, mine + count, all.begin());
            return IGA_OK;
        }
        int64_t *dv = nullptr;
        DCUDA_TRY(cudaMalloc((void **)&dv, sizeof(int64_t) * count * (nranks + 1)));
        cudaMemcpy(dv, mine, sizeof(int64_t) * count, cudaMemcpyHostToDevice);
        const ncclResult_t r = nc->AllGather(dv, dv + count, count * 2, ncclInt32, d->comm, s0);   // int64 as 2 x int32
        cudaError_t e = cudaStreamSynchronize(s0);
        if (r == ncclSuccess && e == cudaSuccess)
            e = cudaMemcpy(all.data(), dv + count, sizeof(int64_t) * count * nranks, cudaMemcpyDeviceToHost);
        cudaFree(dv);
        if (r != ncclSuccess) {
            set_error(std::string("NCCL all-gather: ") + nc->ErrorString(r));
            return IGA_ERR_CUDA;
        }
        return e == cudaSuccess ? IGA_OK : IGA_ERR_CUDA;
    };
    std::vector<int64_t> meta_all(3 * nranks);
    st = gather_all(meta_all, meta.data() + 3 * rank, 3);
    std::vector<int64_t> offsets(nranks + 1, 0);
    std::vector<int> gcount(nranks, 0);
    long long gmax = 0;
    if (!st) {
        for (int q = 0; q < nranks; ++q) {
            offsets[q] = meta_all[3 * q];
            gcount[q] = (int)meta_all[3 * q + 2];
            gmax = std::max<long long>(gmax, gcount[q]);
            if (q + 1 < nranks && meta_all[3 * q] + meta_all[3 * q + 1] != meta_all[3 * (q + 1)]) {
                set_error("iga_dist_create: owned ranges are not contiguous in rank order");
                st = IGA_ERR_ARG;
            }
        }
        offsets[nranks] = meta_all[3 * (nranks - 1)] + meta_all[3 * (nranks - 1) + 1];
    }
    std::vector<int64_t> ghosts_padded, ghosts_all;
    if (!st) {   // ghost lists padded to the longest, all-gathered, then packed in rank order
        ghosts_padded.assign(std::max<long long>(gmax, 1), -1);
        std::copy(ghosts_mine.begin(), ghosts_mine.end(), ghosts_padded.begin());
        std::vector<int64_t> gall(ghosts_padded.size() * nranks);
        st = gather_all(gall, ghosts_padded.data(), ghosts_padded.size());
        for (int q = 0; q < nranks && !st; ++q)
            ghosts_all.insert(ghosts_all.end(), gall.begin() + q * ghosts_padded.size(),
                              gall.begin() + q * ghosts_padded.size() + gcount[q]);
    }
    cudaStreamDestroy(s0);
    if (st) return fail(st);
    d->recv_count.assign(nranks, 0);
    d->send_count.assign(nranks, 0);
    std::vector<int> recv_pos(std::max<long long>(d->nghost, 1));
    long long total_ghosts = (long long)ghosts_all.size();
    std::vector<int> send_idx(std::max<long long>(total_ghosts, 1));
    int64_t nsend = 0;
    if ((st = iga_dist_exchange_maps(nranks, rank, offsets.data(), gcount.data(), ghosts_all.data(),
                                     d->recv_count.data(), recv_pos.data(), d->send_count.data(), send_idx.data(),
                                     (int64_t)send_idx.size(), &nsend)))
        return fail(st);
    d->nsend = nsend;
    d->recv_off.assign(nranks + 1, 0);
    d->send_off.assign(nranks + 1, 0);
    for (int q = 0; q < nranks; ++q) {
        d->recv_off[q + 1] = d->recv_off[q] + d->recv_count[q];
        d->send_off[q + 1] = d->send_off[q] + d->send_count[q];
    }
    std::vector<int> recv_loc(recv_pos.size());
    for (size_t k = 0; k < recv_pos.size(); ++k) recv_loc[k] = (int)(d->nowned + recv_pos[k]);
    // block positions of the owned entries
    std::vector<int32_t> blk2loc(d->nblock);
    if ((st = iga_part_block_map(part, blk2loc.data()))) return fail(st);
    std::vector<int> pos(std::max<long long>(d->nowned, 1), -1);
    for (long long b = 0; b < d->nblock; ++b)
        if (blk2loc[b] >= 0 && blk2loc[b] < d->nowned) pos[blk2loc[b]] = (int)b;
    for (long long i = 0; i < d->nowned; ++i)
        if (pos[i] < 0) {
            set_error("iga_dist_create: an owned entry outside the part's block");
            return fail(IGA_ERR_ARG);
        }
    const long long nl = d->nowned + d->nghost;
    auto dmalloc = [&](auto **p, size_t n) -> int {
        DCUDA_TRY(cudaMalloc((void **)p, sizeof(**p) * std::max<size_t>(n, 1)));
        return IGA_OK;
    };
    if ((st = dmalloc(&d->d_recv_pos, recv_pos.size())) || (st = dmalloc(&d->d_recv_loc, recv_loc.size())) ||
        (st = dmalloc(&d->d_send_idx, send_idx.size())) || (st = dmalloc(&d->d_pos, pos.size())) ||
        (st = dmalloc(&d->sendbuf, std::max<long long>(nsend, d->nghost))) ||
        (st = dmalloc(&d->recvbuf, std::max<long long>(nsend, d->nghost))) || (st = dmalloc(&d->x_local, nl)) ||
        (st = dmalloc(&d->y_local, nl)) || (st = dmalloc(&d->p_local, nl)) || (st = dmalloc(&d->r, d->nowned)) ||
        (st = dmalloc(&d->z, d->nowned)) || (st = dmalloc(&d->q, d->nowned)) || (st = dmalloc(&d->rb, d->nblock)) ||
        (st = dmalloc(&d->zb, d->nblock)) || (st = dmalloc(&d->partials, 4 * kDB)) || (st = dmalloc(&d->s, 1)))
        return fail(st);
    auto up = [&](void *dst, const void *src, size_t bytes) -> int {
        if (bytes) DCUDA_TRY(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
        return IGA_OK;
    };
    if ((st = up(d->d_recv_pos, recv_pos.data(), sizeof(int) * d->nghost)) ||
        (st = up(d->d_recv_loc, recv_loc.data(), sizeof(int) * d->nghost)) ||
        (st = up(d->d_send_idx, send_idx.data(), sizeof(int) * nsend)) ||
        (st = up(d->d_pos, pos.data(), sizeof(int) * d->nowned)))
        return fail(st);
    cudaMemset(d->x_local, 0, sizeof(double) * nl);
    cudaMemset(d->p_local, 0, sizeof(double) * nl);
    if (cudaMallocHost((void **)&d->h_s, sizeof(DistScalars)) != cudaSuccess) return fail(IGA_ERR_NOMEM);
    // the block preconditioner's plan: the part's sub-patch (on-the-fly geometry: no G needed)
    iga_mesh_desc md;
    if ((st = iga_part_mesh(part, &md))) return fail(st);
    iga_opts po;
    iga_opts_default(&po);
    po.geometry = IGA_GEOM_ON_THE_FLY;
    po.device = device;
    if ((st = iga_plan_create(&md, &po, &d->pc_plan))) return fail(st);
    *out = d;
    return IGA_OK;
}

int iga_dist_destroy(iga_dist *d)
{
    if (!d) return IGA_OK;
    cudaSetDevice(d->device);
    cudaDeviceSynchronize();
    for (void *p : {(void *)d->d_recv_pos, (void *)d->d_recv_loc, (void *)d->d_send_idx, (void *)d->d_pos,
                    (void *)d->sendbuf, (void *)d->recvbuf, (void *)d->x_local, (void *)d->y_local, (void *)d->p_local,
                    (void *)d->r, (void *)d->z, (void *)d->q, (void *)d->rb, (void *)d->zb, (void *)d->partials,
                    (void *)d->s})
        if (p) cudaFree(p);
    if (d->h_s) cudaFreeHost(d->h_s);
    if (d->pc_plan) iga_plan_destroy(d->pc_plan);
    delete d;
    return IGA_OK;
}

int iga_dist_apply(iga_dist *d, const double *x_owned, double *y_owned, void *stream)
{
    if (!d || !x_owned || !y_owned) return IGA_ERR_ARG;
    DCUDA_TRY(cudaSetDevice(d->device));
    return dist_matmult(d, x_owned, d->x_local, y_owned, (cudaStream_t)stream);
}

int iga_dist_solve(iga_dist *d, const double *b, double *x, const iga_solve_opts *o_in, iga_solve_stats *stats,
                   void *stream)
{
    if (!d || !b || !x) return IGA_ERR_ARG;
    iga_solve_opts o;
    iga_solve_opts_default(&o);
    if (o_in) o = *o_in;
    if (o.pc != IGA_PC_NONE && o.pc != IGA_PC_FEM_EXACT) {
        set_error("iga_dist_solve: pc is IGA_PC_NONE or IGA_PC_FEM_EXACT (the block FEM preconditioner)");
        return IGA_ERR_UNSUPPORTED;
    }
    DCUDA_TRY(cudaSetDevice(d->device));
    cudaStream_t st = (cudaStream_t)stream;
    const auto t0 = std::chrono::steady_clock::now();
    const long long n = d->nowned;
    double *p = d->p_local;   // owned part of the search direction's local form
    int e;
    zero_kernel<<<grid_for(n), 256, 0, st>>>(x, n);
    copy_kernel<<<grid_for(n), 256, 0, st>>>(d->r, b, n);
    if ((e = precond(d, o.pc, d->r, d->z, st))) return e;
    {
        const double *a[3] = {b, d->r, d->r}, *bb[3] = {b, d->r, d->z};
        if ((e = local_dots<3>(d, a, bb, 0, st)) || (e = allreduce(d, 3, st))) return e;
    }
    init_scalars_kernel<<<1, 1, 0, st>>>(d->s, o.rtol, o.max_it);
    copy_kernel<<<grid_for(n), 256, 0, st>>>(p, d->z, n);
    // Iterations run stream-ordered; the host reads the scalars every kChunk
    // iterations (kernels of iterations past convergence return at once).
    constexpr int kChunk = 8;
    int status = IGA_OK;
    for (int chunk = 0;; ++chunk) {
        for (int k = 0; k < kChunk; ++k) {
            if ((e = dist_matmult(d, p, p, d->q, st))) return e;
            {
                const double *a[1] = {p}, *bb[1] = {d->q};
                if ((e = local_dots<1>(d, a, bb, 0, st)) || (e = allreduce(d, 1, st))) return e;
            }
            alpha_kernel<<<1, 1, 0, st>>>(d->s);
            xr_kernel<<<grid_for(n), 256, 0, st>>>(x, d->r, p, d->q, n, d->s);
            {   // r . z_old before z is replaced
                const double *a[1] = {d->r}, *bb[1] = {d->z};
                if ((e = local_dots<1>(d, a, bb, 2, st))) return e;
            }
            if ((e = precond(d, o.pc, d->r, d->z, st))) return e;
            {
                const double *a[2] = {d->r, d->r}, *bb[2] = {d->r, d->z};
                if ((e = local_dots<2>(d, a, bb, 0, st)) || (e = allreduce(d, 3, st))) return e;
            }
            beta_kernel<<<1, 1, 0, st>>>(d->s);
            p_kernel<<<grid_for(n), 256, 0, st>>>(p, d->z, n, d->s);
        }
        DCUDA_TRY(cudaMemcpyAsync(d->h_s, d->s, sizeof(DistScalars), cudaMemcpyDeviceToHost, st));
        DCUDA_TRY(cudaStreamSynchronize(st));
        if (d->h_s->done) break;
    }
    const DistScalars hs = *d->h_s;
    if (hs.breakdown) status = IGA_ERR_BREAKDOWN;
    else if (!(hs.rr == hs.rr)) status = IGA_ERR_NONFINITE;
    else if (hs.it >= hs.maxit && hs.rr > hs.tol2) status = IGA_ERR_NOT_CONVERGED;
    // true residual ||b - K x|| / ||b||
    if ((e = dist_matmult(d, x, d->x_local, d->q, st))) return e;
    sub_kernel<<<grid_for(n), 256, 0, st>>>(d->r, b, d->q, n);
    {
        const double *a[2] = {d->r, b}, *bb[2] = {d->r, b};
        if ((e = local_dots<2>(d, a, bb, 0, st)) || (e = allreduce(d, 2, st))) return e;
    }
    DCUDA_TRY(cudaMemcpyAsync(d->h_s, d->s, sizeof(DistScalars), cudaMemcpyDeviceToHost, st));
    DCUDA_TRY(cudaStreamSynchronize(st));
    const double relres = d->h_s->red[1] > 0.0 ? std::sqrt(d->h_s->red[0] / d->h_s->red[1]) : 0.0;
    if (stats) {
        stats->status = status;
        stats->iterations = hs.it;
        stats->pc_iterations = 0;
        stats->sweeps = 0;
        stats->relres = relres;
        stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return status;
}

}  // extern "C"
