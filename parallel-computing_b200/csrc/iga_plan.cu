// Plans and the C ABI of the matrix-free operator (include/iga_mf.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <thread>
#include <vector>

#include "iga_apply.cuh"
#include "iga_host.hpp"
#include "iga_plan.hpp"

namespace iga {

// ---------------------------------------------------------------- setup kernels
// Precomputed geometry (the mult_sf path): G = w kappa det(J) J^-1 J^-T at
// every quadrature point, in the order apply_kernel streams it:
// [strip][row][qy][qx][3][column of the strip]. Padding elements get G = 0.
// Quadrature points (padding included) of a strip grid's G.
__host__ __device__ __forceinline__ long long geom_points(const StripGrid &g)
{
    return (long long)g.NSX * g.NSY * g.TY * (g.P + 1) * (g.P + 1) * kSW;
}

// G at point t of grid g, into G64 and / or G32 (either may be null).
__device__ __forceinline__ void geom_point(double *__restrict__ G64, float *__restrict__ G32,
                                           const double *__restrict__ tabX64, const double *__restrict__ tabY64,
                                           const double *__restrict__ CP, const double *__restrict__ qw,
                                           const double *__restrict__ kappa, const StripGrid &g, int *err, long long t)
{
    const int P = g.P, NB = P + 1, NQ = P + 1, NQ2 = NQ * NQ;
    {
        // Point u of the step block, in the order the block is stored, so that
        // consecutive threads write consecutive words: lane-major layouts
        // (g_lane_major) [qy][lane = 2c + h][j] (qx = h QH + j), else
        // [qy][qx][column]. (At p = 3 the column-fastest order scattered the
        // lane-major writes 12 words apart: 2048^2 G64 + G32 18.4 ms.)
        const int u = (int)(t % (NQ2 * kSW));
        long long r = t / (NQ2 * kSW);
        int c, qx, qy;
        if (g_lane_major(NQ)) {
            const int QH = NQ / 2;
            qy = u / (32 * QH);
            const int rem = u - qy * 32 * QH, lane = rem / QH, j = rem - lane * QH;
            c = lane >> 1;
            qx = (lane & 1) * QH + j;
        } else {
            c = u % kSW;
            const int qp = u / kSW;
            qx = qp % NQ;
            qy = qp / NQ;
        }
        const int qp = qy * NQ + qx;
        const int s = (int)(r % g.TY);
        r /= g.TY;
        const int gy = (int)(r % g.NSY);
        const int gx = (int)(r / g.NSY);
        const int ex = kSW * gx + c, ey = g.TY * gy + s;
        double g00 = 0, g01 = 0, g11 = 0;
        if (ex < g.nex && ey < g.ney) {
            double x_xi = 0, x_eta = 0, y_xi = 0, y_eta = 0;
            for (int jl = 0; jl < NB; ++jl) {
                const double n2 = tabY64[((size_t)(ey * 2 + 0) * NQ + qy) * NB + jl];
                const double d2 = tabY64[((size_t)(ey * 2 + 1) * NQ + qy) * NB + jl];
                for (int il = 0; il < NB; ++il) {
                    const double n1 = tabX64[((size_t)(ex * 2 + 0) * NQ + qx) * NB + il];
                    const double d1 = tabX64[((size_t)(ex * 2 + 1) * NQ + qx) * NB + il];
                    const size_t A = (size_t)(ey + jl) * g.m + (ex + il);
                    const double cx = CP[2 * A], cy = CP[2 * A + 1];
                    x_xi += cx * d1 * n2;
                    x_eta += cx * n1 * d2;
                    y_xi += cy * d1 * n2;
                    y_eta += cy * n1 * d2;
                }
            }
            const double det = x_xi * y_eta - x_eta * y_xi;
            if (!(det > 0.0)) atomicExch(err, 1 /* IGA_ERR_ARG: non-positive Jacobian */);
            double wgt = qw[qx] * qw[qy];
            if (kappa) wgt *= kappa[((size_t)ey * g.nex + ex) * NQ2 + qp];
            const double f = wgt / det;
            g00 = f * (x_eta * x_eta + y_eta * y_eta);
            g01 = -f * (x_xi * x_eta + y_xi * y_eta);
            g11 = f * (x_xi * x_xi + y_xi * y_xi);
        }
        const size_t base = (((size_t)gx * g.NSY + gy) * g.TY + s) * NQ2 * 3 * kSW;
        if (G64) {
            double *Gs = G64 + base;
            Gs[g_index(NQ, 8, qy, qx, 0, c)] = g00;
            Gs[g_index(NQ, 8, qy, qx, 1, c)] = g01;
            Gs[g_index(NQ, 8, qy, qx, 2, c)] = g11;
        }
        if (G32) {
            float *Gs = G32 + base;
            Gs[g_index(NQ, 4, qy, qx, 0, c)] = (float)g00;
            Gs[g_index(NQ, 4, qy, qx, 1, c)] = (float)g01;
            Gs[g_index(NQ, 4, qy, qx, 2, c)] = (float)g11;
        }
    }
}

template <typename T>
__global__ void geom_setup_kernel(T *__restrict__ G, const double *__restrict__ tabX64,
                                  const double *__restrict__ tabY64, const double *__restrict__ CP,
                                  const double *__restrict__ qw, const double *__restrict__ kappa, StripGrid g,
                                  int *err)
{
    const long long total = geom_points(g);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x)
        geom_point(sizeof(T) == 8 ? (double *)(void *)G : nullptr, sizeof(T) == 4 ? (float *)(void *)G : nullptr,
                   tabX64, tabY64, CP, qw, kappa, g, err, t);
}

// Every job of a batch's plans in one launch: the CTA finds the job of the
// first point of its 256-point block once (jobs hold at least 2 x 32 x 9 x
// 16 points, so a block straddles at most one boundary) and each thread
// steps to the next job if its point lies past that one's start.
__global__ void geom_jobs_kernel(const GeomJob *__restrict__ jobs, int njobs, long long total)
{
    __shared__ int js;
    for (long long b0 = (long long)blockIdx.x * blockDim.x; b0 < total; b0 += (long long)gridDim.x * blockDim.x) {
        if (threadIdx.x == 0) {
            int lo = 0, hi = njobs - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (jobs[mid].t0 <= b0) lo = mid;
                else hi = mid - 1;
            }
            js = lo;
        }
        __syncthreads();
        const long long t = b0 + threadIdx.x;
        int j = js;
        __syncthreads();
        if (t < total) {
            if (j + 1 < njobs && t >= jobs[j + 1].t0) ++j;
            const GeomJob &J = jobs[j];
            geom_point(J.G64, J.G32, J.tx, J.ty, J.cp, J.qw, J.kappa, J.g, J.err, t - J.t0);
        }
    }
}

__device__ double load_f(int fkind, double x, double y)
{
    const double pi = 3.141592653589793238462643383279;
    if (fkind == 0) return x * (1 - x) * y * (1 - y);
    if (fkind == 1) return 2.0 * pi * pi * sin(pi * x) * sin(pi * y);
    const double r = sqrt(x * x + y * y), th = atan2(y, x);
    return (pi * pi * sin(pi * r) - pi * cos(pi * r) / r + 4.0 * sin(pi * r) / (r * r)) * sin(2.0 * th);
}

// Load vector F = int R f (matrix_free/src/LocalAssemblyMF.cpp:3-29), gathered
// per control point over its supporting elements in a fixed order (the
// atomic-free scheme of matrix_free_gpu_dbd/src/mult.cu:233-340), F[Dir] = 0.
__global__ void rhs_kernel(double *__restrict__ F, const double *__restrict__ tabX64,
                           const double *__restrict__ tabY64, const double *__restrict__ CP,
                           const double *__restrict__ qw, int fkind, StripGrid g)
{
    const int P = g.P, NB = P + 1, NQ = P + 1;
    const long long N = (long long)g.m * g.n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int C = (int)(t % g.m), R = (int)(t / g.m);
        if (R == 0 || C == 0 || R == g.n - 1 || C == g.m - 1) {
            F[t] = 0.0;
            continue;
        }
        double v = 0.0;
        for (int ey = max(0, R - P); ey <= min(R, g.ney - 1); ++ey)
            for (int ex = max(0, C - P); ex <= min(C, g.nex - 1); ++ex) {
                const int il0 = C - ex, jl0 = R - ey;
                for (int qy = 0; qy < NQ; ++qy)
                    for (int qx = 0; qx < NQ; ++qx) {
                        double xq = 0, yq = 0, x_xi = 0, x_eta = 0, y_xi = 0, y_eta = 0;
                        for (int jl = 0; jl < NB; ++jl) {
                            const double n2 = tabY64[((size_t)(ey * 2 + 0) * NQ + qy) * NB + jl];
                            const double d2 = tabY64[((size_t)(ey * 2 + 1) * NQ + qy) * NB + jl];
                            for (int il = 0; il < NB; ++il) {
                                const double n1 = tabX64[((size_t)(ex * 2 + 0) * NQ + qx) * NB + il];
                                const double d1 = tabX64[((size_t)(ex * 2 + 1) * NQ + qx) * NB + il];
                                const size_t A = (size_t)(ey + jl) * g.m + (ex + il);
                                const double cx = CP[2 * A], cy = CP[2 * A + 1];
                                xq += cx * n1 * n2;
                                yq += cy * n1 * n2;
                                x_xi += cx * d1 * n2;
                                x_eta += cx * n1 * d2;
                                y_xi += cy * d1 * n2;
                                y_eta += cy * n1 * d2;
                            }
                        }
                        const double det = x_xi * y_eta - x_eta * y_xi;
                        const double Ra = tabX64[((size_t)(ex * 2) * NQ + qx) * NB + il0] *
                                          tabY64[((size_t)(ey * 2) * NQ + qy) * NB + jl0];
                        v += Ra * load_f(fkind, xq, yq) * qw[qx] * qw[qy] * det;
                    }
            }
        F[t] = v;
    }
}

// Checks the connectivity and equation numbers a reference-shaped call
// passes (device arrays, either may be null) against what this library's
// structured kernels compute: IEN must be the single-patch connectivity of
// matrix_free/src/IENGenerator.cpp:68-103 (element e = ey nex + ex, local
// function a = jl (p+1) + il at control point (ey + jl) m + ex + il); ID may
// be any map into [0, m n) that names no equation twice (negative: no row),
// and is flagged when it differs from the reference's serial numbering
// (matrix_free/src/Partition.cpp:102-108: -1 on the boundary ring, the
// control point's own index elsewhere). seen: (m n + 31) / 32 zeroed words.
__global__ void refentry_check_kernel(const int *__restrict__ IEN, const int *__restrict__ ID, int p, int nex,
                                      int ney, unsigned *__restrict__ seen, int *__restrict__ flags)
{
    const int NB = p + 1, m = nex + p, n = ney + p;
    const long long N = (long long)m * n, nien = IEN ? (long long)nex * ney * NB * NB : 0, nid = ID ? N : 0;
    const long long total = nien > nid ? nien : nid;
    int f = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        if (t < nien) {
            const long long e = t / (NB * NB);
            const int a = (int)(t - e * NB * NB);
            const int ex = (int)(e % nex), ey = (int)(e / nex);
            if (IEN[t] != (long long)(ey + a / NB) * m + ex + a % NB) f |= kCheckIEN;
        }
        if (t < nid) {
            const int e = ID[t];
            const int R = (int)(t / m), C = (int)(t % m);
            const bool ring = R == 0 || C == 0 || R == n - 1 || C == m - 1;
            if (ring ? e >= 0 : e != t) f |= kCheckIDOrder;
            if (e >= N) f |= kCheckIDRange;
            else if (e >= 0) {
                const unsigned bit = 1u << (e & 31);
                if (atomicOr(&seen[e >> 5], bit) & bit) f |= kCheckIDTwice;
            }
        }
    }
    if (f) atomicOr(flags, f);
}

int refentry_check(const int *IEN, const int *ID, int p, int nex, int ney, unsigned *seen, int *flags,
                   cudaStream_t s)
{
    const long long N = (long long)(nex + p) * (ney + p);
    if (cudaMemsetAsync(flags, 0, sizeof(int), s) != cudaSuccess) return IGA_ERR_CUDA;
    if (!IEN && !ID) return IGA_OK;
    if (ID && cudaMemsetAsync(seen, 0, (size_t)((N + 31) / 32) * sizeof(unsigned), s) != cudaSuccess)
        return IGA_ERR_CUDA;
    refentry_check_kernel<<<4 * 148, 256, 0, s>>>(IEN, ID, p, nex, ney, seen, flags);
    return cudaPeekAtLastError() == cudaSuccess ? IGA_OK : IGA_ERR_CUDA;
}

int refentry_status(int flags)
{
    if (flags & kCheckIEN) {
        set_error("d_IEN is not the structured single-patch connectivity (IENGenerator::GenerateIEN2D order)");
        return IGA_ERR_UNSUPPORTED;
    }
    if (flags & kCheckIDRange) {
        set_error("d_ID maps a control point to an equation number >= (nElemX+p)*(nElemY+q)");
        return IGA_ERR_UNSUPPORTED;
    }
    if (flags & kCheckIDTwice) {
        set_error("d_ID gives two control points the same equation number");
        return IGA_ERR_UNSUPPORTED;
    }
    return IGA_OK;
}

// ---------------------------------------------------------------- helpers
#define IGA_CUDA_TRY(call)                                  \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) {                            \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
            return e_ == cudaErrorMemoryAllocation ? IGA_ERR_NOMEM : IGA_ERR_CUDA; \
        }                                                   \
    } while (0)

static thread_local std::string g_last_error;
void set_error(const std::string &s) { g_last_error = s; }
const std::string &last_error() { return g_last_error; }

PlanArena *&plan_arena()
{
    static thread_local PlanArena *a = nullptr;
    return a;
}

cudaError_t PlanArena::alloc(void **p, size_t bytes)
{
    std::lock_guard<std::mutex> lock(mu);
    constexpr size_t kChunk = size_t(256) << 20;
    bytes = (bytes + 255) & ~size_t(255);
    if (chunks.empty() || used + bytes > chunks.back().second) {
        const size_t sz = std::max(kChunk, bytes);
        char *c = nullptr;
        const cudaError_t e = cudaMalloc((void **)&c, sz);
        if (e != cudaSuccess) return e;
        chunks.emplace_back(c, sz);
        used = 0;
    }
    *p = chunks.back().first + used;
    used += bytes;
    return cudaSuccess;
}

static size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

// The last chunk takes no more allocations; once its bytes are all written
// the copy thread (started with the first sealed chunk) sends it.
void PlanArena::seal_last(bool start_copier)
{
    if (dchunks.empty() || dchunks.back()->sealed) return;
    dchunks.back()->sealed = true;
    if (start_copier && !copier.joinable()) {
        int dev = 0;
        cudaGetDevice(&dev);
        copier = std::thread(&PlanArena::copy_loop, this, dev);
    }
    cv.notify_all();
}

void PlanArena::drop_copies(const void *lo, const void *hi)
{
    std::unique_lock<std::mutex> lk(mu);
    auto inside = [&](const void *p) { return p >= lo && p < hi; };
    direct.erase(std::remove_if(direct.begin(), direct.end(), [&](const DirectCopy &d) { return inside(d.src); }),
                 direct.end());
    cv.wait(lk, [&] { return !copying || !inside(copying); });
}

void PlanArena::defer_copy(void *dst, const void *src, size_t bytes)
{
    std::lock_guard<std::mutex> lock(mu);
    direct.push_back(DirectCopy{dst, src, bytes});
    if (!copier.joinable()) {
        int dev = 0;
        cudaGetDevice(&dev);
        copier = std::thread(&PlanArena::copy_loop, this, dev);
    }
    cv.notify_all();
}

void PlanArena::copy_loop(int device)
{
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        DataChunk *ready = nullptr;
        for (auto &c : dchunks)
            if (c->sealed && !c->taken && c->staged == c->used) {
                ready = c.get();
                break;
            }
        if (ready) {
            ready->taken = true;
            lk.unlock();
            const cudaError_t e =
                ready->used ? cudaMemcpy(ready->dev, ready->host.get(), ready->used, cudaMemcpyHostToDevice) : cudaSuccess;
            ready->host.reset();   // a copy from pageable memory has finished reading it on return
            lk.lock();
            if (e != cudaSuccess && copy_err == cudaSuccess) copy_err = e;
            continue;
        }
        if (!direct.empty()) {
            const DirectCopy d = direct.back();
            direct.pop_back();
            copying = d.src;
            lk.unlock();
            const cudaError_t e = cudaMemcpy(d.dst, d.src, d.bytes, cudaMemcpyHostToDevice);
            lk.lock();
            copying = nullptr;
            cv.notify_all();
            if (e != cudaSuccess && copy_err == cudaSuccess) copy_err = e;
            continue;
        }
        if (copier_stop) break;
        cv.wait(lk);
    }
}

void PlanArena::stop_copier()
{
    {
        std::lock_guard<std::mutex> lock(mu);
        copier_stop = true;
        cv.notify_all();
    }
    if (copier.joinable()) copier.join();
    copier_stop = false;
}

cudaError_t PlanArena::alloc_data(void **p, size_t bytes)
{
    std::lock_guard<std::mutex> lock(mu);
    constexpr size_t kChunk = size_t(16) << 20;
    bytes = round256(bytes);
    if (dchunks.empty() || dchunks.back()->used + bytes > dchunks.back()->size) {
        seal_last(true);
        auto c = std::make_unique<DataChunk>();
        c->size = std::max(kChunk, bytes);
        if (dblocks.empty() || dblock_used + c->size > dblocks.back().second) {   // device memory in 128 MB blocks
            const size_t sz = std::max(size_t(128) << 20, c->size);
            char *b = nullptr;
            const cudaError_t e = cudaMalloc((void **)&b, sz);
            if (e != cudaSuccess) return e;
            dblocks.emplace_back(b, sz);
            dblock_used = 0;
        }
        c->dev = dblocks.back().first + dblock_used;
        dblock_used += c->size;
        c->host.reset(new char[c->size]);   // uninitialised: only written bytes are touched
        dchunks.push_back(std::move(c));
    }
    DataChunk &c = *dchunks.back();
    *p = c.dev + c.used;
    c.used += bytes;
    return cudaSuccess;
}

void PlanArena::stage(void *dst, const void *src, size_t bytes)
{
    DataChunk *c = nullptr;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (size_t k = dchunks.size(); k-- > 0;) {
            DataChunk *d = dchunks[k].get();
            if ((char *)dst >= d->dev && (char *)dst < d->dev + d->size) {
                c = d;
                break;
            }
        }
    }
    if (!c) return;
    std::memcpy(c->host.get() + ((char *)dst - c->dev), src, bytes);   // disjoint ranges: no lock needed
    std::lock_guard<std::mutex> lock(mu);
    c->staged += round256(bytes);
    if (c->sealed && c->staged == c->used) cv.notify_all();
}

static bool same_grid(const StripGrid &a, const StripGrid &b)
{
    return a.m == b.m && a.n == b.n && a.nex == b.nex && a.ney == b.ney && a.TY == b.TY && a.NSX == b.NSX &&
           a.NSY == b.NSY && a.P == b.P;
}

void PlanArena::defer_geom(const GeomJob &j)
{
    std::lock_guard<std::mutex> lock(mu);
    for (size_t k = geom.size(); k-- > 0;) {   // the plan's other precision, added just before by the same thread
        GeomJob &o = geom[k];
        if (o.cp == j.cp && o.tx == j.tx && o.kappa == j.kappa && same_grid(o.g, j.g) && !(o.G64 && j.G64) &&
            !(o.G32 && j.G32)) {
            if (j.G64) o.G64 = j.G64;
            if (j.G32) o.G32 = j.G32;
            return;
        }
    }
    geom.push_back(j);
}

cudaError_t PlanArena::flush()
{
    {
        std::lock_guard<std::mutex> lock(mu);
        seal_last(false);
    }
    stop_copier();   // it sends every complete chunk and queued copy before it stops
    for (auto &c : dchunks)   // chunks no copy thread took (a single one, or none started)
        if (!c->taken) {
            c->taken = true;
            const cudaError_t e = c->used ? cudaMemcpy(c->dev, c->host.get(), c->used, cudaMemcpyHostToDevice) : cudaSuccess;
            if (e != cudaSuccess && copy_err == cudaSuccess) copy_err = e;
        }
    if (copy_err != cudaSuccess) {
        const cudaError_t e = copy_err;
        copy_err = cudaSuccess;
        return e;
    }
    // the remaining host shadows are released by a thread of their own
    // (unmapping them takes milliseconds the caller need not wait for)
    {
        std::vector<std::unique_ptr<char[]>> sh;
        for (auto &c : dchunks)
            if (c->host) sh.push_back(std::move(c->host));
        if (!sh.empty()) std::thread([sh = std::move(sh)]() mutable { sh.clear(); }).detach();
    }
    if (!geom.empty()) {
        long long t = 0;
        for (GeomJob &j : geom) {
            j.t0 = t;
            t += geom_points(j.g);
        }
        GeomJob *dj = nullptr;
        cudaError_t e = alloc((void **)&dj, geom.size() * sizeof(GeomJob));
        if (e == cudaSuccess) e = cudaMemcpy(dj, geom.data(), geom.size() * sizeof(GeomJob), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        int nsm = 148, dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            nsm = 148;
        const long long blocks = std::min<long long>((t + 255) / 256, 8LL * nsm);
        geom_jobs_kernel<<<(unsigned)blocks, 256>>>(dj, (int)geom.size(), t);
        geom.clear();
    }
    return cudaGetLastError();
}

bool PlanArena::owns(const void *p) const
{
    std::lock_guard<std::mutex> lock(mu);
    for (const auto &c : chunks)
        if (p >= (const void *)c.first && p < (const void *)(c.first + c.second)) return true;
    for (const auto &c : dblocks)
        if (p >= (const void *)c.first && p < (const void *)(c.first + c.second)) return true;
    return false;
}

void PlanArena::release()
{
    stop_copier();
    direct.clear();
    for (auto &c : chunks) cudaFree(c.first);
    for (auto &c : dblocks) cudaFree(c.first);
    chunks.clear();
    dchunks.clear();
    dblocks.clear();
    dblock_used = 0;
    geom.clear();
    used = 0;
}

template <typename T>
static int upload(T **dst, const void *src, size_t bytes)
{
    PlanArena *a = plan_arena();
    if (a && a->defer && src && bytes) {   // copied by the arena's flush
        IGA_CUDA_TRY(a->alloc_data((void **)dst, bytes));
        a->stage(*dst, src, bytes);
        return IGA_OK;
    }
    if (a) IGA_CUDA_TRY(a->alloc((void **)dst, std::max<size_t>(bytes, 16)));
    else IGA_CUDA_TRY(cudaMalloc((void **)dst, std::max<size_t>(bytes, 16)));
    if (src && bytes) IGA_CUDA_TRY(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    return IGA_OK;
}

// Like upload() for host data that lives as long as the plan (its patch):
// in deferred mode the arena's copy thread copies it straight from there.
template <typename T>
static int upload_persistent(T **dst, const void *src, size_t bytes)
{
    PlanArena *a = plan_arena();
    if (a && a->defer && src && bytes) {
        IGA_CUDA_TRY(a->alloc((void **)dst, bytes));
        a->defer_copy(*dst, src, bytes);
        return IGA_OK;
    }
    return upload(dst, src, bytes);
}

// cudaFree unless the buffer belongs to the plan's arena.
static void plan_free(const iga_plan *pl, void *p)
{
    if (p && !(pl->arena && pl->arena->owns(p))) cudaFree(p);
}

static constexpr size_t kSmemBudget = 220 * 1024;

// Warps per CTA: as many as the shared memory and the kernel's register budget allow.
template <int P, typename T, int GEOM>
static int warps_for_t()
{
    constexpr int NST = apply_stages<P, T>();
    for (int W = apply_max_threads<P, T, GEOM>() / 32; W >= 1; --W)
        if (apply_smem_bytes<P, T, GEOM, NST>(W, 2) <= kSmemBudget) return W;
    return 1;
}

template <typename T, int GEOM>
static int warps_for_g(int P)
{
    switch (P) {
    case 1: return warps_for_t<1, T, GEOM>();
    case 2: return warps_for_t<2, T, GEOM>();
    case 3: return warps_for_t<3, T, GEOM>();
    case 4: return warps_for_t<4, T, GEOM>();
    default: return warps_for_t<5, T, GEOM>();
    }
}

int warps_for(int P, int prec, int geom)
{
    if (prec == IGA_FP64) return geom ? warps_for_g<double, 1>(P) : warps_for_g<double, 0>(P);
    return geom ? warps_for_g<float, 1>(P) : warps_for_g<float, 0>(P);
}

// Rows per strip: the candidate whose CTA count fills the SMs best, with a
// small penalty on short strips (more seam traffic). A MIXED plan launches
// its FP64 and FP32 operators with different warps per CTA on the same
// strips: each precision's cost is taken relative to its own best and the
// candidate with the smallest sum wins. flat: the kernel deals strips to warps
// one by one (apply_txreg), else a CTA covers W strips of one column.
struct WarpShape {
    int W;
    bool flat;
    // also try the strip heights whose CTA count fills whole waves of SMs:
    // the kernels with shared x tables dealt from a flat grid (FP64
    // precomputed p >= 4, FP64 on-the-fly p = 1, 2), which are held back by
    // each SM's own progress rather than by HBM (p=4 1024^2: 57 rows, 144
    // CTAs, 146.4 -> 140.3 us; p=5: 38 rows, 238 -> 230 us; on-the-fly p=2
    // 1024^2 105.5 -> 101.4 us, p=1 50.1 -> 48.1 us), where the p=3 headline
    // at 82% of HBM gained nothing from it (40 or 50 rows: 312 / 314 us)
    bool waves = false;
};

static double strip_cost(int NSX, int ney, int TY, WarpShape ws, int nsm)
{
    const int NSY = (ney + TY - 1) / TY, W = ws.W;
    const long long ctas = ws.flat ? ((long long)NSX * NSY + W - 1) / W : (long long)NSX * ((NSY + W - 1) / W);
    const long long waves = (ctas + nsm - 1) / nsm;
    const double work = (double)waves * W * (TY + 2.0);   // per-SM time in strip-row units
    return work * (1.0 + 0.5 * 3.0 / TY);
}

static int rows_for(int nex, int ney, const std::vector<WarpShape> &Ws, int nsm)
{
    const int NSX = (nex + kSW - 1) / kSW;
    std::vector<int> cands = {64, 56, 48, 40, 32, 28, 24, 20, 16};
    for (const WarpShape &ws : Ws)
        if (ws.waves && ws.flat)
            for (int k = 1; k <= 16; ++k) {
                const long long nsy = (long long)k * nsm * ws.W / NSX;   // strip rows of k full waves
                if (nsy < 1) continue;
                const int TY = (int)((ney + nsy - 1) / nsy);
                if (TY >= 16 && TY <= 64 && std::find(cands.begin(), cands.end(), TY) == cands.end()) cands.push_back(TY);
            }
    std::vector<double> best_w(Ws.size(), 1e300);
    for (size_t k = 0; k < Ws.size(); ++k)
        for (int TY : cands) best_w[k] = std::min(best_w[k], strip_cost(NSX, ney, TY, Ws[k], nsm));
    int best = 64;
    double best_cost = 1e300;
    for (int TY : cands) {
        double c = 0.0;
        for (size_t k = 0; k < Ws.size(); ++k) c += strip_cost(NSX, ney, TY, Ws[k], nsm) / best_w[k];
        if (c < best_cost - 1e-9) {
            best_cost = c;
            best = TY;
        }
    }
    return best;
}

// The single-plan kernel deals strips to warps one by one in every
// configuration (shared x tables included) but the FP64 on-the-fly p = 5
// one (apply_percolumn).
static bool apply_flat(int P, int prec, int geom) { return !(P == 5 && prec == IGA_FP64 && geom == IGA_GEOM_ON_THE_FLY); }

}  // namespace iga

using namespace iga;

// ---------------------------------------------------------------- plan
template <typename T>
static int build_operator(iga_plan *pl, OperatorData &op, const Patch &P, const Tables1D &tx, const Tables1D &ty)
{
    const int p = P.p, NB = p + 1, NQ = p + 1, NQ2 = NQ * NQ;
    const StripGrid &g = op.grid;
    // x tables regrouped per column strip: [gx][kind][j][il][lane], lane = 2c + h
    // holding element column 16 gx + c at quadrature column lane_qx(NQ, sizeof(T), h, j).
    const int QH = (NQ + 1) / 2;
    std::vector<T> hx((size_t)g.NSX * 2 * QH * NB * 32, T(0));
    for (int gx = 0; gx < g.NSX; ++gx)
        for (int kind = 0; kind < 2; ++kind)
            for (int j = 0; j < QH; ++j)
                for (int il = 0; il < NB; ++il)
                    for (int lane = 0; lane < 32; ++lane) {
                        const int ex = kSW * gx + lane / 2, qx = lane_qx(NQ, (int)sizeof(T), lane % 2, j);
                        double v = 0.0;
                        if (ex < P.nex && qx < NQ) v = (kind ? tx.der : tx.val)[((size_t)ex * NQ + qx) * NB + il];
                        hx[((((size_t)gx * 2 + kind) * QH + j) * NB + il) * 32 + lane] = (T)v;
                    }
    const int TYW = tab_row_len(NB, NQ, (int)sizeof(T));   // rows padded to 16 bytes
    std::vector<T> hy((size_t)P.ney * TYW, T(0));
    for (int ey = 0; ey < P.ney; ++ey)
        for (int kind = 0; kind < 2; ++kind)
            for (int qy = 0; qy < NQ; ++qy)
                for (int jl = 0; jl < NB; ++jl)
                    hy[(size_t)ey * TYW + tab_y_index(NB, NQ, (int)sizeof(T), kind, qy, jl)] =
                        (T)(kind ? ty.der : ty.val)[((size_t)ey * NQ + qy) * NB + jl];
    int st;
    if ((st = upload((T **)&op.tabX, hx.data(), hx.size() * sizeof(T)))) return st;
    if ((st = upload((T **)&op.tabY, hy.data(), hy.size() * sizeof(T)))) return st;
    std::vector<T> hw(NQ2);
    std::vector<double> qx(NQ), qw(NQ);
    gauss01(NQ, qx.data(), qw.data());
    for (int a = 0; a < NQ; ++a)
        for (int b = 0; b < NQ; ++b) hw[a * NQ + b] = (T)(qw[a] * qw[b]);
    if ((st = upload((T **)&op.wq, hw.data(), hw.size() * sizeof(T)))) return st;
    if (pl->geometry == IGA_GEOM_ON_THE_FLY) {
        if (!P.kappa.empty()) {
            std::vector<T> hk(P.kappa.begin(), P.kappa.end());
            if ((st = upload((T **)&op.kappa, hk.data(), hk.size() * sizeof(T)))) return st;
        }
        std::vector<T> hc(P.CP.begin(), P.CP.end());
        if ((st = upload((T **)&op.CP, hc.data(), hc.size() * sizeof(T)))) return st;
    }
    size_t fbytes = (size_t)g.NSX * g.NSY * g.FS * sizeof(T);
    if ((st = upload((T **)&op.frame, nullptr, fbytes))) return st;
    if (pl->geometry == IGA_GEOM_PRECOMPUTED) {
        const size_t gelems = (size_t)g.NSX * g.NSY * g.TY * NQ2 * 3 * kSW;
        op.geom_bytes = gelems * sizeof(T);
        if ((st = upload((T **)&op.G, nullptr, op.geom_bytes))) return st;
        if (pl->arena && pl->arena->defer) {   // after the arena's flush has sent the tables
            GeomJob j;
            if (sizeof(T) == 8) j.G64 = (double *)op.G;
            else j.G32 = (float *)op.G;
            j.tx = pl->tabX64;
            j.ty = pl->tabY64;
            j.cp = pl->CP;
            j.qw = pl->qw;
            j.kappa = pl->kappa_dev;
            j.g = g;
            j.err = pl->d_err;
            pl->arena->defer_geom(j);
            op.ready = true;
            return IGA_OK;
        }
        geom_setup_kernel<T><<<1184, 256>>>((T *)op.G, pl->tabX64, pl->tabY64, pl->CP, pl->qw, pl->kappa_dev, g,
                                            pl->d_err);
        // in an arena (a batch's set-up) the caller synchronises once for all plans
        cudaError_t e = pl->arena ? cudaPeekAtLastError() : cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            set_error(std::string("geometry setup: ") + cudaGetErrorString(e));
            return IGA_ERR_CUDA;
        }
    }
    op.ready = true;
    return IGA_OK;
}

// Win: a window of strip rows (gyn >= 0: strip rows gy0 .. gy0 + gyn - 1, and
// the seams of control-point rows R0 .. R1 - 1 instead of all seams); ID:
// equation numbers of the rows (ApplyParams::ID), null for the natural order.
struct Win {
    int gy0 = 0, gyn = -1, R0 = 0, R1 = 0;
    const int *ID = nullptr;
};

template <int P, typename T, int GEOM, int NST>
static int launch_apply_t(iga_plan *pl, const OperatorData &op, const T *x, T *y, cudaStream_t s, int sign, int bc,
                          Win win = Win())
{
    ApplyParams<T> a;
    a.x = x;
    a.y = y;
    a.G = (const T *)op.G;
    a.tabX = (const T *)op.tabX;
    a.tabY = (const T *)op.tabY;
    a.CP = (const T *)op.CP;
    a.wq = (const T *)op.wq;
    a.kappa = (const T *)op.kappa;
    a.frame = (T *)op.frame;
    a.g = op.grid;
    a.sign = (T)sign;
    a.bc = bc;
    a.err = pl->d_err;
    a.ID = win.ID;
    if (pl->wait_polls >= 0) a.wait_polls = pl->wait_polls;
    auto kern = apply_kernel<P, T, GEOM, NST>;
    static bool attr_set = false;   // per template instance: the most any launch below asks for
    if (!attr_set) {
        IGA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)apply_smem_bytes<P, T, GEOM, NST>(op.warps, 2)));
        attr_set = true;
    }
    const StripGrid &g = op.grid;
    const int rows = win.gyn >= 0 ? std::min(win.gyn, g.NSY - win.gy0) : g.NSY;
    // shared x tables: a CTA's strips lie in at most two column strips when
    // W - 1 <= rows, in one when W divides rows (one slot: the shared memory
    // of the one-column layout, which matters where a kernel's spills live
    // in L1: FP64 on-the-fly p=5 512^2 189 -> 257 us with a second slot)
    constexpr bool percol = apply_percolumn<P, T, GEOM>();
    const int W = apply_txshared<P, T, GEOM>() && !percol ? std::max(1, std::min(op.warps, rows + 1)) : op.warps;
    const size_t smem = apply_smem_bytes<P, T, GEOM, NST>(W, !percol && rows % W ? 2 : 1);
    if (win.gyn >= 0) {
        a.gy0 = win.gy0;
        a.gyn = rows;
    }
    const long long nstrips = (long long)g.NSX * rows;
    const dim3 grid = percol ? dim3(g.NSX, (rows + W - 1) / W) : dim3((unsigned)((nstrips + W - 1) / W));
    dim3 block(32, W);
    if (rows > 0) IGA_CUDA_TRY(launch_k(kern, grid, block, smem, s, a));
    if (win.gyn < 0) {
        const long long nseam = (long long)(g.NSX - 1) * P * g.n + (long long)(g.NSY - 1) * P * g.m;
        if (nseam > 0) {
            // about one seam point per thread, so that the points' frame loads
            // (L2 hits) are all in flight at once (p=3 2048^2 FP64 MatMult:
            // 309.5 us with 7 points per thread, 306 us with one)
            const int blocks = (int)std::min<long long>((nseam + 255) / 256, 32 * 148);
            IGA_CUDA_TRY(launch_k(seam_fixup_kernel<P, T>, dim3(blocks), dim3(256), 0, s, (const T *)op.frame, x, y,
                                  g, (T)sign, bc, win.ID));
        }
    } else if (win.R1 > win.R0) {
        const long long nseam = (long long)(g.NSX - 1) * P * (win.R1 - win.R0) + (long long)2 * P * g.m * (rows + 1);
        const int blocks = (int)std::max<long long>(1, std::min<long long>((nseam + 255) / 256, 4 * 148));
        seam_fixup_rows_kernel<P, T><<<blocks, 256, 0, s>>>((const T *)op.frame, x, y, g, (T)sign, bc, win.R0,
                                                             win.R1, win.ID);
    }
    IGA_CUDA_TRY(cudaGetLastError());
    return IGA_OK;
}

template <int P, typename T>
static int launch_apply_p(iga_plan *pl, const OperatorData &op, const T *x, T *y, cudaStream_t s, int sign, int bc,
                          Win win = Win())
{
    constexpr int NST = apply_stages<P, T>();
    if (pl->geometry == IGA_GEOM_PRECOMPUTED) return launch_apply_t<P, T, 0, NST>(pl, op, x, y, s, sign, bc, win);
    return launch_apply_t<P, T, 1, NST>(pl, op, x, y, s, sign, bc, win);
}

template <typename T>
static int launch_apply(iga_plan *pl, const OperatorData &op, const T *x, T *y, cudaStream_t s, int sign, int bc,
                        Win win = Win())
{
    switch (pl->p) {
    case 1: return launch_apply_p<1, T>(pl, op, x, y, s, sign, bc, win);
    case 2: return launch_apply_p<2, T>(pl, op, x, y, s, sign, bc, win);
    case 3: return launch_apply_p<3, T>(pl, op, x, y, s, sign, bc, win);
    case 4: return launch_apply_p<4, T>(pl, op, x, y, s, sign, bc, win);
    case 5: return launch_apply_p<5, T>(pl, op, x, y, s, sign, bc, win);
    default: return IGA_ERR_UNSUPPORTED;
    }
}

int iga_apply_internal_sb(iga_plan *pl, int prec, const void *x, void *y, cudaStream_t s, int sign, int bc)
{
    if (prec == IGA_FP64) {
        if (!pl->op64.ready) return IGA_ERR_ARG;
        return launch_apply<double>(pl, pl->op64, (const double *)x, (double *)y, s, sign, bc);
    }
    if (!pl->op32.ready) return IGA_ERR_ARG;
    return launch_apply<float>(pl, pl->op32, (const float *)x, (float *)y, s, sign, bc);
}

int iga_apply_internal(iga_plan *pl, int prec, const void *x, void *y, cudaStream_t s)
{
    if (pl->eq_id) {   // rows in the caller's equation numbering (reference-shaped entry)
        if (prec != IGA_FP64 || !pl->op64.ready) return IGA_ERR_ARG;
        Win w;
        w.ID = pl->eq_id;
        return launch_apply<double>(pl, pl->op64, (const double *)x, (double *)y, s, pl->sign, IGA_BC_NONE, w);
    }
    return iga_apply_internal_sb(pl, prec, x, y, s, pl->sign, pl->bc);
}

int iga_check_error_flag(iga_plan *pl)
{
    int h = 0;
    IGA_CUDA_TRY(cudaMemcpy(&h, pl->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        cudaMemset(pl->d_err, 0, sizeof(int));
        return h;
    }
    return IGA_OK;
}

template <typename T>
__global__ void kappa_convert_kernel(T *__restrict__ dst, const double *__restrict__ src, long long n)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        dst[t] = (T)src[t];
}

static void free_op(const iga_plan *pl, OperatorData &op)
{
    for (void *p : {op.tabX, op.tabY, op.G, op.frame, op.wq, op.kappa, op.CP}) plan_free(pl, p);
    op = OperatorData{};
}

extern "C" {

void iga_opts_default(iga_opts *o)
{
    if (!o) return;
    o->precision = IGA_FP64;
    o->geometry = IGA_GEOM_PRECOMPUTED;
    o->sign = IGA_SIGN_REFERENCE;
    o->bc = IGA_BC_REFERENCE;
    o->device = 0;
    o->rows_per_strip = 0;
}

const char *iga_status_str(int s)
{
    switch (s) {
    case IGA_OK: return "ok";
    case IGA_ERR_ARG: return "invalid argument";
    case IGA_ERR_UNSUPPORTED: return "unsupported input";
    case IGA_ERR_CUDA: return "CUDA error";
    case IGA_ERR_NOMEM: return "out of device memory";
    case IGA_ERR_NOT_CONVERGED: return "not converged";
    case IGA_ERR_BREAKDOWN: return "Krylov breakdown";
    case IGA_ERR_NONFINITE: return "non-finite value";
    case IGA_ERR_TIMEOUT: return "bounded device wait timed out";
    default: return "unknown status";
    }
}

const char *iga_last_error(void) { return last_error().c_str(); }

int iga_mesh_unit_square(int p, int nex, int ney, double Lx, double Ly, double *CP, double *C1, double *C2)
{
    if (p < 1 || p > 8 || nex < 1 || ney < 1 || !CP || !C1 || !C2 || !(Lx > 0) || !(Ly > 0)) return IGA_ERR_ARG;
    const std::vector<double> S = open_knots(p, nex, Lx), T = open_knots(p, ney, Ly);
    const std::vector<double> gx = greville(p, S), gy = greville(p, T);
    const std::vector<double> c1 = extraction(p, S), c2 = extraction(p, T);
    const int m = nex + p, n = ney + p;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            CP[2 * ((size_t)j * m + i)] = gx[i];
            CP[2 * ((size_t)j * m + i) + 1] = gy[j];
        }
    std::memcpy(C1, c1.data(), c1.size() * sizeof(double));
    std::memcpy(C2, c2.data(), c2.size() * sizeof(double));
    return IGA_OK;
}

int iga_mesh_quarter_annulus(int p, int nex, int ney, double r_in, double r_out, double *CP, double *W, double *C1,
                             double *C2)
{
    if (p < 2 || p > 8 || nex < 1 || ney < 1 || !CP || !W || !C1 || !C2 || !(r_in > 0) || !(r_out > r_in))
        return IGA_ERR_ARG;
    std::vector<double> cp, w, c1, c2;
    quarter_annulus(p, nex, ney, r_in, r_out, cp, w, c1, c2);
    std::memcpy(CP, cp.data(), cp.size() * sizeof(double));
    std::memcpy(W, w.data(), w.size() * sizeof(double));
    std::memcpy(C1, c1.data(), c1.size() * sizeof(double));
    std::memcpy(C2, c2.data(), c2.size() * sizeof(double));
    return IGA_OK;
}

int iga_plan_create(const iga_mesh_desc *d, const iga_opts *opts_in, iga_plan **out)
{
    if (!d || !out) return IGA_ERR_ARG;
    *out = nullptr;
    iga_opts opts;
    iga_opts_default(&opts);
    if (opts_in) opts = *opts_in;
    if (opts.precision < IGA_FP64 || opts.precision > IGA_MIXED) return IGA_ERR_ARG;
    if (opts.geometry != IGA_GEOM_PRECOMPUTED && opts.geometry != IGA_GEOM_ON_THE_FLY) return IGA_ERR_ARG;
    if (opts.sign != IGA_SIGN_REFERENCE && opts.sign != IGA_SIGN_SPD) return IGA_ERR_ARG;
    if (opts.bc != IGA_BC_REFERENCE && opts.bc != IGA_BC_IDENTITY && opts.bc != IGA_BC_NONE) return IGA_ERR_ARG;
    Patch Pb;
    MeshDescView v{d->p, d->q, d->nElemX, d->nElemY, d->CP, d->weights, d->C1, d->C2, d->IEN, d->ID, d->Dir,
                   d->nDir, d->kappa};
    std::string err = build_patch(v, Pb);
    if (!err.empty()) {
        set_error(err);
        return (err.find("requires") != std::string::npos || err.find("must be in") != std::string::npos)
                   ? IGA_ERR_UNSUPPORTED
                   : IGA_ERR_ARG;
    }
    IGA_CUDA_TRY(cudaSetDevice(opts.device));
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, opts.device);

    iga_plan *pl = new iga_plan();
    pl->patch = std::move(Pb);   // the plan keeps the patch; no copy of its control points
    const Patch &P = pl->patch;
    pl->p = P.p;
    pl->nex = P.nex;
    pl->ney = P.ney;
    pl->m = P.m;
    pl->n = P.n;
    pl->nfunc = (long long)P.m * P.n;
    pl->precision = opts.precision;
    pl->geometry = opts.geometry;
    pl->sign = opts.sign;
    pl->bc = opts.bc;
    pl->device = opts.device;
    pl->arena = plan_arena();
    // Rows per strip, per operator: a MIXED plan's FP64 and FP32 operators
    // have their own G layouts, so each gets the strip height that fills the
    // SMs best with its own warps per CTA (or the caller's rows_per_strip).
    auto rows_of = [&](int prec) {
        if (opts.rows_per_strip > 0) return opts.rows_per_strip;
        const bool shared_flat = prec == IGA_FP64 && (opts.geometry == IGA_GEOM_PRECOMPUTED ? P.p >= 4 : P.p <= 2);
        return rows_for(P.nex, P.ney, {{warps_for(P.p, prec, opts.geometry), apply_flat(P.p, prec, opts.geometry),
                                         shared_flat}},
                        nsm);
    };
    auto make_grid = [&](int TY) {
        StripGrid g;
        g.m = P.m;
        g.n = P.n;
        g.nex = P.nex;
        g.ney = P.ney;
        g.TY = TY;
        g.NSX = (P.nex + kSW - 1) / kSW;
        g.NSY = (P.ney + TY - 1) / TY;
        g.P = P.p;
        g.FS = frame_size(P.p, TY);
        return g;
    };
    const int TY64 = opts.precision != IGA_FP32 ? rows_of(IGA_FP64) : 0;
    const int TY32 = opts.precision != IGA_FP64 ? rows_of(IGA_FP32) : 0;
    for (int TY : {TY64, TY32})
        if (TY != 0 && (TY < P.p || TY > 1024)) {
            delete pl;
            set_error("rows_per_strip must be in [p, 1024]");
            return IGA_ERR_ARG;
        }
    if (TY64) pl->op64.grid = make_grid(TY64);
    if (TY32) pl->op32.grid = make_grid(TY32);
    pl->grid = TY64 ? pl->op64.grid : pl->op32.grid;   // sizes for the operator-independent kernels

    int st = IGA_OK;
    auto fail = [&](int code) {
        iga_plan_destroy(pl);
        return code;
    };
    const Tables1D tx = tables_1d(P.p, P.nex, P.C1.data(), P.w1.empty() ? nullptr : P.w1.data());
    const Tables1D ty = tables_1d(P.q, P.ney, P.C2.data(), P.w2.empty() ? nullptr : P.w2.data());
    {
        const int NB = P.p + 1, NQ = NB;
        std::vector<double> h64x((size_t)P.nex * 2 * NQ * NB), h64y((size_t)P.ney * 2 * NQ * NB);
        for (int e = 0; e < P.nex; ++e)
            for (int k = 0; k < NQ * NB; ++k) {
                h64x[((size_t)e * 2 + 0) * NQ * NB + k] = tx.val[(size_t)e * NQ * NB + k];
                h64x[((size_t)e * 2 + 1) * NQ * NB + k] = tx.der[(size_t)e * NQ * NB + k];
            }
        for (int e = 0; e < P.ney; ++e)
            for (int k = 0; k < NQ * NB; ++k) {
                h64y[((size_t)e * 2 + 0) * NQ * NB + k] = ty.val[(size_t)e * NQ * NB + k];
                h64y[((size_t)e * 2 + 1) * NQ * NB + k] = ty.der[(size_t)e * NQ * NB + k];
            }
        std::vector<double> qx(NQ), qw(NQ);
        gauss01(NQ, qx.data(), qw.data());
        if ((st = upload(&pl->tabX64, h64x.data(), h64x.size() * 8))) return fail(st);
        if ((st = upload(&pl->tabY64, h64y.data(), h64y.size() * 8))) return fail(st);
        if ((st = upload_persistent(&pl->CP, P.CP.data(), P.CP.size() * 8))) return fail(st);
        if ((st = upload(&pl->qw, qw.data(), qw.size() * 8))) return fail(st);
        const int zero = 0;
        if (pl->arena && pl->arena->defer) {
            if ((st = upload(&pl->d_err, &zero, sizeof(int)))) return fail(st);
        } else {
            if ((st = upload(&pl->d_err, nullptr, sizeof(int)))) return fail(st);
            cudaMemset(pl->d_err, 0, sizeof(int));
        }
        if (!P.kappa.empty()) {
            if ((st = upload(&pl->kappa_dev, P.kappa.data(), P.kappa.size() * 8))) return fail(st);
            pl->kappa_version = 1;
        }
    }
    if (opts.precision != IGA_FP32) {
        pl->op64.warps = warps_for(P.p, IGA_FP64, opts.geometry);
        if ((st = build_operator<double>(pl, pl->op64, P, tx, ty))) return fail(st);
    }
    if (opts.precision != IGA_FP64) {
        pl->op32.warps = warps_for(P.p, IGA_FP32, opts.geometry);
        if ((st = build_operator<float>(pl, pl->op32, P, tx, ty))) return fail(st);
    }
    int herr = 0;
    if (!pl->arena) cudaMemcpy(&herr, pl->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (herr) {
        set_error("geometry has a non-positive Jacobian determinant");
        return fail(IGA_ERR_ARG);
    }
    *out = pl;
    return IGA_OK;
}

int iga_plan_destroy(iga_plan *pl)
{
    if (!pl) return IGA_OK;
    if (pl->arena && !pl->patch.CP.empty())   // a copy thread may still read the control points
        pl->arena->drop_copies(pl->patch.CP.data(), pl->patch.CP.data() + pl->patch.CP.size());
    cudaSetDevice(pl->device);
    cudaDeviceSynchronize();
    free_op(pl, pl->op64);
    free_op(pl, pl->op32);
    for (void *p : {(void *)pl->tabX64, (void *)pl->tabY64, (void *)pl->CP, (void *)pl->qw, (void *)pl->d_err,
                    (void *)pl->kappa_dev, (void *)pl->eq_id,
                    (void *)pl->h_stage_x, (void *)pl->d_stage_x, (void *)pl->d_stage_y})
        plan_free(pl, p);
    if (pl->h_pinned) cudaFreeHost(pl->h_pinned);
    for (cudaStream_t hs : pl->host_st)
        if (hs) cudaStreamDestroy(hs);
    for (auto &row : pl->host_ev)
        for (cudaEvent_t e : row)
            if (e) cudaEventDestroy(e);
    if (pl->host_ev0) cudaEventDestroy(pl->host_ev0);
    iga_solver_release(pl);
    delete pl;
    return IGA_OK;
}

int iga_plan_get_info(const iga_plan *pl, iga_plan_info *info)
{
    if (!pl || !info) return IGA_ERR_ARG;
    info->nfunc = pl->nfunc;
    info->nelem = (long long)pl->nex * pl->ney;
    const int NQ2 = (pl->p + 1) * (pl->p + 1);
    info->geom_bytes = pl->op64.ready ? pl->op64.geom_bytes : pl->op32.geom_bytes;
    // Algorithmic bytes: read x, write y, plus geometry (3 values per
    // quadrature point precomputed, or control points + 1-D tables on the fly).
    for (int k = 0; k < 2; ++k) {
        const long long s = k == 0 ? 8 : 4;
        long long b = 2 * s * pl->nfunc;
        if (pl->geometry == IGA_GEOM_PRECOMPUTED) b += 3 * s * NQ2 * info->nelem;
        else b += 16LL * pl->nfunc + 8LL * 2 * NQ2 * (pl->nex + pl->ney);
        (k == 0 ? info->algo_bytes_f64 : info->algo_bytes_f32) = b;
    }
    info->rows_per_strip = pl->grid.TY;
    info->warps_per_cta = pl->op64.ready ? pl->op64.warps : pl->op32.warps;
    return IGA_OK;
}

int iga_plan_set_kappa(iga_plan *pl, const double *kappa, void *stream)
{
    if (!pl || !kappa) return IGA_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const long long nq = (long long)pl->nex * pl->ney * (pl->p + 1) * (pl->p + 1);
    if (!pl->kappa_dev) IGA_CUDA_TRY(cudaMalloc((void **)&pl->kappa_dev, nq * sizeof(double)));
    IGA_CUDA_TRY(cudaMemcpyAsync(pl->kappa_dev, kappa, nq * sizeof(double), cudaMemcpyDeviceToDevice, s));
    ++pl->kappa_version;
    OperatorData *ops[2] = {&pl->op64, &pl->op32};
    for (int k = 0; k < 2; ++k) {
        OperatorData &op = *ops[k];
        if (!op.ready) continue;
        if (pl->geometry == IGA_GEOM_PRECOMPUTED) {
            if (k == 0)
                geom_setup_kernel<double><<<1184, 256, 0, s>>>((double *)op.G, pl->tabX64, pl->tabY64, pl->CP, pl->qw,
                                                              pl->kappa_dev, op.grid, pl->d_err);
            else
                geom_setup_kernel<float><<<1184, 256, 0, s>>>((float *)op.G, pl->tabX64, pl->tabY64, pl->CP, pl->qw,
                                                             pl->kappa_dev, op.grid, pl->d_err);
        } else {
            const size_t es = k == 0 ? sizeof(double) : sizeof(float);
            if (!op.kappa) IGA_CUDA_TRY(cudaMalloc(&op.kappa, nq * es));
            if (k == 0) kappa_convert_kernel<double><<<296, 256, 0, s>>>((double *)op.kappa, pl->kappa_dev, nq);
            else kappa_convert_kernel<float><<<296, 256, 0, s>>>((float *)op.kappa, pl->kappa_dev, nq);
        }
    }
    IGA_CUDA_TRY(cudaGetLastError());
    return IGA_OK;
}

static bool aligned_vectors(int prec, const void *x, const void *y)
{
    const uintptr_t es = prec == IGA_FP32 ? 4 : 8;
    if ((uintptr_t)x % es == 0 && (uintptr_t)y % es == 0) return true;
    set_error("x and y must be aligned to their element size");
    return false;
}

int iga_apply(iga_plan *pl, const void *x, void *y, void *stream)
{
    if (!pl || !x || !y) return IGA_ERR_ARG;
    const int prec = pl->precision == IGA_FP32 ? IGA_FP32 : IGA_FP64;
    if (!aligned_vectors(prec, x, y)) return IGA_ERR_ARG;
    return iga_apply_internal(pl, prec, x, y, (cudaStream_t)stream);
}

int iga_apply_prec(iga_plan *pl, int prec, const void *x, void *y, void *stream)
{
    if (!pl || !x || !y || (prec != IGA_FP64 && prec != IGA_FP32)) return IGA_ERR_ARG;
    if (!aligned_vectors(prec, x, y)) return IGA_ERR_ARG;
    return iga_apply_internal(pl, prec, x, y, (cudaStream_t)stream);
}

int iga_plan_device_status(iga_plan *pl, void *stream)
{
    if (!pl) return IGA_ERR_ARG;
    IGA_CUDA_TRY(cudaSetDevice(pl->device));
    IGA_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    const int st = iga_check_error_flag(pl);
    if (st == IGA_ERR_TIMEOUT) set_error("a bounded device wait of this plan's kernels gave up");
    else if (st) set_error("this plan's kernels recorded an error");
    return st;
}

int iga_plan_set_wait_limit(iga_plan *pl, long long polls)
{
    if (!pl) return IGA_ERR_ARG;
    pl->wait_polls = polls < 0 ? -1 : polls;
    return IGA_OK;
}

// Host buffers: the patch is applied in up to kHostSlabs slabs of strip rows
// (about one wave of strips each),
// so that the upload of x, the kernels and the download of y overlap on three
// streams (PCIe carries both directions at once). Slab k needs the x rows
// its strips touch (up to P rows past its last element row); after its strips
// and the seams of its control-point rows (those shared with slab k - 1
// included) its y rows are final and go back while slab k + 1 computes. Each
// point is computed exactly as by iga_apply: the result is bitwise the same.
constexpr int kHostSlabs = 8;

int iga_apply_host(iga_plan *pl, const double *xh, double *yh)
{
    if (!pl || !xh || !yh || !pl->op64.ready) return IGA_ERR_ARG;
    const size_t bytes = (size_t)pl->nfunc * sizeof(double);
    IGA_CUDA_TRY(cudaSetDevice(pl->device));
    if (!pl->d_stage_x) {
        IGA_CUDA_TRY(cudaMalloc((void **)&pl->d_stage_x, bytes));
        IGA_CUDA_TRY(cudaMalloc((void **)&pl->d_stage_y, bytes));
    }
    if (!pl->host_st[0]) {
        for (int k = 0; k < 3; ++k) IGA_CUDA_TRY(cudaStreamCreateWithFlags(&pl->host_st[k], cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k)
            for (int i = 0; i < kHostSlabs; ++i)
                IGA_CUDA_TRY(cudaEventCreateWithFlags(&pl->host_ev[k][i], cudaEventDisableTiming));
        IGA_CUDA_TRY(cudaEventCreateWithFlags(&pl->host_ev0, cudaEventDisableTiming));
    }
    cudaStream_t sin = pl->host_st[0], scmp = pl->host_st[1], sout = pl->host_st[2];
    // after the caller's work on the legacy stream
    IGA_CUDA_TRY(cudaEventRecord(pl->host_ev0, 0));
    for (int k = 0; k < 3; ++k) IGA_CUDA_TRY(cudaStreamWaitEvent(pl->host_st[k], pl->host_ev0, 0));
    const StripGrid &g = pl->op64.grid;
    // slabs of about one wave of strips each (fewer strips leave SMs idle)
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, pl->device);
    const long long wave = (long long)nsm * pl->op64.warps;
    const int K = (int)std::max<long long>(1, std::min<long long>({(long long)kHostSlabs, (long long)g.NSY,
                                                                    ((long long)g.NSX * g.NSY + wave / 2) / wave}));
    const int m = g.m, n = g.n, P = g.P;
    int in_rows = 0;   // x rows uploaded so far
    for (int k = 0; k < K; ++k) {
        const int gA = (int)((long long)g.NSY * k / K), gB = (int)((long long)g.NSY * (k + 1) / K);
        const int R0 = g.TY * gA, R1 = k + 1 == K ? n : g.TY * gB;
        const int need = k + 1 == K ? n : std::min(n, g.TY * gB + P);
        if (need > in_rows) {
            const size_t o = (size_t)in_rows * m, c = (size_t)(need - in_rows) * m;
            IGA_CUDA_TRY(cudaMemcpyAsync(pl->d_stage_x + o, xh + o, c * sizeof(double), cudaMemcpyHostToDevice, sin));
            in_rows = need;
        }
        IGA_CUDA_TRY(cudaEventRecord(pl->host_ev[0][k], sin));
        IGA_CUDA_TRY(cudaStreamWaitEvent(scmp, pl->host_ev[0][k], 0));
        Win w;
        w.gy0 = gA;
        w.gyn = gB - gA;
        w.R0 = R0;
        w.R1 = R1;
        const int st = launch_apply<double>(pl, pl->op64, pl->d_stage_x, pl->d_stage_y, scmp, pl->sign, pl->bc, w);
        if (st) return st;
        IGA_CUDA_TRY(cudaEventRecord(pl->host_ev[1][k], scmp));
        IGA_CUDA_TRY(cudaStreamWaitEvent(sout, pl->host_ev[1][k], 0));
        if (R1 > R0) {
            const size_t o = (size_t)R0 * m, c = (size_t)(R1 - R0) * m;
            IGA_CUDA_TRY(cudaMemcpyAsync(yh + o, pl->d_stage_y + o, c * sizeof(double), cudaMemcpyDeviceToHost, sout));
        }
    }
    IGA_CUDA_TRY(cudaStreamSynchronize(sout));
    return iga_check_error_flag(pl);
}

int iga_rhs(iga_plan *pl, int fkind, double *F, void *stream)
{
    if (!pl || !F || fkind < 0 || fkind > 2) return IGA_ERR_ARG;
    rhs_kernel<<<2 * 148, 256, 0, (cudaStream_t)stream>>>(F, pl->tabX64, pl->tabY64, pl->CP, pl->qw, fkind,
                                                         pl->grid);
    IGA_CUDA_TRY(cudaGetLastError());
    return IGA_OK;
}

// ------------------------------------------------- reference-shaped entry point
namespace {
// Cached plans, keyed by the device and every array pointer of the call; the
// arrays' contents are assumed unchanged while a plan is cached (a caller
// that rewrites them in place calls iga_MatrixFreeMatMultCUDA_release first).
using CacheKey = std::array<long long, 16>;
std::mutex g_cache_mu;
std::map<CacheKey, iga_plan *> g_cache;

// The caller's Bernstein tables and Gauss weights (matrix_free_gpu/src/
// GlobalAssemblyMF.cu:156-169: B[k][i] at quadrature point k) must be the
// (p+1)-point Gauss rule this library integrates with.
int check_rule(int p, const double *dB1, const double *dB2, const double *ddB1, const double *ddB2,
               const double *dqw1, const double *dqw2)
{
    const double *ptrs[6] = {dB1, dB2, ddB1, ddB2, dqw1, dqw2};
    int given = 0;
    for (const double *q : ptrs) given += q != nullptr;
    if (given == 0) return IGA_OK;   // not passed: the library's own rule
    if (given != 6) {
        set_error("d_B1, d_B2, d_dB1, d_dB2, qw1 and qw2 must be given together (or all NULL)");
        return IGA_ERR_ARG;
    }
    const int NB = p + 1, NQ = p + 1;
    std::vector<double> qx(NQ), qw(NQ), B((size_t)NQ * NB), dB((size_t)NQ * NB);
    gauss01(NQ, qx.data(), qw.data());
    for (int k = 0; k < NQ; ++k) bernstein(p, qx[k], B.data() + k * NB, dB.data() + k * NB);
    const std::vector<double> *want[6] = {&B, &B, &dB, &dB, &qw, &qw};
    for (int t = 0; t < 6; ++t) {
        std::vector<double> got(want[t]->size());
        IGA_CUDA_TRY(cudaMemcpy(got.data(), ptrs[t], got.size() * 8, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < got.size(); ++i)
            if (!(std::fabs(got[i] - (*want[t])[i]) <= 1e-13 * (1.0 + std::fabs((*want[t])[i])))) {
                set_error("the Bernstein tables / quadrature weights passed differ from the (p+1)-point "
                          "Gauss rule this library integrates with");
                return IGA_ERR_UNSUPPORTED;
            }
    }
    return IGA_OK;
}

// Builds the cached plan of one reference-shaped call: mesh tables copied
// once to the host, IEN / ID checked on the device, a plan with on-the-fly
// geometry (the reference kernel recomputes geometry too) and, for an ID
// other than the reference's serial numbering, a copy of ID for the rows.
int build_cached(int p, int q, int nex, int ney, const double *d_C1, const double *d_C2, const int *d_IEN,
                 const int *d_ID, const double *d_CP, iga_plan **out)
{
    const long long nf = (long long)(nex + p) * (ney + q);
    std::vector<double> CP(2 * nf), C1((size_t)nex * (p + 1) * (p + 1)), C2((size_t)ney * (q + 1) * (q + 1));
    IGA_CUDA_TRY(cudaMemcpy(CP.data(), d_CP, CP.size() * 8, cudaMemcpyDeviceToHost));
    IGA_CUDA_TRY(cudaMemcpy(C1.data(), d_C1, C1.size() * 8, cudaMemcpyDeviceToHost));
    IGA_CUDA_TRY(cudaMemcpy(C2.data(), d_C2, C2.size() * 8, cudaMemcpyDeviceToHost));
    int flags = 0;
    if (d_IEN || d_ID) {
        unsigned *seen = nullptr;
        int *dflags = nullptr;
        IGA_CUDA_TRY(cudaMalloc((void **)&seen, (size_t)((nf + 31) / 32) * sizeof(unsigned) + 16));
        cudaError_t e = cudaMalloc((void **)&dflags, sizeof(int));
        int st = e == cudaSuccess ? refentry_check(d_IEN, d_ID, p, nex, ney, seen, dflags, 0) : IGA_ERR_NOMEM;
        if (st == IGA_OK && cudaMemcpy(&flags, dflags, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
            st = IGA_ERR_CUDA;
        cudaFree(seen);
        if (dflags) cudaFree(dflags);
        if (st) {
            set_error("checking d_IEN / d_ID failed");
            return st;
        }
        if ((st = refentry_status(flags))) return st;
    }
    iga_mesh_desc d{};
    d.p = p;
    d.q = q;
    d.nElemX = nex;
    d.nElemY = ney;
    d.CP = CP.data();
    d.C1 = C1.data();
    d.C2 = C2.data();
    iga_opts o;
    iga_opts_default(&o);
    IGA_CUDA_TRY(cudaGetDevice(&o.device));
    o.geometry = IGA_GEOM_ON_THE_FLY;
    iga_plan *pl = nullptr;
    int st = iga_plan_create(&d, &o, &pl);
    if (st) return st;
    if (flags & kCheckIDOrder) {
        cudaError_t e = cudaMalloc((void **)&pl->eq_id, nf * sizeof(int));
        if (e == cudaSuccess) e = cudaMemcpy(pl->eq_id, d_ID, nf * sizeof(int), cudaMemcpyDeviceToDevice);
        if (e != cudaSuccess) {
            iga_plan_destroy(pl);
            set_error(std::string("copying d_ID: ") + cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? IGA_ERR_NOMEM : IGA_ERR_CUDA;
        }
    }
    *out = pl;
    return IGA_OK;
}
}  // namespace

int iga_MatrixFreeMatMultCUDA(int p, int q, int nex, int ney, const double *d_B1, const double *d_B2,
                              const double *d_dB1, const double *d_dB2, const double *d_C1, const double *d_C2,
                              const double *, const double *, const int *d_IEN, const int *d_ID, const double *d_CP,
                              const double *qw1, const double *qw2, const double *d_in, double *d_out)
{
    if (!d_C1 || !d_C2 || !d_CP || !d_in || !d_out || nex < 1 || ney < 1 || p < 1 || q < 1) return IGA_ERR_ARG;
    if ((uintptr_t)d_in % 8 || (uintptr_t)d_out % 8) {
        set_error("d_F_array_in / d_F_array_out must be 8-byte aligned");
        return IGA_ERR_ARG;
    }
    int dev = 0;
    IGA_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_cache_mu);
    const void *ptrs[11] = {d_CP, d_C1, d_C2, d_IEN, d_ID, d_B1, d_B2, d_dB1, d_dB2, qw1, qw2};
    CacheKey key{dev, p, q, nex, ney};
    for (int k = 0; k < 11; ++k) key[5 + k] = (long long)(uintptr_t)ptrs[k];
    auto it = g_cache.find(key);
    if (it == g_cache.end()) {
        if (p != q) {
            set_error("this library requires p == q");
            return IGA_ERR_UNSUPPORTED;
        }
        int st = check_rule(p, d_B1, d_B2, d_dB1, d_dB2, qw1, qw2);
        if (st) return st;
        iga_plan *pl = nullptr;
        if ((st = build_cached(p, q, nex, ney, d_C1, d_C2, d_IEN, d_ID, d_CP, &pl))) return st;
        it = g_cache.emplace(key, pl).first;
    }
    // Synchronous, as the reference's entry (cudaDeviceSynchronize after its
    // kernel, matrix_free_gpu/src/mult.cu:550): the status covers the launch
    // and every bounded wait of the kernels.
    const int st = iga_apply_internal(it->second, IGA_FP64, d_in, d_out, 0);
    if (st) return st;
    return iga_plan_device_status(it->second, nullptr);
}

int iga_MatrixFreeMatMultCUDA_release(void)
{
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (auto &kv : g_cache) iga_plan_destroy(kv.second);
    g_cache.clear();
    return IGA_OK;
}

}  // extern "C"
