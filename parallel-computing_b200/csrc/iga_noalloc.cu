// Allocation-free variant of the reference-shaped MatMult entry point.
//
// Some callers cannot allocate device memory at the moment they need a
// MatMult: a host application whose memory pool already owns the whole GPU
// (a framework caching allocator, a solver library with its own pool), or a
// Krylov loop that must not hit the implicit device synchronisation of
// cudaMalloc/cudaFree. iga_MatrixFreeMatMultCUDA_noalloc serves them: the
// caller passes every input and output as device arrays (the argument list of
// the reference's MatrixFreeMatMultCUDA plus a stream), and the only scratch
// the kernels need - the per-element-column / per-element-row basis tables and
// the seam frames of the atomic-free reduction - lives in the fixed array
// g_noalloc_scratch below, which every GPU that loads this library holds until
// the process exits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>

#include "iga_apply.cuh"
#include "iga_plan.hpp"

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;   // 16 MiB per device
constexpr int kMaxDevices = 64;

// File-scope device scratch. In host code this name is only a stand-in for
// the symbol, never a device address: the address comes from
// cudaGetSymbolAddress, per device, in scratch_on_current_device().
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void *g_addr[kMaxDevices] = {};
bool g_attr[kMaxDevices][6] = {};

// One-time set-up per device (first call on that device, under a lock): fetch
// the scratch address with the device current. Returns null on failure.
void *scratch_on_current_device(int &dev)
{
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return nullptr;
        g_addr[dev] = p;
    }
    return g_addr[dev];
}

// Basis tables of the apply kernel from the caller's Bernstein tables
// (B[k][i]: quadrature point k, Bernstein function i, the layout of
// matrix_free_gpu/src/GlobalAssemblyMF.cu:156-169) and extraction operators:
// N = C_e B (matrix_free/src/RefElement.cpp:20-57), in reference-element
// coordinates (no division by the element size).
__global__ void noalloc_tables_kernel(double *__restrict__ tabX, double *__restrict__ tabY,
                                      double *__restrict__ wq, int *__restrict__ err,
                                      const double *__restrict__ B1, const double *__restrict__ dB1,
                                      const double *__restrict__ B2, const double *__restrict__ dB2,
                                      const double *__restrict__ C1, const double *__restrict__ C2,
                                      const double *__restrict__ qw1, const double *__restrict__ qw2, int P,
                                      int nex, int ney, int NSX)
{
    const int NB = P + 1, NQ = P + 1, QH = (NQ + 1) / 2;
    const long long nX = (long long)NSX * 2 * QH * NB * 32;
    const int NBP = iga::tab_nbp(NB, (int)sizeof(double));
    const long long nY = (long long)ney * 2 * NQ * NBP;
    const long long tid0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (tid0 == 0) *err = 0;
    for (long long t = tid0; t < nX + nY + NQ * NQ; t += (long long)gridDim.x * blockDim.x) {
        if (t < nX) {   // [gx][kind][j][il][lane]: lane 2c+h = column 16 gx + c, qx = lane_qx(NQ, 8, h, j)
            const int lane = (int)(t % 32);
            long long r = t / 32;
            const int il = (int)(r % NB);
            r /= NB;
            const int j = (int)(r % QH);
            r /= QH;
            const int kind = (int)(r % 2);
            const int gx = (int)(r / 2);
            const int ex = iga::kSW * gx + lane / 2, qx = iga::lane_qx(NQ, 8, lane % 2, j);
            double v = 0.0;
            if (ex < nex && qx < NQ) {
                const double *Ce = C1 + (size_t)ex * NB * NB + il * NB;
                const double *Bq = (kind ? dB1 : B1) + qx * NB;
                for (int k = 0; k < NB; ++k) v += Ce[k] * Bq[k];
            }
            tabX[t] = v;
        } else if (t < nX + nY) {   // [ey][kind][qy][jl], jl < NBP (zero past NB)
            const long long u = t - nX;
            const int jl = (int)(u % NBP);
            long long r = u / NBP;
            const int qy = (int)(r % NQ);
            r /= NQ;
            const int kind = (int)(r % 2);
            const int ey = (int)(r / 2);
            double v = 0.0;
            if (jl < NB) {
                const double *Ce = C2 + (size_t)ey * NB * NB + jl * NB;
                const double *Bq = (kind ? dB2 : B2) + qy * NB;
                for (int k = 0; k < NB; ++k) v += Ce[k] * Bq[k];
            }
            tabY[u] = v;
        } else {
            const int k = (int)(t - nX - nY);
            wq[k] = qw1[k % NQ] * qw2[k / NQ];
        }
    }
}

// Scratch layout: a 256-byte head (the kernels' error slot at byte 0, the
// IEN / ID check flags at byte 4), the words marking ID values already seen
// (when d_ID is given), then the tables and the seam frames.
struct Layout {
    size_t off_err, off_flags, off_seen, off_wq, off_tabX, off_tabY, off_frame, total;
};

size_t up256(size_t v) { return (v + 255) & ~size_t(255); }

Layout layout_for(int P, int nex, int ney, int TY, bool with_id)
{
    const int NB = P + 1, NQ = P + 1, QH = (NQ + 1) / 2;
    const long long NSX = (nex + iga::kSW - 1) / iga::kSW, NSY = (ney + TY - 1) / TY;
    const long long N = (long long)(nex + P) * (ney + P);
    Layout L;
    L.off_err = 0;
    L.off_flags = 4;
    L.off_seen = 256;
    L.off_wq = L.off_seen + (with_id ? up256(sizeof(unsigned) * (size_t)((N + 31) / 32)) : 0);
    L.off_tabX = L.off_wq + up256(sizeof(double) * NQ * NQ);
    L.off_tabY = L.off_tabX + up256(sizeof(double) * NSX * 2 * QH * NB * 32);
    L.off_frame = L.off_tabY + up256(sizeof(double) * (size_t)ney * 2 * NQ * iga::tab_nbp(NB, (int)sizeof(double)));
    L.total = L.off_frame + up256(sizeof(double) * NSX * NSY * iga::frame_size(P, TY));
    return L;
}

template <int P>
int launch(int dev, unsigned char *base, const Layout &Ly, int TY, int nex, int ney, const double *d_CP,
           const int *d_ID, const double *d_in, double *d_out, cudaStream_t s)
{
    using namespace iga;
    int W = apply_max_threads<P, double, 1>() / 32;
    while (W > 1 && apply_smem_bytes<P, double, 1, 2>(W, 2) > 220 * 1024) --W;
    const size_t smem_max = apply_smem_bytes<P, double, 1, 2>(W, 2);
    auto kern = apply_kernel<P, double, 1, 2>;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_attr[dev][P]) {
            const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max);
            if (e != cudaSuccess) {
                set_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
                return IGA_ERR_CUDA;
            }
            g_attr[dev][P] = true;
        }
    }
    StripGrid g;
    g.m = nex + P;
    g.n = ney + P;
    g.nex = nex;
    g.ney = ney;
    g.TY = TY;
    g.NSX = (nex + kSW - 1) / kSW;
    g.NSY = (ney + TY - 1) / TY;
    g.P = P;
    g.FS = frame_size(P, TY);
    ApplyParams<double> a;
    a.x = d_in;
    a.y = d_out;
    a.G = nullptr;
    a.tabX = reinterpret_cast<const double *>(base + Ly.off_tabX);
    a.tabY = reinterpret_cast<const double *>(base + Ly.off_tabY);
    a.CP = d_CP;
    a.wq = reinterpret_cast<const double *>(base + Ly.off_wq);
    a.kappa = nullptr;
    a.frame = reinterpret_cast<double *>(base + Ly.off_frame);
    a.g = g;
    a.sign = -1.0;   // the reference operator A_ref = -K
    // the reference's serial numbering: y[Dir] = 0; any other ID: rows through ID
    a.bc = d_ID ? IGA_BC_NONE : IGA_BC_REFERENCE;
    a.ID = d_ID;
    a.err = reinterpret_cast<int *>(base + Ly.off_err);
    // strips dealt to warps one by one; with shared tables the CTA's strips
    // lie in at most two column strips (W - 1 <= NSY)
    constexpr bool percol = apply_percolumn<P, double, 1>();
    if (apply_txshared<P, double, 1>() && !percol) W = std::max(1, std::min(W, g.NSY + 1));
    const long long nstrips = (long long)g.NSX * g.NSY;
    const dim3 grid = percol ? dim3(g.NSX, (g.NSY + W - 1) / W) : dim3((unsigned)((nstrips + W - 1) / W)),
               block(32, W);
    kern<<<grid, block, apply_smem_bytes<P, double, 1, 2>(W, !percol && g.NSY % W ? 2 : 1), s>>>(a);
    cudaError_t e = cudaPeekAtLastError();
    const long long nseam = (long long)(g.NSX - 1) * P * g.n + (long long)(g.NSY - 1) * P * g.m;
    if (e == cudaSuccess && nseam > 0) {
        seam_fixup_kernel<P, double><<<(int)std::min<long long>((nseam + 255) / 256, 592), 256, 0, s>>>(
            a.frame, d_in, d_out, g, -1.0, a.bc, d_ID);
        e = cudaPeekAtLastError();
    }
    if (e != cudaSuccess) {
        set_error(std::string("iga_MatrixFreeMatMultCUDA_noalloc launch: ") + cudaGetErrorString(e));
        return IGA_ERR_CUDA;
    }
    return IGA_OK;
}

// Reads one int of the scratch back to the host after the stream's work
// (into a host variable: nothing is allocated).
int read_back(const unsigned char *base, size_t off, cudaStream_t s, int &out)
{
    cudaError_t e = cudaMemcpyAsync(&out, base + off, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        iga::set_error(std::string("iga_MatrixFreeMatMultCUDA_noalloc: ") + cudaGetErrorString(e));
        return IGA_ERR_CUDA;
    }
    return IGA_OK;
}

}  // namespace

extern "C" int iga_MatrixFreeMatMultCUDA_noalloc(int p, int q, int nex, int ney, const double *d_B1,
                                                 const double *d_B2, const double *d_dB1, const double *d_dB2,
                                                 const double *d_C1, const double *d_C2, const double *,
                                                 const double *, const int *d_IEN, const int *d_ID,
                                                 const double *d_CP, const double *qw1, const double *qw2,
                                                 const double *d_in, double *d_out, void *stream)
{
    if (p < 1 || q < 1 || nex < 1 || ney < 1) return IGA_ERR_ARG;
    if (p > 5 || q != p) {
        iga::set_error("iga_MatrixFreeMatMultCUDA_noalloc handles p == q with 1 <= p <= 5");
        return IGA_ERR_UNSUPPORTED;
    }
    if (!d_B1 || !d_B2 || !d_dB1 || !d_dB2 || !d_C1 || !d_C2 || !d_CP || !qw1 || !qw2 || !d_in || !d_out)
        return IGA_ERR_ARG;
    // d_CP is read as 16-byte (x, y) pairs, the double arrays as doubles, IEN/ID as ints.
    bool aligned = (uintptr_t)d_CP % 16 == 0 && (uintptr_t)d_IEN % 4 == 0 && (uintptr_t)d_ID % 4 == 0;
    for (const double *q8 : {d_B1, d_B2, d_dB1, d_dB2, d_C1, d_C2, qw1, qw2, d_in, (const double *)d_out})
        aligned = aligned && (uintptr_t)q8 % 8 == 0;
    if (!aligned) {
        iga::set_error("iga_MatrixFreeMatMultCUDA_noalloc: d_CP must be 16-byte aligned, the other double "
                       "arrays 8-byte and d_IEN / d_ID 4-byte aligned");
        return IGA_ERR_ARG;
    }
    // Strip height: the smallest of these whose tables and frames fit the scratch.
    int TY = 0;
    Layout Ly{};
    for (int cand : {32, 64, 128, 256, 512, 1024}) {
        if (cand < p) continue;
        Ly = layout_for(p, nex, ney, cand, d_ID != nullptr);
        if (Ly.total <= kScratchBytes) {
            TY = cand;
            break;
        }
    }
    if (!TY) {
        iga::set_error("mesh too large for the fixed 16 MiB scratch of iga_MatrixFreeMatMultCUDA_noalloc");
        return IGA_ERR_UNSUPPORTED;
    }
    (void)cudaGetLastError();   // an earlier, unrelated launch error is not this call's
    int dev = 0;
    unsigned char *base = static_cast<unsigned char *>(scratch_on_current_device(dev));
    if (!base) {
        iga::set_error("cudaGetSymbolAddress of the no-alloc scratch failed");
        return IGA_ERR_CUDA;
    }
    cudaStream_t s = (cudaStream_t)stream;
    // IEN / ID first: a call they do not fit is refused before y is touched.
    const int *id_rows = nullptr;
    if (d_IEN || d_ID) {
        int st = iga::refentry_check(d_IEN, d_ID, p, nex, ney, reinterpret_cast<unsigned *>(base + Ly.off_seen),
                                     reinterpret_cast<int *>(base + Ly.off_flags), s);
        int flags = 0;
        if (st == IGA_OK) st = read_back(base, Ly.off_flags, s, flags);
        if (st == IGA_OK) st = iga::refentry_status(flags);
        if (st) return st;
        if (flags & iga::kCheckIDOrder) id_rows = d_ID;
    }
    const int NSX = (nex + iga::kSW - 1) / iga::kSW;
    noalloc_tables_kernel<<<148, 256, 0, s>>>(
        reinterpret_cast<double *>(base + Ly.off_tabX), reinterpret_cast<double *>(base + Ly.off_tabY),
        reinterpret_cast<double *>(base + Ly.off_wq), reinterpret_cast<int *>(base + Ly.off_err), d_B1, d_dB1, d_B2,
        d_dB2, d_C1, d_C2, qw1, qw2, p, nex, ney, NSX);
    int st;
    switch (p) {
    case 1: st = launch<1>(dev, base, Ly, TY, nex, ney, d_CP, id_rows, d_in, d_out, s); break;
    case 2: st = launch<2>(dev, base, Ly, TY, nex, ney, d_CP, id_rows, d_in, d_out, s); break;
    case 3: st = launch<3>(dev, base, Ly, TY, nex, ney, d_CP, id_rows, d_in, d_out, s); break;
    case 4: st = launch<4>(dev, base, Ly, TY, nex, ney, d_CP, id_rows, d_in, d_out, s); break;
    default: st = launch<5>(dev, base, Ly, TY, nex, ney, d_CP, id_rows, d_in, d_out, s); break;
    }
    if (st) return st;
    // Synchronous, like the reference's entry: the kernels' own error slot
    // (a bounded wait that gave up) is read back before returning.
    int err = 0;
    if ((st = read_back(base, Ly.off_err, s, err))) return st;
    if (err) {
        iga::set_error("iga_MatrixFreeMatMultCUDA_noalloc: a kernel recorded an error");
        return err;
    }
    return IGA_OK;
}
