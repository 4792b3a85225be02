// Device-side building blocks shared by the IGA kernels: PTX wrappers for the
// bulk-copy engine (TMA, cp.async.bulk) with mbarrier completion, Ampere-style
// cp.async for small ragged rows, bounded waits, and strip geometry.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include <utility>

namespace iga {

// ---------------------------------------------------------------- dependent launches
// Kernels that run inside the solver's captured loop start with pdl_begin():
// griddepcontrol.wait blocks until the preceding grid has completed and its
// memory is visible (a no-op when the kernel was launched without a
// programmatic dependency), then launch_dependents lets the next grid be
// scheduled while this one runs. A kernel whose CTAs all passed pdl_begin()
// can therefore have its successor's CTAs resident and waiting, which hides
// the launch gap between graph nodes.
__device__ __forceinline__ void pdl_begin()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// The two halves of pdl_begin() for kernels that first fetch operands no
// earlier grid writes (tables, geometry, eigenvectors) and set up shared
// memory and tensor memory while the preceding grid drains: pdl_launch() at
// the start, pdl_wait() before the first read of data an earlier grid
// produced and before the first global write. pdl_wait() is per thread.
__device__ __forceinline__ void pdl_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Host side: while pdl_capture() is true on this thread (the solver's loop
// capture), launch_k() launches with a programmatic stream serialisation
// attribute, so that stream capture records programmatic edges; otherwise
// it is an ordinary launch. Only kernels that begin with pdl_begin() may be
// launched through it.
inline bool &pdl_capture()
{
    static thread_local bool on = false;
    return on;
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                            Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    if (pdl_capture()) {
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
    }
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// Upper bound on mbarrier polls before a wait gives up and reports
// IGA_ERR_TIMEOUT; each try_wait suspends for a hardware-defined interval, so
// this is seconds of wall time, far beyond any legitimate copy latency.
constexpr long long kWaitLimit = 1LL << 24;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// 1-D bulk copy global -> shared through the async (TMA) proxy; completion is
// signalled on *bar as transaction bytes. dst, src 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of *bar; returns false after `limit` polls
// (limit 0: gives up at once, which tests use to exercise the timeout path).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, long long limit = kWaitLimit)
{
    for (long long it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// cp.async (LDGSTS) of 4, 8 or 16 bytes with zero fill when `valid` is false.
template <int BYTES>
__device__ __forceinline__ void cp_async_zfill(void *dst, const void *src, bool valid)
{
    const int src_size = valid ? BYTES : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES),
                 "r"(src_size)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Entries per (kind, qy) row of the apply kernel's y tables: the NB basis
// values padded so that a row is a whole number of 16-byte words (vector
// loads, 16-byte copies).
__host__ __device__ constexpr int tab_nbp(int NB, int esz)
{
    return (NB * esz) % 16 == 0 ? NB : ((NB * esz + 15) / 16 * 16) / esz;
}

// FP32 y tables up to p = 4 hold (value, derivative) pairs side by side, one
// row of NB pairs per qy padded to whole 16-byte words: the operands of packed
// f32x2 FMAs where the apply kernel uses them, and no more vector loads per
// row than two padded rows elsewhere (p=4 unchanged; at p = 5 the paired rows
// were slower, 144 -> 157 us at 1024^2); the others keep separate rows per
// kind. Entries of one element row: tab_row_len(NB, NQ, esz).
__host__ __device__ constexpr bool tab_paired(int NB, int esz) { return esz == 4 && NB <= 5; }
__host__ __device__ constexpr int tab_nbp2(int NB) { return (2 * NB * 4 + 15) / 16 * 16 / 4; }
__host__ __device__ constexpr int tab_row_len(int NB, int NQ, int esz)
{
    return tab_paired(NB, esz) ? NQ * tab_nbp2(NB) : 2 * NQ * tab_nbp(NB, esz);
}
// Offset of entry (kind, qy, jl) within an element row of y tables.
__host__ __device__ constexpr int tab_y_index(int NB, int NQ, int esz, int kind, int qy, int jl)
{
    return tab_paired(NB, esz) ? qy * tab_nbp2(NB) + 2 * jl + kind : (kind * NQ + qy) * tab_nbp(NB, esz) + jl;
}

// ---------------------------------------------------------------- strips
// Element columns per warp strip (two lanes per element column).
constexpr int kSW = 16;

// Whether the two lane halves share the middle quadrature column (odd NQ;
// esz = bytes per value): at NQ = 5 it saves 2 of 15 quadrature points per
// lane and element row (p=4 FP32 82 -> 75 us at 1024^2); at NQ = 3 it pays in
// FP32 (p=2 2048^2 153 -> 150 us) but not in FP64, where the split's extra
// table loads cost more than the idle slot (185 -> 192 us).
__host__ __device__ constexpr bool mid_shared(int NQ, int esz) { return NQ % 2 == 1 && (NQ >= 5 || esz == 4); }


// Quadrature column of x-table slot j (j < QH = ceil(NQ / 2)) of the lane
// half h: h QH + j (past NQ: an idle slot); where mid_shared(NQ, esz) the last
// slot of both halves is the middle column QH - 1 instead, whose quadrature
// rows the two halves split (h takes qy = h, h + 2, ...).
__host__ __device__ constexpr int lane_qx(int NQ, int esz, int h, int j)
{
    return (mid_shared(NQ, esz) && j == (NQ + 1) / 2 - 1) ? j : h * ((NQ + 1) / 2) + j;
}

// Layout of one element-row step of a strip's G (NQ^2 points x 3 values x
// kSW columns), per quadrature row qy. Even NQ: [lane = 2c + h][j][3] with
// qx = h QH + j, a lane's values contiguous (vector loads). Where the lane
// halves share the middle column at NQ = 3 (g_mid_lane_major): [lane][3] for
// the column of its own (qx = 0 or 2), then [c][3] for the middle column
// (p=2 2048^2 FP32 148.8 -> 144.9 us; at NQ = 5 the vector-loaded values
// spill under the FP32 kernel's 128-register cap, 75.6 -> 81.3 us, so p = 4
// keeps the columns apart). Otherwise: [qx][3][c].
__host__ __device__ constexpr bool g_lane_major(int NQ) { return NQ % 2 == 0; }
__host__ __device__ constexpr bool g_mid_lane_major(int NQ, int esz) { return mid_shared(NQ, esz) && NQ < 5; }
__host__ __device__ inline int g_index(int NQ, int esz, int qy, int qx, int comp, int c)
{
    const int QH = (NQ + 1) / 2, QB = NQ * 3 * kSW;
    if (g_lane_major(NQ)) {
        const int h = qx / QH, j = qx - h * QH;
        return qy * QB + ((2 * c + h) * QH + j) * 3 + comp;
    }
    if (g_mid_lane_major(NQ, esz)) {
        if (qx == QH - 1) return qy * QB + 32 * (QH - 1) * 3 + c * 3 + comp;
        const int h = qx < QH - 1 ? 0 : 1, j = h ? qx - QH : qx;
        return qy * QB + ((2 * c + h) * (QH - 1) + j) * 3 + comp;
    }
    return ((qy * NQ + qx) * 3 + comp) * kSW + c;
}

// The element grid is cut into warp strips of kSW element columns by TY
// element rows (nominal sizes; strips that overhang the mesh are padded with
// empty elements). A control-point row R (or column C) is covered by the
// strips whose element range, widened by p to the right/top, contains it:
// strip R/TY (if it exists) and strip R/TY - 1 when R % TY < p.
struct StripGrid {
    int m, n;       // control points per direction
    int nex, ney;
    int TY;         // element rows per strip
    int NSX, NSY;   // strips per direction
    int P;
    int FS;         // frame slots per strip
};

__host__ __device__ __forceinline__ int frame_size(int P, int TY) { return 2 * P * (TY + P) + 2 * P * (kSW - P); }

// Number of strips covering coordinate c along a direction of strip width w
// with NS strips, and the first (lowest) of them.
__host__ __device__ __forceinline__ int cover(int c, int w, int NS, int P, int &first)
{
    const int s = c / w;
    const bool has_s = s < NS;
    const bool has_prev = (c - s * w) < P && s >= 1 && (s - 1) < NS;
    first = has_prev ? s - 1 : s;
    return (int)has_s + (int)has_prev;
}

// Slot of footprint position (lr, lc) in a strip's frame (only positions that
// can be covered by another strip: lc < P, lc >= kSW, lr < P or lr >= TY).
__host__ __device__ __forceinline__ int frame_index(int lr, int lc, int P, int TY)
{
    if (lc < P) return lr * P + lc;
    if (lc >= kSW) return P * (TY + P) + lr * P + (lc - kSW);
    if (lr < P) return 2 * P * (TY + P) + lr * (kSW - P) + (lc - P);
    return 2 * P * (TY + P) + P * (kSW - P) + (lr - TY) * (kSW - P) + (lc - P);
}

}  // namespace iga
