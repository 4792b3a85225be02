// Dense GEMMs of the exact FEM preconditioner without a BLAS library
// (interface and operand conventions in iga_gemm.hpp).
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>

#include "iga_gemm.hpp"
#include "iga_plan.hpp"
#include "iga_umma.cuh"

namespace iga {

// ------------------------------------------------------------ TF32 on tcgen05
// One CTA computes a 128 x 128 tile of C with the FP32 accumulator in 128
// TMEM columns. Thread 0 of warp 0 feeds a ring of 3 or 4 stages with the
// tensor-memory accelerator: per stage a 32-wide K slice of A (128 rows) and
// of B (128 rows), 16 KiB each, in the canonical swizzled layouts of the UMMA
// descriptors (K-major: 128-byte rows of 32 k values, 8-row groups 1 KiB
// apart; MN-major: four 4 KiB boxes of 32 k rows x 32 values, one per 32-wide
// MN atom, in the 32-byte-atom swizzle). Thread 0 of warp 1 issues four 128 x 128 x 8 MMAs per
// stage and commits them to the stage's "empty" barrier, which releases the
// stage to the copy thread. After the last slice a commit to "done" hands
// the accumulator to the epilogue: every warp reads its 32 TMEM lanes
// (tcgen05.ld 32x32b) and stores its rows of C. No cluster multicast.
// Two CTAs fit an SM (96 KiB of stages each), so a 2064 x 2064 product
// (17 x 17 tiles) runs in one wave on 148 SMs.
// The tile width BN is 128, or 64 where the 128-wide grid would leave SMs
// idle (the 1040 x 1040 transforms of a 1024^2 patch: 81 tiles of 128 x 128
// on 148 SMs, 153 of 128 x 64).
constexpr int kGM = 128, kGK = 32;
constexpr int kGTileA = kGM * kGK * 4;   // bytes of one A slice
// Ring stages: 3 for 128-wide tiles (96 KiB, two CTAs per SM); 4 for 64-wide
// ones (96 KiB as well), whose short k loops (the 1040^2 transforms: 17
// slices) are bound by the copies' round trips, not the MMAs.
template <int BN>
__host__ __device__ constexpr int gemm_tf32_stages() { return BN == 64 ? 4 : 3; }
template <int BN>
constexpr int gemm_tf32_smem() { return 1024 + gemm_tf32_stages<BN>() * (kGTileA + BN * kGK * 4) + 256; }

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Descriptors of the operand tiles (layout type in bits [61, 64)):
// K-major tiles use the 128-byte swizzle (type 2; 128-byte rows of 32 k
// values, 8-row groups SBO apart); MN-major TF32 tiles must use the 128-byte
// swizzle with 32-byte atoms (type 1: 128-byte K rows, 4-row groups SBO apart,
// 32-value MN atoms LBO apart), the only MN-major layout the tensor cores
// take for 32-bit operands; the copy engine writes it with
// CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B.
__device__ __forceinline__ uint64_t sw128_desc(const void *p, uint32_t lbo, uint32_t sbo)
{
    return umma::smem_desc(p, lbo, sbo) | ((uint64_t)2 << 61);
}
__device__ __forceinline__ uint64_t sw128_32b_desc(const void *p, uint32_t lbo, uint32_t sbo)
{
    return umma::smem_desc(p, lbo, sbo) | ((uint64_t)1 << 61);
}

// Output tile of a CTA and its k range. Without a split, tile (bx, by) is
// rows bx TM .., columns by TN .., all of k. With a block-diagonal operand
// split at kb, the tiles along the split dimension are laid out block by
// block (ceil(kb / T) tiles from 0, then tiles from kb), so that no tile
// straddles kb: each runs over its block's k range only, and stores rows (or
// columns) below its block's end only (the rest of a last partial tile
// belongs to the other block's tiles).
struct TileRange {
    int m0, n0, klo, khi, mlim, nlim;
};
__device__ __forceinline__ TileRange tile_range(const GemmSplit &sp, int bx, int by, int TM, int TN, int K, int Mst,
                                                int Nst)
{
    TileRange t{bx * TM, by * TN, 0, K, Mst, Nst};
    if (sp.kb > 0) {
        const int T = sp.on_n ? TN : TM, idx = sp.on_n ? by : bx;
        const int te = (sp.kb + T - 1) / T;
        const bool even = idx < te;
        const int s0 = even ? idx * T : sp.kb + (idx - te) * T;
        const int lim = even ? sp.kb : (sp.on_n ? Nst : Mst);
        t.klo = even ? 0 : sp.kb;
        t.khi = even ? sp.kb : K;
        if (sp.on_n) {
            t.n0 = s0;
            t.nlim = lim;
        } else {
            t.m0 = s0;
            t.mlim = lim;
        }
    }
    return t;
}
// Tiles along a dimension of extent `ext` cut into tiles of T (split at kb when kb > 0).
__host__ __forceinline__ int tiles_along(int ext, int T, int kb)
{
    return kb > 0 ? (kb + T - 1) / T + (ext - kb + T - 1) / T : (ext + T - 1) / T;
}

// OUT: 0 C, 1 scatter into an FP32 vector, 2 into an FP64 vector (GemmScatter).
template <bool AMN, bool BMN, int OUT, int BN>
__global__ void __launch_bounds__(128) gemm_tf32_kernel(const __grid_constant__ CUtensorMap ta,
                                                        const __grid_constant__ CUtensorMap tb, int K, int Mst, int Nst,
                                                        float *__restrict__ C, int ldc, int *__restrict__ err,
                                                        GemmScatter sc, GemmSplit split, int const_op)
{
    constexpr int kGTileB = BN * kGK * 4;
    constexpr int kGS = gemm_tf32_stages<BN>();
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm =
        reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char *As = sm, *Bs = sm + kGS * kGTileA;
    uint64_t *full = reinterpret_cast<uint64_t *>(sm + kGS * (kGTileA + kGTileB));
    uint64_t *empty = full + kGS, *done = empty + kGS;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(done + 1);
    int *cnt = reinterpret_cast<int *>(tslot + 1);   // [0] slices loaded, [1] slices consumed, [2] failure
    // Tensor memory, barriers and (const_op) the first stages of the operand
    // no earlier grid writes are set up before the wait for the preceding
    // grid; the other operand's loads and every global write come after it.
    pdl_launch();
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const TileRange tr = tile_range(split, blockIdx.x, blockIdx.y, kGM, BN, K, Mst, Nst);
    const int m0 = tr.m0, n0 = tr.n0, klo = tr.klo;
    const int nk = (tr.khi - klo + kGK - 1) / kGK;

    if (warp == 0) {
        umma::alloc(tslot, BN);
        umma::relinquish();
    }
    if (tid == 32) {
        for (int s = 0; s < kGS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        cnt[0] = cnt[1] = cnt[2] = 0;
        fence_mbar_init();
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;

    if (warp == 0 && lane == 0) {   // copy thread
        auto load_a = [&](int s, int k0) {
            unsigned char *a = As + s * kGTileA;
            if (AMN) {
                for (int j = 0; j < kGM / 32; ++j) tma_load_2d(a + j * 4096, &ta, m0 + 32 * j, k0, &full[s]);
            } else {
                tma_load_2d(a, &ta, k0, m0, &full[s]);
            }
        };
        auto load_b = [&](int s, int k0) {
            unsigned char *b = Bs + s * kGTileB;
            if (BMN) {
                for (int j = 0; j < BN / 32; ++j) tma_load_2d(b + j * 4096, &tb, n0 + 32 * j, k0, &full[s]);
            } else {
                tma_load_2d(b, &tb, k0, n0, &full[s]);
            }
        };
        // stages 0 .. npre-1: the constant operand now, the other after the wait
        const int npre = const_op ? min(nk, kGS) : 0;
        for (int kt = 0; kt < npre; ++kt) {
            mbar_arrive_expect_tx(&full[kt], kGTileA + kGTileB);
            if (const_op == 1) load_a(kt, klo + kt * kGK);
            else load_b(kt, klo + kt * kGK);
        }
        pdl_wait();
        int kt = 0;
        for (; kt < nk; ++kt) {
            const int s = kt % kGS;
            if (kt >= kGS && !mbar_wait_bounded(&empty[s], (uint32_t)((kt / kGS - 1) & 1))) {
                cnt[2] = 1;
                break;
            }
            const int k0 = klo + kt * kGK;
            if (kt >= npre) mbar_arrive_expect_tx(&full[s], kGTileA + kGTileB);
            if (kt >= npre || const_op != 1) load_a(s, k0);
            if (kt >= npre || const_op != 2) load_b(s, k0);
        }
        cnt[0] = kt;
    } else if (warp == 1 && lane == 0) {   // MMA thread
        constexpr uint32_t IDESC =
            umma::idesc_tf32<kGM, BN>() | ((uint32_t)AMN << 15) | ((uint32_t)BMN << 16);
        int kt = 0;
        for (; kt < nk; ++kt) {
            const int s = kt % kGS;
            if (!mbar_wait_bounded(&full[s], (uint32_t)((kt / kGS) & 1))) {
                cnt[2] = 1;
                break;
            }
            umma::fence_after_sync();
            const unsigned char *a = As + s * kGTileA, *b = Bs + s * kGTileB;
#pragma unroll
            for (int j = 0; j < kGK / 8; ++j) {
                // K substep j: 8 k values = 32 bytes along a K-major row, or 8
                // K rows (two 512-byte swizzle groups) of an MN-major tile
                const uint64_t ad = AMN ? sw128_32b_desc(a + j * 1024, 4096, 512) : sw128_desc(a + j * 32, 16, 1024);
                const uint64_t bd = BMN ? sw128_32b_desc(b + j * 1024, 4096, 512) : sw128_desc(b + j * 32, 16, 1024);
                umma::mma_tf32(tmem, ad, bd, IDESC, (kt > 0 || j > 0) ? 1u : 0u);
            }
            umma::commit(&empty[s]);
        }
        cnt[1] = kt;
        umma::commit(done);   // arrives once every MMA issued above has completed
    }
    __syncwarp();
    const bool ok = !__syncthreads_or(!mbar_wait_bounded(done, 0));   // uniform over the CTA
    pdl_wait();   // (long since passed by the copy thread) before this thread's global reads and writes
    const bool failed = !ok || cnt[2] || cnt[1] < nk;
    if (!failed) {
        umma::fence_after_sync();
        const int row = m0 + 32 * warp + lane;
        double f = 1.0;
        if (OUT != 0 && sc.rr) {
            const double rr = *sc.rr;
            f = (rr > 0.0 && rr < 1e300) ? sqrt(rr) : 1.0;
        }
        // scatter output: each warp's 32 x 16 chunk goes through shared memory
        // (the drained A stages) so that a half-warp stores 16 consecutive
        // entries of one row instead of each lane its own row
        float *stage = reinterpret_cast<float *>(As) + warp * 32 * 17;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            umma::ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
            umma::wait_ld();
            const int col = n0 + c0;
            if (OUT != 0) {
#pragma unroll
                for (int c = 0; c < 16; ++c) stage[lane * 17 + c] = v[c];
                __syncwarp();
                const int cl = lane & 15, r0 = m0 + 32 * warp;
#pragma unroll 4
                for (int rr = 0; rr < 16; ++rr) {
                    const int rl = 2 * rr + (lane >> 4), row_s = r0 + rl;
                    if (row_s < sc.rows && col + cl < sc.cols && row_s < tr.mlim && col + cl < tr.nlim) {
                        const double val = f * (double)stage[rl * 17 + cl];
                        const size_t at = (size_t)(row_s + 1) * sc.ld + col + cl + 1;
                        if (OUT == 1) static_cast<float *>(sc.out)[at] = (float)val;
                        else static_cast<double *>(sc.out)[at] = val;
                    }
                }
                __syncwarp();
                continue;
            }
            if (row >= tr.mlim || col >= tr.nlim) continue;
            float *dst = C + (size_t)row * ldc + col;
            if (col + 16 <= tr.nlim) {
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    reinterpret_cast<float4 *>(dst)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            } else {
#pragma unroll
                for (int c = 0; c < 16; ++c)
                    if (c < tr.nlim - col) dst[c] = v[c];
            }
        }
    } else {
        if (tid == 0) {
            atomicExch(err, 8 /* IGA_ERR_TIMEOUT */);
            // the copies issued and not consumed land before the stages are released
            for (int kt = cnt[1]; kt < cnt[0]; ++kt) mbar_wait_bounded(&full[kt % kGS], (uint32_t)((kt / kGS) & 1));
        }
        if (!ok) mbar_wait_bounded(done, 0);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::dealloc(tmem, BN);
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encoder()
{
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Tensor map of one operand: K-major X[rows][k] (box 32 k x box_rows rows,
// 128-byte swizzle) or MN-major X[k][rows] (box 32 rows x 32 k, 128-byte
// swizzle with 32-byte atoms), FP32, reads outside [0, inner) x [0, outer)
// zero-filled.
int make_map(CUtensorMap &map, const GemmOperand &op, int rows, int K, int box_rows)
{
    auto enc = encoder();
    if (!enc) {
        set_error("cuTensorMapEncodeTiled is not available from the driver");
        return IGA_ERR_CUDA;
    }
    if ((uintptr_t)op.ptr % 16 || (op.ld * 4) % 16) {
        set_error("TF32 GEMM operands need 16-byte aligned rows");
        return IGA_ERR_ARG;
    }
    const cuuint64_t inner = op.mn_major ? rows : K, outer = op.mn_major ? K : rows;
    const cuuint64_t dims[2] = {inner, outer};
    const cuuint64_t strides[1] = {(cuuint64_t)op.ld * 4};
    const cuuint32_t box[2] = {32u, op.mn_major ? 32u : (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(op.ptr), dims, strides, box,
                           estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           op.mn_major ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B : CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
        return IGA_ERR_CUDA;
    }
    return IGA_OK;
}

template <bool AMN, bool BMN, int OUT, int BN>
int launch_tf32_t(const GemmTF32 &g, cudaStream_t s, int *err, const GemmScatter &sc)
{
    constexpr int smem = gemm_tf32_smem<BN>();
    static bool attr = false;   // per instantiation
    if (!attr) {
        if (cudaFuncSetAttribute(gemm_tf32_kernel<AMN, BMN, OUT, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem) != cudaSuccess)
            return IGA_ERR_CUDA;
        attr = true;
    }
    const dim3 grid(tiles_along(g.Mst, kGM, g.split.on_n ? 0 : g.split.kb),
                    tiles_along(g.Nst, BN, g.split.on_n ? g.split.kb : 0));
    return launch_k(gemm_tf32_kernel<AMN, BMN, OUT, BN>, grid, dim3(128), smem, s, g.ta, g.tb, g.K, g.Mst, g.Nst, g.C,
                    g.ldc, err, sc, g.split, g.const_op) == cudaSuccess
               ? IGA_OK
               : IGA_ERR_CUDA;
}

template <bool AMN, bool BMN, int BN>
int launch_tf32_bn(const GemmTF32 &g, cudaStream_t s, int *err, const GemmScatter &sc)
{
    if (!sc.out) return launch_tf32_t<AMN, BMN, 0, BN>(g, s, err, sc);
    return sc.f64 ? launch_tf32_t<AMN, BMN, 2, BN>(g, s, err, sc) : launch_tf32_t<AMN, BMN, 1, BN>(g, s, err, sc);
}

template <bool AMN, bool BMN>
int launch_tf32(const GemmTF32 &g, cudaStream_t s, int *err, const GemmScatter &sc)
{
    return g.bn == 64 ? launch_tf32_bn<AMN, BMN, 64>(g, s, err, sc) : launch_tf32_bn<AMN, BMN, 128>(g, s, err, sc);
}
}  // namespace

int gemm_tf32_prepare(GemmTF32 &g, GemmOperand A, GemmOperand B, float *C, int ldc, int M, int N, int K, int Mst,
                      int Nst, GemmSplit split)
{
    g.ready = false;
    // 128-wide tiles when they fill the SMs about one and a half times over, else 64-wide
    int nsm = 148, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        nsm = 148;
    const long long tiles128 = (long long)((Mst + kGM - 1) / kGM) * ((Nst + 127) / 128);
    g.bn = tiles128 >= 3LL * nsm / 2 ? 128 : 64;
    int st;
    if ((st = make_map(g.ta, A, M, K, kGM)) || (st = make_map(g.tb, B, N, K, g.bn))) return st;
    if ((uintptr_t)C % 16 || ldc % 4) {
        set_error("TF32 GEMM output needs 16-byte aligned rows");
        return IGA_ERR_ARG;
    }
    g.a_mn = A.mn_major;
    g.b_mn = B.mn_major;
    g.M = M;
    g.N = N;
    g.K = K;
    g.Mst = Mst;
    g.Nst = Nst;
    g.C = C;
    g.ldc = ldc;
    g.split = split.kb > 0 && split.kb < K ? split : GemmSplit();
    g.ready = true;
    return IGA_OK;
}

int gemm_tf32_launch(const GemmTF32 &g, cudaStream_t s, int *err, const GemmScatter &sc)
{
    if (!g.ready) return IGA_ERR_ARG;
    // the two operand layouts the preconditioner uses (both K-major, both MN-major)
    if (g.a_mn && g.b_mn) return launch_tf32<true, true>(g, s, err, sc);
    if (!g.a_mn && !g.b_mn) return launch_tf32<false, false>(g, s, err, sc);
    set_error("TF32 GEMM: mixed operand layouts are not built");
    return IGA_ERR_UNSUPPORTED;
}

// ------------------------------------------------------------ FP64 on DMMA
// A CTA of WMW x WNW warps computes a (16 WI WMW) x (32 WNW) tile of C; a
// warp tile is WI x 4 blocks of the 16 x 8 x 8 FP64 MMA. K slices of 16 are
// staged by 16-byte cp.async into a 3-deep ring: K-major operands as
// [row][k] with 20 doubles per row, MN-major ones as [k][row] with ROWS + 4
// per k, both of which make a warp's fragment loads conflict-free. Rows and k
// past an operand's extent are zero-filled (the matrices are zero-padded, so
// a 16-byte chunk never straddles the end of the data). Three shapes:
//   0: 128 x 128, 8 warps of 64 x 32 (one CTA per SM);
//   1: 128 x 64, 8 warps of 32 x 32 (two CTAs per SM);
//   2: 64 x 64, 4 warps of 32 x 32 (three CTAs per SM), the default.
constexpr int kDK = 16, kDS = 3;
constexpr int kDLK = 20;

template <bool MN, int ROWS>
struct DTile {
    static constexpr int LR = ROWS + 4;
    static constexpr int elems = MN ? kDK * LR : ROWS * kDLK;
    __device__ static int at(int row, int k) { return MN ? k * LR + row : row * kDLK + k; }
};

// D (16 x 8) += A (16 x 8) B (8 x 8), FP64. Fragments (g = lane / 4,
// t = lane % 4): a = A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4];
// b = B[t][g], B[t+4][g]; d = D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1].
__device__ __forceinline__ void dmma(double (&d)[4], const double (&a)[4], const double (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Stages the slice k0 .. k0 + 15 of an operand tile (rows r0 .. r0 + ROWS - 1).
template <bool MN, int ROWS, int NT>
__device__ __forceinline__ void stage_f64(double *dst, const double *__restrict__ src, int ld, int rows, int K, int r0,
                                          int k0, int tid)
{
    constexpr int CHUNKS = ROWS * kDK / 2;   // 16-byte chunks
#pragma unroll
    for (int c = tid; c < CHUNKS; c += NT) {
        int row, k;
        if (MN) {   // [k][row] chunks along rows
            k = c / (ROWS / 2);
            row = 2 * (c % (ROWS / 2));
        } else {    // [row][k] chunks along k
            row = c / (kDK / 2);
            k = 2 * (c % (kDK / 2));
        }
        const int gr = r0 + row, gk = k0 + k;
        const bool v = gr < rows && gk < K;
        const double *g = v ? (MN ? src + (size_t)gk * ld + gr : src + (size_t)gr * ld + gk) : src;
        cp_async_zfill<16>(dst + DTile<MN, ROWS>::at(row, k), g, v);
    }
}

template <int CFG>
struct DCfg;
template <>
struct DCfg<0> {
    static constexpr int WI = 4, WMW = 2, WNW = 4, MINB = 1;
};
template <>
struct DCfg<1> {
    static constexpr int WI = 2, WMW = 4, WNW = 2, MINB = 2;
};
template <>
struct DCfg<2> {
    static constexpr int WI = 2, WMW = 2, WNW = 2, MINB = 3;
};

template <int CFG, bool AMN, bool BMN, bool SCATTER>
__global__ void __launch_bounds__(32 * DCfg<CFG>::WMW * DCfg<CFG>::WNW, DCfg<CFG>::MINB)
    gemm_f64_kernel(const double *__restrict__ A, int lda, const double *__restrict__ B, int ldb,
                    double *__restrict__ C, int ldc, int M, int N, int K, int Mst, int Nst, GemmScatter sc,
                    GemmSplit split)
{
    using Cf = DCfg<CFG>;
    constexpr int WI = Cf::WI, NT = 32 * Cf::WMW * Cf::WNW;
    constexpr int TM = 16 * WI * Cf::WMW, TN = 32 * Cf::WNW;
    using TA = DTile<AMN, TM>;
    using TB = DTile<BMN, TN>;
    pdl_begin();
    extern __shared__ __align__(16) double dsm[];
    double *As = dsm, *Bs = dsm + kDS * TA::elems;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int wm = (w % Cf::WMW) * 16 * WI, wn = (w / Cf::WMW) * 32;
    const TileRange tr = tile_range(split, blockIdx.x, blockIdx.y, TM, TN, K, Mst, Nst);
    const int m0 = tr.m0, n0 = tr.n0, klo = tr.klo;
    const int nk = (tr.khi - klo + kDK - 1) / kDK;
    double acc[WI][4][4];
#pragma unroll
    for (int i = 0; i < WI; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[i][j][c] = 0.0;
    for (int s = 0; s < kDS - 1; ++s) {
        if (s < nk) {
            stage_f64<AMN, TM, NT>(As + s * TA::elems, A, lda, M, K, m0, klo + s * kDK, tid);
            stage_f64<BMN, TN, NT>(Bs + s * TB::elems, B, ldb, N, K, n0, klo + s * kDK, tid);
        }
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait<kDS - 2>();
        __syncthreads();
        {   // refill the stage consumed one iteration ago
            const int nt = kt + kDS - 1, s = nt % kDS;
            if (nt < nk) {
                stage_f64<AMN, TM, NT>(As + s * TA::elems, A, lda, M, K, m0, klo + nt * kDK, tid);
                stage_f64<BMN, TN, NT>(Bs + s * TB::elems, B, ldb, N, K, n0, klo + nt * kDK, tid);
            }
            cp_async_commit();
        }
        const double *a = As + (kt % kDS) * TA::elems, *b = Bs + (kt % kDS) * TB::elems;
#pragma unroll
        for (int kk = 0; kk < kDK; kk += 8) {
            double av[WI][4], bv[4][2];
#pragma unroll
            for (int i = 0; i < WI; ++i) {
                const int r = wm + 16 * i + g;
                av[i][0] = a[TA::at(r, kk + t4)];
                av[i][1] = a[TA::at(r + 8, kk + t4)];
                av[i][2] = a[TA::at(r, kk + t4 + 4)];
                av[i][3] = a[TA::at(r + 8, kk + t4 + 4)];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                bv[j][0] = b[TB::at(wn + 8 * j + g, kk + t4)];
                bv[j][1] = b[TB::at(wn + 8 * j + g, kk + t4 + 4)];
            }
#pragma unroll
            for (int i = 0; i < WI; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc[i][j], av[i], bv[j]);
        }
    }
    cp_async_wait<0>();
    // accumulator (i, j, c): row wm + 16 i + g + 8 (c / 2), column wn + 8 j + 2 t4 + c % 2
    if constexpr (SCATTER) {
        double f = 1.0;
        if (sc.rr) {
            const double rr = *sc.rr;
            f = (rr > 0.0 && rr < 1e300) ? sqrt(rr) : 1.0;
        }
        double *out = static_cast<double *>(sc.out);
#pragma unroll
        for (int i = 0; i < WI; ++i)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = m0 + wm + 16 * i + g + 8 * h;
                if (row >= sc.rows || row >= tr.mlim) continue;
#pragma unroll
                for (int j = 0; j < 4; ++j)
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const int col = n0 + wn + 8 * j + 2 * t4 + c;
                        if (col < sc.cols && col < tr.nlim) out[(size_t)(row + 1) * sc.ld + col + 1] = f * acc[i][j][2 * h + c];
                    }
            }
    } else {
#pragma unroll
        for (int i = 0; i < WI; ++i)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = m0 + wm + 16 * i + g + 8 * h;
                if (row >= tr.mlim) continue;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int col = n0 + wn + 8 * j + 2 * t4;
                    double *dst = C + (size_t)row * ldc + col;
                    if (col + 1 < tr.nlim)
                        *reinterpret_cast<double2 *>(dst) = make_double2(acc[i][j][2 * h], acc[i][j][2 * h + 1]);
                    else if (col < tr.nlim) dst[0] = acc[i][j][2 * h];
                }
            }
    }
}

namespace {
int g_f64_shape = -1;   // forced CTA shape (timing runs); -1: the default 64 x 64 shape

template <int CFG, bool AMN, bool BMN, bool SCATTER>
int launch_f64(GemmOperand A, GemmOperand B, double *C, int ldc, int M, int N, int K, int Mst, int Nst, cudaStream_t s,
               const GemmScatter &sc, GemmSplit split)
{
    using Cf = DCfg<CFG>;
    constexpr int TM = 16 * Cf::WI * Cf::WMW, TN = 32 * Cf::WNW, NT = 32 * Cf::WMW * Cf::WNW;
    const size_t smem = (size_t)kDS * (DTile<AMN, TM>::elems + DTile<BMN, TN>::elems) * sizeof(double);
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(gemm_f64_kernel<CFG, AMN, BMN, SCATTER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return IGA_ERR_CUDA;
        attr = true;
    }
    const dim3 grid(tiles_along(Mst, TM, split.on_n ? 0 : split.kb), tiles_along(Nst, TN, split.on_n ? split.kb : 0));
    return launch_k(gemm_f64_kernel<CFG, AMN, BMN, SCATTER>, grid, dim3(NT), smem, s,
                    static_cast<const double *>(A.ptr), A.ld, static_cast<const double *>(B.ptr), B.ld, C, ldc, M, N, K,
                    Mst, Nst, sc, split) == cudaSuccess
               ? IGA_OK
               : IGA_ERR_CUDA;
}

template <int CFG>
int launch_f64_layout(GemmOperand A, GemmOperand B, double *C, int ldc, int M, int N, int K, int Mst, int Nst,
                      cudaStream_t s, const GemmScatter &sc, GemmSplit split)
{
    // the two operand layouts the preconditioner uses (both K-major, both MN-major)
    if (!A.mn_major && !B.mn_major && !sc.out)
        return launch_f64<CFG, false, false, false>(A, B, C, ldc, M, N, K, Mst, Nst, s, sc, split);
    if (A.mn_major && B.mn_major) {
        if (sc.out) return launch_f64<CFG, true, true, true>(A, B, C, ldc, M, N, K, Mst, Nst, s, sc, split);
        return launch_f64<CFG, true, true, false>(A, B, C, ldc, M, N, K, Mst, Nst, s, sc, split);
    }
    set_error("FP64 GEMM: this operand layout / output combination is not built");
    return IGA_ERR_UNSUPPORTED;
}
}  // namespace

void gemm_f64_force_shape(int shape) { g_f64_shape = shape; }

int gemm_f64_launch(GemmOperand A, GemmOperand B, double *C, int ldc, int M, int N, int K, int Mst, int Nst,
                    cudaStream_t s, const GemmScatter &sc, GemmSplit split)
{
    if (!(split.kb > 0 && split.kb < K)) split = GemmSplit();
    if ((uintptr_t)A.ptr % 16 || (uintptr_t)B.ptr % 16 || A.ld % 2 || B.ld % 2 || (uintptr_t)C % 16 || ldc % 2 ||
        (sc.out && !sc.f64)) {
        set_error("FP64 GEMM operands need 16-byte aligned rows (and an FP64 scatter target)");
        return IGA_ERR_ARG;
    }
    // 64 x 64 tiles, three CTAs per SM, measured fastest at every size the
    // preconditioner meets (2064^2: 586 us = 30.0 TFLOP/s against 614 us with
    // 128 x 128; 1040^2: 78 us against 158 us; 528^2: 27 against 84 us)
    const int shape = g_f64_shape >= 0 ? g_f64_shape : 2;
    switch (shape) {
    case 0: return launch_f64_layout<0>(A, B, C, ldc, M, N, K, Mst, Nst, s, sc, split);
    case 1: return launch_f64_layout<1>(A, B, C, ldc, M, N, K, Mst, Nst, s, sc, split);
    default: return launch_f64_layout<2>(A, B, C, ldc, M, N, K, Mst, Nst, s, sc, split);
    }
}

}  // namespace iga
