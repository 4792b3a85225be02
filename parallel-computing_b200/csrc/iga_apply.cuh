// Matrix-free IGA Poisson operator y = sign * K x for sm_100a.
//
// Maths (reference: LocalAssemblyMF::LocalMatMulMF, matrix_free/src/LocalAssemblyMF.cpp:31-67,
// and ElementMF, matrix_free/src/ElementMF.cpp:106-296): per element e and
// quadrature point q,
//     y_e += sign * sum_q  grad_xi N^T  G_q  grad_xi u,
//     G_q  = w_q kappa_q det(J) J^-1 J^-T   (symmetric 2x2, 3 values),
// with N the tensor product of the element's 1-D B-spline (or 1-D rational)
// bases, derivatives in reference-element coordinates. The element operator
// is applied by sum factorisation: two 1-D contractions in, a 2x2 multiply per
// quadrature point, two 1-D contractions out.
//
// Work decomposition: a WARP owns a strip of SW = 16 element columns and
// marches over TY element rows. Two lanes share an element column: lane
// 2c + h handles column c and the quadrature columns qx = h*QH + j, j < QH
// (QH = ceil((p+1)/2)). Per row step every lane
//   1. contracts the new control-point row along x for its qx (rolling xs),
//   2. contracts along y with the row's tables (warp-uniform loads),
//   3. applies G: streamed into shared memory by the bulk-copy (TMA) engine
//      (GEOM = 0, the mult_sf path) or computed in registers from the control
//      points by the same rolling sum factorisation (GEOM = 1, the mult_mf path),
//   4. accumulates the y-transposed contraction into rolling row buffers acc,
//   5. finalises the control-point row no later element touches: sums its qx
//      half with the partner lane, then the p+1 neighbouring columns' values
//      with rotate-shuffles.
// Values a strip completes alone are stored to y; values other strips also
// touch (p-wide seams) go to a per-strip frame and are summed in a fixed order
// by seam_fixup_kernel. No atomics: bitwise reproducible.
#pragma once
#include <type_traits>
#include "iga_device.cuh"

namespace iga {

template <typename T>
struct ApplyParams {
    const T *x;
    T *y;
    const T *G;       // GEOM 0: [strip][TY][NQ][NQ][3][SW]
    const T *tabX;    // [NSX][2][QH][NB][32]  (kind 0: value, 1: d/dxi)
    const T *tabY;    // [ney][2][NQ][NBP] (NB values, zero-padded to 16-byte rows)
    const T *CP;      // GEOM 1: (x, y) per control point, in T
    const T *wq;      // GEOM 1: w_qx * w_qy, [NQ*NQ] (qx fastest)
    const T *kappa;   // GEOM 1: per quadrature point or null
    T *frame;         // [NSX*NSY][FS]
    StripGrid g;
    T sign;
    int bc;
    int *err;
    // apply_kernel's window of strip rows: gy0 .. gy0 + gyn - 1 (default: all;
    // a host-buffer MatMult applies the patch slab by slab to overlap copies)
    int gy0 = 0, gyn = 1 << 30;
    // Equation numbers (the reference's ID array, matrix_free_gpu/src/mult.cu:
    // 455-460): when set, control point A's value goes to y[ID[A]] if
    // 0 <= ID[A] < m n and nowhere otherwise (use with bc = 2: every row the
    // full element sum, x read everywhere).
    const int *ID = nullptr;
    // Polls of each wait for a G stage before it reports IGA_ERR_TIMEOUT.
    long long wait_polls = kWaitLimit;
};

// Stores sign * v for control point i = R m + C under boundary rule bc
// (0: y[boundary] = 0, 1: y[boundary] = x[boundary], 2: none) or, when ID is
// set, at equation ID[i] (skipped for ID[i] < 0 or out of range).
template <typename T>
__device__ __forceinline__ void store_point(const StripGrid &g, const T *__restrict__ x, T *__restrict__ y,
                                            const int *__restrict__ ID, T sign, int bc, int R, int C, T v)
{
    const size_t i = (size_t)R * g.m + C;
    if (ID) {
        const int e = ID[i];
        if (e >= 0 && (long long)e < (long long)g.m * g.n) y[e] = sign * v;
        return;
    }
    const bool bnd = bc != 2 && (R == 0 || C == 0 || R == g.n - 1 || C == g.m - 1);
    y[i] = bnd ? (bc == 1 ? x[i] : T(0)) : sign * v;
}

template <int P, typename T>
struct ApplyShape {
    static constexpr int NB = P + 1;
    static constexpr int NQ = P + 1;
    static constexpr int QH = (NQ + 1) / 2;
    static constexpr int NQ2 = NQ * NQ;
    static constexpr int GE = NQ2 * 3 * kSW;            // one row step of G for a warp
    static constexpr int GBYTES = GE * (int)sizeof(T);
    static constexpr int TABX = 2 * QH * NB * 32;       // x tables of a column strip
    static constexpr int XR = 8;                        // x / CP rows in flight per warp
    static constexpr int XW = 24;                       // >= SW + P, padded
    static constexpr int NBP = tab_nbp(NB, (int)sizeof(T));   // y-table row length
    static constexpr int TYW = tab_row_len(NB, NQ, (int)sizeof(T));   // one element row's y tables
    static_assert(GBYTES % 16 == 0, "bulk copy size must be a multiple of 16 bytes");
    static_assert(kSW + P <= XW, "row buffer too narrow");
};

// Stages of each warp's G ring: about 12 KiB per warp (at least 2, at most 8),
// except FP32 at p = 3, where 2 stages (6 KiB) leave room for 16 instead of
// 15 warps per SM (measured 1.13x faster at 2048^2).
template <int P, typename T>
__host__ __device__ constexpr int apply_stages()
{
    return (P == 3 && sizeof(T) == 4) ? 2 : 12288 / ApplyShape<P, T>::GBYTES < 2 ? 2
                                                 : (12288 / ApplyShape<P, T>::GBYTES > 8 ? 8 : 12288 / ApplyShape<P, T>::GBYTES);
}

// Whether a lane keeps its x-direction tables in registers (16 values at
// p = 3) or reads them from shared memory: registers except where they are
// the scarcer resource (FP64 p >= 4, FP64 on-the-fly geometry at p <= 2). In
// registers they save 32 shared loads per element row of a p=3 FP64 strip
// (12 instead of 13 warps per SM: 1.12x faster), and the warps of a CTA need
// not share a column strip, so strips are dealt to warps one by one and every
// SM gets work. The FP64 on-the-fly kernel at p = 3 keeps them in registers
// at 8 warps per SM (244 registers, no spills; shared tables: 10 warps with
// spills): 2048^2 673 -> 536 us, 1024^2 208 -> 149 us. At p = 2 the same
// change was slower (2048^2 392 -> 435 us).
template <int P, typename T, int GEOM>
__host__ __device__ constexpr bool apply_txreg()
{
    return sizeof(T) == 4 || (GEOM == 0 ? P <= 3 : P == 3);
}

// Where the tables are not in registers they are either copied to shared
// memory by a CTA that takes W strips of one column strip, or read by each
// lane straight from global memory (its own entries, L1-resident: a strip's
// tables are a few KB reused for every element row), which lets the kernel
// deal strips to warps one by one and fill the SMs. Measured (B200, warm):
// FP64 p=4 on-the-fly 1024^2 333 -> 302 us from global memory; FP64 p=4
// precomputed 152.6 -> 164.8 us and p=5 (both geometry modes) 249 -> 278 /
// 726 -> 890 us slower that way, so shared memory everywhere else.
template <int P, typename T, int GEOM>
__host__ __device__ constexpr bool apply_txshared()
{
    return !apply_txreg<P, T, GEOM>() && !(GEOM == 1 && P == 4);
}

// The FP64 on-the-fly kernel at p = 5 (255 registers, spilling) keeps one
// CTA per column strip: dealt from the flat grid its spills grew (608 ->
// 880 B a thread) and it ran 187 -> 255 us at 512^2.
template <int P, typename T, int GEOM>
__host__ __device__ constexpr bool apply_percolumn()
{
    return apply_txshared<P, T, GEOM>() && GEOM == 1 && P == 5;
}

// Shared memory of a CTA of W warps: barriers, then each warp's G ring, x
// (and control-point) rows and y-table rows, then (apply_txshared) ntab
// slots of column-strip x tables, 128-byte aligned.
template <int P, typename T, int GEOM, int NST>
__host__ __device__ constexpr size_t apply_tab_offset(int W)
{
    using S = ApplyShape<P, T>;
    return (((256 + (size_t)W * NST * 8 + 127) & ~size_t(127)) + (GEOM == 0 ? (size_t)W * NST * S::GBYTES : 0) +
            (size_t)W * S::XR * S::XW * sizeof(T) * (GEOM == 1 ? 3 : 1) + (size_t)W * S::XR * S::TYW * sizeof(T) +
            127) &
           ~size_t(127);
}

template <int P, typename T, int GEOM, int NST>
__host__ __device__ constexpr size_t apply_smem_bytes(int W, int ntab = 1)
{
    return apply_tab_offset<P, T, GEOM, NST>(W) +
           (apply_txshared<P, T, GEOM>() ? (size_t)ntab * ApplyShape<P, T>::TABX * sizeof(T) : 0);
}

// The CTA's x-table slots in shared memory (apply_txshared kernels).
template <int P, typename T, int GEOM, int NST>
__device__ __forceinline__ T *apply_tab_slots()
{
    extern __shared__ __align__(128) unsigned char smem[];
    return reinterpret_cast<T *>(smem + apply_tab_offset<P, T, GEOM, NST>(blockDim.y));
}

// Copies the x tables of column strips gx0 .. gx0 + n - 1 into the slots (all
// threads of the CTA; the caller synchronises).
template <int P, typename T, int GEOM, int NST>
__device__ __forceinline__ void apply_load_tabs(const T *__restrict__ tabX, int gx0, int n, T *slots)
{
    constexpr int TABX = ApplyShape<P, T>::TABX;
    const int t = threadIdx.y * 32 + threadIdx.x, nt = 32 * blockDim.y;
    for (int k = 0; k < n; ++k) {
        const T *src = tabX + (size_t)(gx0 + k) * TABX;
        for (int i = t; i < TABX; i += nt) slots[(size_t)k * TABX + i] = src[i];
    }
}

template <typename T>
__device__ __forceinline__ T shfl_idx(T v, int src)
{
    return __shfl_sync(0xffffffffu, v, src);
}

// 1 / v for the Jacobian determinant of the on-the-fly geometry (v > 0 and
// far from the extremes of the exponent range). FP64: the hardware's
// approximate reciprocal (rcp.approx.ftz.f64) refined by two Newton-Raphson
// steps y <- y + y (1 - v y), each of which squares the relative error, so
// the result is within a few units in the last place of 1 / v; five FP64
// instructions in place of the correctly rounded reciprocal's longer
// sequence with its special-case branch. The operator is checked against
// the oracle at 1e-12 relative.
template <typename T>
__device__ __forceinline__ T recip(T v);
template <>
__device__ __forceinline__ double recip<double>(double v)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(v));
    double e = fma(-v, y, 1.0);
    y = fma(y, e, y);
    e = fma(-v, y, 1.0);
    return fma(y, e, y);
}
template <>
__device__ __forceinline__ float recip<float>(float v) { return __frcp_rn(v); }

// Threads per CTA the register budget allows (one CTA per SM): the kernel's
// per-thread state grows with p and doubles in FP64. FP64 precomputed p >= 4
// runs 8 warps without register spills (at 10 warps it spilled and ran 1.8x
// slower at p = 4); the FP64 on-the-fly kernels at p >= 4 need more than the
// 255 registers a thread can have and spill at any bound.
template <int P, typename T, int GEOM>
__host__ __device__ constexpr int apply_max_threads()
{
    return sizeof(T) == 4 ? (P <= 3 ? 512 : (GEOM ? 384 : 512))
                          : (P <= 2 ? (GEOM ? 384 : 512) : P == 3 ? (GEOM ? 256 : 384) : 256);
}

// One warp: strip (gx, gy). tab_slot: the slot of the CTA's shared memory
// holding the column strip's x tables (apply_txshared), loaded by the caller.
template <int P, typename T, int GEOM, int NST>
__device__ __forceinline__ void apply_tile(const ApplyParams<T> &a, const T *__restrict__ x, T *__restrict__ y, const int gx,
                                           const int gy, const int tab_slot)
{
    using S = ApplyShape<P, T>;
    constexpr int NB = S::NB, NQ = S::NQ, QH = S::QH;
    constexpr bool TXREG = apply_txreg<P, T, GEOM>();
    const StripGrid &g = a.g;
    const int lane = threadIdx.x, w = threadIdx.y, W = blockDim.y;
    const int c = lane >> 1, h = lane & 1;

    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    size_t off = 256 + (size_t)W * NST * 8;
    off = (off + 127) & ~size_t(127);
    T *Gs = reinterpret_cast<T *>(smem + off) + (size_t)w * NST * S::GE;
    if (GEOM == 0) off += (size_t)W * NST * S::GBYTES;
    T *xr = reinterpret_cast<T *>(smem + off) + (size_t)w * S::XR * S::XW;
    off += (size_t)W * S::XR * S::XW * sizeof(T);
    T *cr = reinterpret_cast<T *>(smem + off) + (size_t)w * S::XR * S::XW * 2;   // GEOM 1: CP rows (x, y)
    if (GEOM == 1) off += (size_t)W * S::XR * S::XW * 2 * sizeof(T);
    T *yr = reinterpret_cast<T *>(smem + off) + (size_t)w * S::XR * S::TYW;     // y tables of upcoming rows
    uint64_t *wbar = bars + w * NST;
    // (addressed from the shared array itself, so that the compiler emits shared loads)
    const T *tabXs = reinterpret_cast<const T *>(smem + apply_tab_offset<P, T, GEOM, NST>(W)) + (size_t)tab_slot * S::TABX;

    if (gx >= g.NSX || gy >= g.NSY) return;
    const int ex0 = kSW * gx, ey0 = g.TY * gy;
    const int nsteps = min(g.TY, g.ney - ey0);
    if (nsteps <= 0) return;
    const int ex = ex0 + c;
    const T *Gstrip = GEOM == 0 ? a.G + (size_t)(gx * g.NSY + gy) * g.TY * S::GE : nullptr;

    if (GEOM == 0) {
        if (lane == 0) {
            for (int i = 0; i < NST; ++i) mbar_init(&wbar[i], 1);
            fence_mbar_init();
        }
        __syncwarp();
        if (lane == 0)
            for (int s = 0; s < NST && s < nsteps; ++s) {
                mbar_arrive_expect_tx(&wbar[s], S::GBYTES);
                bulk_g2s(Gs + (size_t)s * S::GE, Gstrip + (size_t)s * S::GE, S::GBYTES, &wbar[s]);
            }
    }

    // Control-point rows consumed in order k = 0, 1, ... (row ey0 + k); lanes
    // 0 .. SW+P-1 each fetch one column (zero outside the patch). The same
    // group brings the y tables of element row ey0 + k - P, used at step k - P.
    const int nrows = nsteps + P;
    auto fetch_row = [&](int k) {
        if (k < nrows && lane < kSW + P) {
            const int R = ey0 + k, C = ex0 + lane;
            const bool v = R < g.n && C < g.m;
            // IGA_BC_IDENTITY: boundary entries of x enter the operator as zero
            const bool xb = a.bc == 1 && (R == 0 || C == 0 || R == g.n - 1 || C == g.m - 1);
            const size_t gi = v ? (size_t)R * g.m + C : 0;
            cp_async_zfill<sizeof(T)>(xr + (k % S::XR) * S::XW + lane, x + gi, v && !xb);
            if (GEOM == 1) cp_async_zfill<2 * sizeof(T)>(cr + ((k % S::XR) * S::XW + lane) * 2, a.CP + 2 * gi, v);
        }
        if (k >= P && k < nrows) {   // 16-byte copies (rows are whole 16-byte words)
            constexpr int CH = S::TYW * (int)sizeof(T) / 16;
            const unsigned char *src = reinterpret_cast<const unsigned char *>(a.tabY + (size_t)(ey0 + k - P) * S::TYW);
            unsigned char *dst = reinterpret_cast<unsigned char *>(yr + (k % S::XR) * S::TYW);
            for (int t = lane; t < CH; t += 32) cp_async_zfill<16>(dst + 16 * t, src + 16 * t, true);
        }
        cp_async_commit();
    };
    constexpr int D = S::XR - 1;

    // This lane's x-direction tables, [kind][j][il][lane] per column strip
    // (apply_txreg: registers, loaded straight from global memory; else the
    // CTA's shared copy). The FP32 precomputed-geometry kernel at p <= 3
    // (PAIR) keeps them as (derivative, value) pairs and forms both kinds of
    // every 1-D contraction with one packed f32x2 FMA (sm_100). Measured
    // (B200, FP32, cold L2): p=2 2048^2 157 -> 146 us, p=3 181 -> 175 us; at
    // p = 4, 5 the pairs' registers spill (83 -> 97 us, 144 -> 216 us), and
    // the on-the-fly kernels were slower too (p=3 1024^2 87 -> 101 us), so
    // those keep scalar FMAs (reading paired y tables up to p = 4: on-the-fly
    // p=3 1024^2 87 -> 85 us, p=2 62.4 -> 60.4 us).
    constexpr bool TPAIR = tab_paired(NB, (int)sizeof(T));
    constexpr bool PAIR = TPAIR && GEOM == 0 && P <= 3;
    static_assert(!PAIR || TXREG, "FP32 x tables live in registers");
    T txr[TXREG && !PAIR ? 2 : 1][TXREG && !PAIR ? QH : 1][TXREG && !PAIR ? NB : 1];
    float2 tpr[PAIR ? QH : 1][PAIR ? NB : 1];
    if constexpr (PAIR) {
        const T *src = a.tabX + (size_t)gx * S::TABX;
#pragma unroll
        for (int j = 0; j < QH; ++j)
#pragma unroll
            for (int il = 0; il < NB; ++il)
                tpr[j][il] = make_float2(src[((QH + j) * NB + il) * 32 + lane], src[(j * NB + il) * 32 + lane]);
    } else if constexpr (TXREG) {
        const T *src = a.tabX + (size_t)gx * S::TABX;
#pragma unroll
        for (int kind = 0; kind < 2; ++kind)
#pragma unroll
            for (int j = 0; j < QH; ++j)
#pragma unroll
                for (int il = 0; il < NB; ++il) txr[kind][j][il] = src[((kind * QH + j) * NB + il) * 32 + lane];
    }
    const T *txg = a.tabX + (size_t)gx * S::TABX + lane;
    auto tx = [&](int kind, int j, int il) -> T {
        if constexpr (PAIR) return kind ? tpr[j][il].x : tpr[j][il].y;
        else if constexpr (TXREG) return txr[kind][j][il];
        else if constexpr (apply_txshared<P, T, GEOM>()) return tabXs[((kind * QH + j) * NB + il) * 32 + lane];
        else return __ldg(txg + ((kind * QH + j) * NB + il) * 32);
    };
    // Everything above reads only the plan's constant tables and geometry;
    // x (an earlier grid's output) and every write come after the wait.
    pdl_wait();
    for (int k = 0; k < D; ++k) fetch_row(k);

    constexpr int NR = PAIR ? 1 : NB;
    T xs0[NR][QH], xs1[NR][QH];     // x contracted with value / derivative tables, rows ey..ey+P
    T acc0[NR][QH], acc1[NR][QH];   // y-transposed partial sums for control-point rows ey..ey+P
    T cs[2][2][GEOM == 1 && !PAIR ? NB : 1][QH];   // GEOM 1: CP coordinates contracted likewise
    // PAIR: X = (xs1, xs0), A = (acc0, acc1), CX = (cs[0][1], cs[0][0]), CY = (cs[1][1], cs[1][0])
    float2 X[PAIR ? NB : 1][QH], A[PAIR ? NB : 1][QH];
    float2 CX[PAIR && GEOM == 1 ? NB : 1][QH], CY[PAIR && GEOM == 1 ? NB : 1][QH];

    // x contraction of control-point row k into state row `slot` (0 .. P)
    auto contract_row = [&](int k, int slot) {
        cp_async_wait<D - 1>();
        __syncwarp();
        const T *src = xr + (k % S::XR) * S::XW;
        T xv[NB];
#pragma unroll
        for (int il = 0; il < NB; ++il) xv[il] = src[c + il];
        T px[NB], py[NB];
        if constexpr (GEOM == 1) {
            const T *cp = cr + (k % S::XR) * S::XW * 2;
#pragma unroll
            for (int il = 0; il < NB; ++il) {
                px[il] = cp[2 * (c + il)];
                py[il] = cp[2 * (c + il) + 1];
            }
        }
        __syncwarp();
        fetch_row(k + D);
        if constexpr (PAIR) {
#pragma unroll
            for (int j = 0; j < QH; ++j) {
                float2 s2 = __fmul2_rn(tpr[j][0], make_float2(xv[0], xv[0]));
#pragma unroll
                for (int il = 1; il < NB; ++il) s2 = __ffma2_rn(tpr[j][il], make_float2(xv[il], xv[il]), s2);
                X[slot][j] = s2;
            }
            if constexpr (GEOM == 1) {
#pragma unroll
                for (int j = 0; j < QH; ++j) {
                    float2 ax = __fmul2_rn(tpr[j][0], make_float2(px[0], px[0]));
                    float2 ay = __fmul2_rn(tpr[j][0], make_float2(py[0], py[0]));
#pragma unroll
                    for (int il = 1; il < NB; ++il) {
                        ax = __ffma2_rn(tpr[j][il], make_float2(px[il], px[il]), ax);
                        ay = __ffma2_rn(tpr[j][il], make_float2(py[il], py[il]), ay);
                    }
                    CX[slot][j] = ax;
                    CY[slot][j] = ay;
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < QH; ++j) {
                T s0 = 0, s1 = 0;
#pragma unroll
                for (int il = 0; il < NB; ++il) {
                    s0 = fma(tx(0, j, il), xv[il], s0);
                    s1 = fma(tx(1, j, il), xv[il], s1);
                }
                xs0[slot][j] = s0;
                xs1[slot][j] = s1;
            }
            if constexpr (GEOM == 1) {
#pragma unroll
                for (int j = 0; j < QH; ++j) {
                    T a0 = 0, a1 = 0, b0 = 0, b1 = 0;
#pragma unroll
                    for (int il = 0; il < NB; ++il) {
                        a0 = fma(tx(0, j, il), px[il], a0);
                        a1 = fma(tx(1, j, il), px[il], a1);
                        b0 = fma(tx(0, j, il), py[il], b0);
                        b1 = fma(tx(1, j, il), py[il], b1);
                    }
                    cs[0][0][slot][j] = a0;
                    cs[0][1][slot][j] = a1;
                    cs[1][0][slot][j] = b0;
                    cs[1][1][slot][j] = b1;
                }
            }
        }
    };

    auto store = [&](int R, int C, T v) { store_point<T>(g, x, y, a.ID, a.sign, a.bc, R, C, v); };
    T *frame = a.frame + (size_t)(gx * g.NSY + gy) * g.FS;
    // finishes control-point row ey0 + lr from state row 0 of the partial sums
    auto write_row = [&](int lr) {
        T out[NB];
#pragma unroll
        for (int il = 0; il < NB; ++il) {
            T s = 0;
            if constexpr (PAIR) {   // the derivative-table and value-table sums, then their total
                float2 s2 = __fmul2_rn(tpr[0][il], A[0][0]);
#pragma unroll
                for (int j = 1; j < QH; ++j) s2 = __ffma2_rn(tpr[j][il], A[0][j], s2);
                s = s2.x + s2.y;
            } else {
#pragma unroll
                for (int j = 0; j < QH; ++j) {
                    s = fma(tx(1, j, il), acc0[0][j], s);
                    s = fma(tx(0, j, il), acc1[0][j], s);
                }
            }
            out[il] = s + __shfl_xor_sync(0xffffffffu, s, 1);   // both qx halves, same order on both lanes
        }
        // Column c collects out[il] from column c-il (lane - 2 il); lanes of
        // columns c < il receive the wrapped value, which belongs to column SW+c.
        T tot = out[0], spill = 0;
#pragma unroll
        for (int il = 1; il < NB; ++il) {
            const T v = shfl_idx(out[il], (lane - 2 * il) & 31);
            if (c >= il) tot += v;
            else spill += v;
        }
        const int R = ey0 + lr;
        if (R >= g.n) return;
        // Strips covering row R / column C (closed form of cover()): the
        // first P rows/columns of a strip are shared with the strip before
        // it (if any), the P rows/columns past its end with the one after it.
        const bool row_single = lr < g.TY ? (lr >= P || gy == 0) : (gy + 1 >= g.NSY);
        const int lc = h ? kSW + c : c;
        const int C = ex0 + lc;
        if ((h == 0 || c < P) && C < g.m) {
            const T v = h ? spill : tot;
            const bool col_single = h ? (gx + 1 >= g.NSX) : (c >= P || gx == 0);
            if (row_single && col_single) store(R, C, v);
            else frame[frame_index(lr, lc, P, g.TY)] = v;
        }
    };

    // Prologue: rows ey0 .. ey0+P-1.
#pragma unroll
    for (int r = 0; r < P; ++r) contract_row(r, r);
#pragma unroll
    for (int r = 0; r < NB; ++r)
#pragma unroll
        for (int q = 0; q < QH; ++q) {
            if constexpr (PAIR) A[r][q] = make_float2(0.f, 0.f);
            else acc0[r][q] = acc1[r][q] = 0;
        }
    // state rows r+1 -> r (the next element row); the partial sums of row P restart
    auto shift_rows = [&](bool inputs) {
#pragma unroll
        for (int r = 0; r < P; ++r)
#pragma unroll
            for (int q = 0; q < QH; ++q) {
                if constexpr (PAIR) {
                    A[r][q] = A[r + 1][q];
                    if (inputs) {
                        X[r][q] = X[r + 1][q];
                        if constexpr (GEOM == 1) {
                            CX[r][q] = CX[r + 1][q];
                            CY[r][q] = CY[r + 1][q];
                        }
                    }
                } else {
                    acc0[r][q] = acc0[r + 1][q];
                    acc1[r][q] = acc1[r + 1][q];
                    if (inputs) {
                        xs0[r][q] = xs0[r + 1][q];
                        xs1[r][q] = xs1[r + 1][q];
                        if constexpr (GEOM == 1) {
                            cs[0][0][r][q] = cs[0][0][r + 1][q];
                            cs[0][1][r][q] = cs[0][1][r + 1][q];
                            cs[1][0][r][q] = cs[1][0][r + 1][q];
                            cs[1][1][r][q] = cs[1][1][r + 1][q];
                        }
                    }
                }
            }
#pragma unroll
        for (int q = 0; q < QH; ++q) {
            if constexpr (PAIR) A[P][q] = make_float2(0.f, 0.f);
            else acc0[P][q] = acc1[P][q] = 0;
        }
    };

    bool ok = true;
    int failed_step = 0;
    for (int s = 0; s < nsteps; ++s) {
        const int ey = ey0 + s;
        contract_row(s + P, P);
        const int slot = s % NST;
        const T *Gst = Gs + (size_t)slot * S::GE;
        if (GEOM == 0) {
            if (!mbar_wait_bounded(&wbar[slot], (uint32_t)((s / NST) & 1), a.wait_polls)) {
                ok = false;
                failed_step = s;
                break;
            }
        }
        const T *ty = yr + ((s + P) % S::XR) * S::TYW;   // landed with x row s + P
        constexpr bool MID = mid_shared(NQ, (int)sizeof(T));
        constexpr int QJ = MID ? QH - 1 : QH;   // slots of this lane half's own columns
        // y tables of quadrature row qy: value n2 and derivative d2, or their
        // pairs nd (PAIR)
        struct YRow {
            T n2[PAIR ? 1 : NB], d2[PAIR ? 1 : NB];
            float2 nd[PAIR ? NB : 1];
        };
        auto load_tab = [&](int qy, YRow &t) {
            if constexpr (PAIR) {   // rows of NB pairs padded to 16 bytes: two pairs per vector load
                const float4 *v = reinterpret_cast<const float4 *>(ty + qy * tab_nbp2(NB));
#pragma unroll
                for (int u = 0; 2 * u < NB; ++u) {
                    const float4 q = v[u];
                    t.nd[2 * u] = make_float2(q.x, q.y);
                    if (2 * u + 1 < NB) t.nd[2 * u + 1] = make_float2(q.z, q.w);
                }
            } else if constexpr (TPAIR) {   // the same rows, split into the two kinds
                const float4 *v = reinterpret_cast<const float4 *>(ty + qy * tab_nbp2(NB));
#pragma unroll
                for (int u = 0; 2 * u < NB; ++u) {
                    const float4 q = v[u];
                    t.n2[2 * u] = q.x;
                    t.d2[2 * u] = q.y;
                    if (2 * u + 1 < NB) {
                        t.n2[2 * u + 1] = q.z;
                        t.d2[2 * u + 1] = q.w;
                    }
                }
            } else {
                // rows of NBP entries, 16-byte aligned in the ring: vector loads
                constexpr int V = 16 / sizeof(T), NBP = S::NBP;
                using VT = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
                const VT *va = reinterpret_cast<const VT *>(ty + qy * NBP);
                const VT *vb = reinterpret_cast<const VT *>(ty + (NQ + qy) * NBP);
#pragma unroll
                for (int v = 0; v < NBP / V; ++v) {
                    const VT ua = va[v], ub = vb[v];
                    const T *pa = reinterpret_cast<const T *>(&ua), *pb = reinterpret_cast<const T *>(&ub);
#pragma unroll
                    for (int e = 0; e < V; ++e) {
                        if (v * V + e < NB) {
                            t.n2[v * V + e] = pa[e];
                            t.d2[v * V + e] = pb[e];
                        }
                    }
                }
            }
        };
        // quadrature point (qy, qx) in slot j: gradient of u, times G, back
        // onto the slot's y-transposed partial sums (valid false: adds zero)
        // gv: this lane's G values of row qy (lane-major G), else read here
        auto qpoint = [&](int qy, int qx, int j, bool valid, const YRow &t, const T *gv) {
            T uxi = 0, ueta = 0;
            if constexpr (PAIR) {   // (n2 . xs1, d2 . xs0) together
                float2 u2 = __fmul2_rn(t.nd[0], X[0][j]);
#pragma unroll
                for (int jl = 1; jl < NB; ++jl) u2 = __ffma2_rn(t.nd[jl], X[jl][j], u2);
                uxi = u2.x;
                ueta = u2.y;
            } else {
#pragma unroll
                for (int jl = 0; jl < NB; ++jl) {
                    uxi = fma(t.n2[jl], xs1[jl][j], uxi);
                    ueta = fma(t.d2[jl], xs0[jl][j], ueta);
                }
            }
            T g00 = 0, g01 = 0, g11 = 0;
            T vxi, veta;
            if constexpr (GEOM == 0) {
                if constexpr (g_lane_major(NQ)) {
                    g00 = gv[3 * j];
                    g01 = gv[3 * j + 1];
                    g11 = gv[3 * j + 2];
                } else if constexpr (g_mid_lane_major(NQ, (int)sizeof(T))) {
                    if (j + 1 < QH) {   // a column of this lane half
                        g00 = gv[3 * j];
                        g01 = gv[3 * j + 1];
                        g11 = gv[3 * j + 2];
                    } else if (valid) {   // the middle column, row qy of this half
                        const T *gp = Gst + qy * (NQ * 3 * kSW) + 32 * (QH - 1) * 3 + c * 3;
                        g00 = gp[0];
                        g01 = gp[1];
                        g11 = gp[2];
                    }
                } else if (valid) {
                    const T *gp = Gst + ((qy * NQ + qx) * 3) * kSW + c;
                    g00 = gp[0];
                    g01 = gp[kSW];
                    g11 = gp[2 * kSW];
                }
            } else {
                T x_xi = 0, x_eta = 0, y_xi = 0, y_eta = 0;
                if constexpr (PAIR) {
                    float2 cx = __fmul2_rn(t.nd[0], CX[0][j]), cy = __fmul2_rn(t.nd[0], CY[0][j]);
#pragma unroll
                    for (int jl = 1; jl < NB; ++jl) {
                        cx = __ffma2_rn(t.nd[jl], CX[jl][j], cx);
                        cy = __ffma2_rn(t.nd[jl], CY[jl][j], cy);
                    }
                    x_xi = cx.x;
                    x_eta = cx.y;
                    y_xi = cy.x;
                    y_eta = cy.y;
                } else {
#pragma unroll
                    for (int jl = 0; jl < NB; ++jl) {
                        x_xi = fma(t.n2[jl], cs[0][1][jl][j], x_xi);
                        x_eta = fma(t.d2[jl], cs[0][0][jl][j], x_eta);
                        y_xi = fma(t.n2[jl], cs[1][1][jl][j], y_xi);
                        y_eta = fma(t.d2[jl], cs[1][0][jl][j], y_eta);
                    }
                }
                // G grad u = f adj(J) adj(J)^T grad u with adj(J) = [[y_eta,
                // -x_eta], [-y_xi, x_xi]] and f = w kappa / det J: ten
                // operations instead of forming G's three entries (thirteen)
                vxi = veta = 0;
                if (valid && ex < g.nex) {
                    T wgt = a.wq[qy * NQ + qx];
                    if (a.kappa) wgt *= a.kappa[((size_t)ey * g.nex + ex) * S::NQ2 + qy * NQ + qx];
                    const T f = wgt * recip(x_xi * y_eta - x_eta * y_xi);
                    const T t0 = f * fma(y_eta, uxi, -(y_xi * ueta));
                    const T t1 = f * fma(x_xi, ueta, -(x_eta * uxi));
                    vxi = fma(y_eta, t0, -(x_eta * t1));
                    veta = fma(x_xi, t1, -(y_xi * t0));
                }
            }
            if constexpr (GEOM == 0) {
                vxi = fma(g00, uxi, g01 * ueta);
                veta = fma(g01, uxi, g11 * ueta);
            }
            if constexpr (PAIR) {   // (acc0 += n2 vxi, acc1 += d2 veta) together
                const float2 v2 = make_float2(vxi, veta);
#pragma unroll
                for (int jl = 0; jl < NB; ++jl) A[jl][j] = __ffma2_rn(t.nd[jl], v2, A[jl][j]);
            } else {
#pragma unroll
                for (int jl = 0; jl < NB; ++jl) {
                    acc0[jl][j] = fma(t.n2[jl], vxi, acc0[jl][j]);
                    acc1[jl][j] = fma(t.d2[jl], veta, acc1[jl][j]);
                }
            }
        };

#pragma unroll
        for (int qy = 0; qy < NQ; ++qy) {
            YRow t;
            load_tab(qy, t);
            // this lane's G values of row qy for its own columns: 3 QJ contiguous
            // values (lane-major G rows), widest aligned loads
            constexpr int GVN = (g_lane_major(NQ) || g_mid_lane_major(NQ, (int)sizeof(T))) ? 3 * QJ : 1;
            T gv[GVN];
            if constexpr (GEOM == 0 && GVN > 1) {
                const T *src = Gst + (size_t)qy * (NQ * 3 * kSW) + (size_t)lane * GVN;
                constexpr int BYTES = GVN * (int)sizeof(T);
                constexpr int VB = BYTES % 16 == 0 ? 16 : BYTES % 8 == 0 ? 8 : (int)sizeof(T);
                using VT = typename std::conditional<VB == 16, float4, typename std::conditional<VB == 8, float2, T>::type>::type;
#pragma unroll
                for (int v = 0; v < BYTES / VB; ++v) {
                    const VT u = reinterpret_cast<const VT *>(src)[v];
                    const T *pu = reinterpret_cast<const T *>(&u);
#pragma unroll
                    for (int e = 0; e < VB / (int)sizeof(T); ++e) gv[v * (VB / (int)sizeof(T)) + e] = pu[e];
                }
            }
#pragma unroll
            for (int j = 0; j < QJ; ++j) {
                const int qx = h * QH + j;   // only h = 1's last slot can lie past NQ
                qpoint(qy, qx, j, (NQ % 2 == 0 || j + 1 < QH) || qx < NQ, t, gv);
            }
        }
        if constexpr (MID) {   // middle column QH - 1: half h takes rows qy = 2 t + h
#pragma unroll
            for (int tq = 0; tq < QH; ++tq) {
                const int qy = min(2 * tq + h, NQ - 1);
                YRow t;
                load_tab(qy, t);
                qpoint(qy, QH - 1, QH - 1, 2 * tq + h < NQ, t, nullptr);
            }
        }
        if (GEOM == 0) {
            __syncwarp();
            if (lane == 0 && s + NST < nsteps) {
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&wbar[slot], S::GBYTES);
                bulk_g2s(Gs + (size_t)slot * S::GE, Gstrip + (size_t)(s + NST) * S::GE, S::GBYTES, &wbar[slot]);
            }
        }
        write_row(s);
        shift_rows(true);
    }
    if (!ok) {
        if (lane == 0) atomicExch(a.err, 8 /* IGA_ERR_TIMEOUT */);
        // Let the copies already issued (steps failed_step .. failed_step+NST-1)
        // land before the CTA's shared memory is released; bounded as well,
        // always with the full poll limit.
        for (int t = failed_step; t < nsteps && t < failed_step + NST; ++t)
            mbar_wait_bounded(&wbar[t % NST], (uint32_t)((t / NST) & 1));
        cp_async_wait<0>();
        return;
    }
    // Rows above the last element row: partial sums for rows ey_last+1 .. ey_last+P.
#pragma unroll
    for (int r = 0; r < P; ++r) {
        write_row(nsteps + r);
        shift_rows(false);
    }
    cp_async_wait<0>();
}

// Strips to warps: warp k of the 1-D grid takes strip k in column-major
// order (gx outer), so the grid covers NSX * rows strips with no partly idle
// CTAs and the strip height can make the strip count fill the SMs. With the
// tables in shared memory (apply_txshared) the CTA copies the tables of the
// column strips its warps' strips lie in: two slots, as the launch keeps W - 1
// <= rows. (One CTA per column strip, W strips of it each, left 20 of 148
// SMs idle for the FP64 p=4 operator on a 1024-wide patch: 64 columns.)
template <int P, typename T, int GEOM, int NST>
__global__ void __launch_bounds__(apply_max_threads<P, T, GEOM>(), 1) apply_kernel(ApplyParams<T> a)
{
    pdl_launch();   // apply_tile waits for the preceding grid once its constant operands are in flight
    const int rows = min(a.gyn, a.g.NSY - a.gy0);   // strip rows of the window
    if constexpr (apply_percolumn<P, T, GEOM>()) {   // CTA = W strips of column strip blockIdx.x
        apply_load_tabs<P, T, GEOM, NST>(a.tabX, blockIdx.x, 1, apply_tab_slots<P, T, GEOM, NST>());
        __syncthreads();
        const int r = blockIdx.y * blockDim.y + threadIdx.y;
        apply_tile<P, T, GEOM, NST>(a, a.x, a.y, blockIdx.x, r < rows ? a.gy0 + r : a.g.NSY, 0);
        return;
    }
    const int s0 = blockIdx.x * blockDim.y, sid = s0 + threadIdx.y;   // strips: NSX * NSY < 2^31
    const int gx = sid / rows;
    int slot = 0;
    if constexpr (apply_txshared<P, T, GEOM>()) {
        const int total = a.g.NSX * rows;
        const int gx_lo = s0 / rows, gx_hi = (min(s0 + (int)blockDim.y, total) - 1) / rows;
        apply_load_tabs<P, T, GEOM, NST>(a.tabX, gx_lo, gx_hi - gx_lo + 1, apply_tab_slots<P, T, GEOM, NST>());
        __syncthreads();
        if (sid >= total) return;
        slot = gx - gx_lo;
    }
    apply_tile<P, T, GEOM, NST>(a, a.x, a.y, gx, a.gy0 + (sid - gx * rows), slot);
}

// Many independent patches in one launch, with that problem's parameters
// per work item, or nothing when the problem is marked inactive (converged)
// or the item is padding (problem -1). Tables in registers (apply_txreg):
// warp k of the grid runs strip items[k] = (problem, column strip, strip
// row), so the warps of a CTA may take strips of different problems and
// columns; else CTA b runs items[b] = (problem, column strip, block of W
// strips of that column).
template <int P, typename T, int NST>
__global__ void __launch_bounds__(apply_max_threads<P, T, 0>(), 1)
    apply_batch_kernel(const ApplyParams<T> *__restrict__ params, const int4 *__restrict__ items,
                       const int *__restrict__ active, const long long *__restrict__ offs, const T *__restrict__ xb,
                       T *__restrict__ yb)
{
    constexpr bool flat = !apply_txshared<P, T, 0>();
    const int4 it = items[flat ? blockIdx.x * blockDim.y + threadIdx.y : blockIdx.x];
    if (it.x < 0 || !active[it.x]) return;   // uniform over the CTA unless flat (no CTA barrier then)
    const long long o = offs[it.x];
    if constexpr (!flat) {   // the item's column strip, slot 0
        apply_load_tabs<P, T, 0, NST>(params[it.x].tabX, it.y, 1, apply_tab_slots<P, T, 0, NST>());
        __syncthreads();
    }
    apply_tile<P, T, 0, NST>(params[it.x], xb + o, yb + o, it.y, flat ? it.z : it.z * blockDim.y + threadIdx.y, 0);
}

// Sums the frames of the strips covering each seam control point, strip
// (row, then column) in ascending order, and stores sign * sum (boundary
// rules as in apply_kernel: bc 0 zero, 1 identity, 2 none). idx enumerates the seam points of grid g.
// The seam control point (R, C): the covering strips' frame values summed
// in fixed strip order, stored with the boundary rule.
template <int P, typename T>
__device__ __forceinline__ void seam_point_rc(const T *__restrict__ frame, const T *__restrict__ x, T *__restrict__ y,
                                              const StripGrid &g, T sign, int bc, const int *__restrict__ ID, int R,
                                              int C)
{
    int fa, fb;
    const int ca = cover(C, kSW, g.NSX, P, fa);
    const int cb = cover(R, g.TY, g.NSY, P, fb);
    T v = 0;
    for (int bi = 0; bi < cb; ++bi) {
        const int b = fb + bi;
        for (int ai = 0; ai < ca; ++ai) {
            const int aa = fa + ai;
            v += frame[(size_t)(aa * g.NSY + b) * g.FS + frame_index(R - g.TY * b, C - kSW * aa, P, g.TY)];
        }
    }
    store_point<T>(g, x, y, ID, sign, bc, R, C, v);
}

template <int P, typename T>
__device__ __forceinline__ void seam_point(const T *__restrict__ frame, const T *__restrict__ x, T *__restrict__ y,
                                           const StripGrid &g, T sign, int bc, const int *__restrict__ ID,
                                           long long idx)
{
    const long long per = (long long)g.n * P;            // points of one vertical seam
    const long long nV = (long long)(g.NSX - 1) * per;
    int R, C;
    if (idx < nV) {
        // seam by seam, row by row, its P columns fastest: consecutive
        // threads read consecutive slots of the two strips' frames
        const int cg = (int)(idx / per);
        const int rem = (int)(idx - cg * per);
        R = rem / P;
        C = kSW * (1 + cg) + rem % P;
        if (C >= g.m) return;
    } else {
        const long long j = idx - nV;
        C = (int)(j % g.m);
        const int rid = (int)(j / g.m);
        R = g.TY * (1 + rid / P) + rid % P;
        if (R >= g.n) return;
        const int s = C / kSW;
        if (C % kSW < P && s >= 1 && s < g.NSX) return;   // handled as a vertical seam
    }
    seam_point_rc<P, T>(frame, x, y, g, sign, bc, ID, R, C);
}

// The seam points of control-point rows R0 .. R1 - 1, where R0 = TY * s0 is a
// strip-row boundary: the vertical seams' points in those rows and the
// horizontal seams TY * s .. TY * s + P - 1 for 1 <= s, s0 <= s, TY * s < R1.
// Valid once every strip covering those rows has written its frame.
template <int P, typename T>
__global__ void seam_fixup_rows_kernel(const T *__restrict__ frame, const T *__restrict__ x, T *__restrict__ y,
                                       StripGrid g, T sign, int bc, int R0, int R1, const int *__restrict__ ID)
{
    const int s0 = max(R0 / g.TY, 1), s1 = (R1 + g.TY - 1) / g.TY;   // horizontal seams s0 .. s1 - 1
    const long long nv = (long long)(g.NSX - 1) * P * (R1 - R0);
    const long long nh = (long long)max(0, min(s1, g.NSY) - s0) * P * g.m;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < nv + nh;
         idx += (long long)gridDim.x * blockDim.x) {
        int R, C;
        if (idx < nv) {   // seam by seam, row by row, its P columns fastest
            const long long per = (long long)(R1 - R0) * P;
            const int cg = (int)(idx / per);
            const int rem = (int)(idx - cg * per);
            R = R0 + rem / P;
            C = kSW * (1 + cg) + rem % P;
            if (C >= g.m) continue;
        } else {
            const long long j = idx - nv;
            C = (int)(j % g.m);
            const int rid = (int)(j / g.m);
            R = g.TY * (s0 + rid / P) + rid % P;
            if (R >= R1 || R >= g.n) continue;
            const int s = C / kSW;
            if (C % kSW < P && s >= 1 && s < g.NSX) continue;   // a vertical seam's point
        }
        seam_point_rc<P, T>(frame, x, y, g, sign, bc, ID, R, C);
    }
}

__host__ __device__ __forceinline__ long long seam_count(const StripGrid &g)
{
    return (long long)(g.NSX - 1) * g.P * g.n + (long long)(g.NSY - 1) * g.P * g.m;
}

template <int P, typename T>
__global__ void seam_fixup_kernel(const T *__restrict__ frame, const T *__restrict__ x, T *__restrict__ y,
                                  StripGrid g, T sign, int bc, const int *__restrict__ ID)
{
    pdl_begin();
    const long long total = seam_count(g);
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x)
        seam_point<P, T>(frame, x, y, g, sign, bc, ID, idx);
}

template <int P, typename T>
__device__ __forceinline__ void seam_loop(const ApplyParams<T> &a, const T *__restrict__ x, T *__restrict__ y)
{
    const long long total = seam_count(a.g);
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x)
        seam_point<P, T>(a.frame, x, y, a.g, a.sign, a.bc, a.ID, idx);
}

// Seams of every active problem of a batch: blockIdx.y = problem.
template <typename T>
__global__ void seam_fixup_batch_kernel(const ApplyParams<T> *__restrict__ params, const int *__restrict__ active,
                                        const long long *__restrict__ offs, const T *__restrict__ xb,
                                        T *__restrict__ yb)
{
    const int pr = blockIdx.y;
    if (!active[pr]) return;
    const ApplyParams<T> &a = params[pr];
    const long long o = offs[pr];
    switch (a.g.P) {
    case 1: seam_loop<1, T>(a, xb + o, yb + o); break;
    case 2: seam_loop<2, T>(a, xb + o, yb + o); break;
    case 3: seam_loop<3, T>(a, xb + o, yb + o); break;
    case 4: seam_loop<4, T>(a, xb + o, yb + o); break;
    default: seam_loop<5, T>(a, xb + o, yb + o); break;
    }
}

}  // namespace iga
