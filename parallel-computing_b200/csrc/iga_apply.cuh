// Matrix-free IGA Poisson operator y = sign * K x for sm_100a.
//
// Maths (reference: LocalAssemblyMF::LocalMatMulMF, matrix_free/src/LocalAssemblyMF.cpp:31-67,
// and ElementMF, matrix_free/src/ElementMF.cpp:106-296): per element e and
// quadrature point q,
//     y_e += sign * sum_q  grad_xi N^T  G_q  grad_xi u,
//     G_q  = w_q kappa_q det(J) J^-1 J^-T   (symmetric 2x2, 3 values),
// with N the tensor product of the element's 1-D B-spline (or 1-D rational)
// bases. The element operator is applied by sum factorisation: two 1-D
// contractions in, a 2x2 multiply per quadrature point, two 1-D contractions out.
//
// Work decomposition: a WARP owns a strip of 32 element columns (lane = column)
// and marches over TY element rows. Per row step every lane
//   1. contracts the new control-point row along x (rolling buffer xs),
//   2. contracts along y with the row's tables (warp-uniform, broadcast loads),
//   3. applies G (streamed into shared memory by the bulk-copy engine),
//   4. accumulates the y-transposed contraction into rolling row buffers acc,
//   5. finalises the control-point row that no later element touches, and
//      sums the p+1 neighbouring lanes' contributions with rotate-shuffles.
// Values a strip can complete on its own are stored to y; values other strips
// also touch (p-wide seams) go to a per-strip frame and are summed in a fixed
// order by seam_fixup_kernel. No atomics anywhere: results are bitwise
// reproducible run to run.
#pragma once
#include "iga_device.cuh"

namespace iga {

template <typename T>
struct ApplyParams {
    const T *x;
    T *y;
    const T *G;      // precomputed: [NSX][NSY][TY][NQ*NQ*3][32]
    const T *tabX;   // [NSX][2][NQ][NB][32]  (kind 0: value, 1: d/dxi)
    const T *tabY;   // [ney][2][NQ][NB]
    const double *CP;  // on the fly: (x,y) per control point
    const T *wq;     // on the fly: quadrature weight products w_qx w_qy, [NQ*NQ]
    const T *kappa;  // on the fly: per quadrature point or null
    T *frame;        // [NSX*NSY][FS]
    StripGrid g;
    T sign;
    int bc;
    int *err;
};

template <int P, typename T>
struct ApplyShape {
    static constexpr int NB = P + 1;
    static constexpr int NQ = P + 1;
    static constexpr int NQ2 = NQ * NQ;
    static constexpr int GELEMS = NQ2 * 3 * 32;        // one row step of G for a warp
    static constexpr int GBYTES = GELEMS * (int)sizeof(T);
    static constexpr int TABX = 2 * NQ * NB * 32;      // x tables of a CTA column strip
    static constexpr int XR = 8;                       // x rows in flight per warp
    static constexpr int XW = 40;                      // >= 32 + P, padded
    static_assert(GBYTES % 16 == 0, "bulk copy size must be a multiple of 16 bytes");
};

template <int P, typename T, int NST>
__host__ __device__ constexpr size_t apply_smem_bytes(int W)
{
    using S = ApplyShape<P, T>;
    return 128 /* barriers, padded */ + (size_t)W * NST * 8 + S::TABX * sizeof(T) + 128 +
           (size_t)W * NST * S::GBYTES + (size_t)W * S::XR * S::XW * sizeof(T);
}

template <typename T>
__device__ __forceinline__ T shfl_idx(T v, int src)
{
    return __shfl_sync(0xffffffffu, v, src);
}

// GEOM = 0: G streamed from the precomputed array (the mult_sf path).
// GEOM = 1: G computed in the warp from the control points (the mult_mf path).
template <int P, typename T, int GEOM, int NST>
__global__ void __launch_bounds__(256, 1) apply_kernel(ApplyParams<T> a)
{
    using S = ApplyShape<P, T>;
    constexpr int NB = S::NB, NQ = S::NQ;
    const StripGrid &g = a.g;
    const int lane = threadIdx.x, w = threadIdx.y, W = blockDim.y;
    const int gx = blockIdx.x, gy = blockIdx.y * W + w;

    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    size_t off = 128 + (size_t)W * NST * 8;
    off = (off + 127) & ~size_t(127);
    T *tabXs = reinterpret_cast<T *>(smem + off);
    off += S::TABX * sizeof(T);
    off = (off + 127) & ~size_t(127);
    T *Gs = reinterpret_cast<T *>(smem + off) + (size_t)w * NST * S::GELEMS;
    off += (size_t)W * NST * S::GBYTES;
    T *xr = reinterpret_cast<T *>(smem + off) + (size_t)w * S::XR * S::XW;
    uint64_t *wbar = bars + w * NST;

    // x tables of this column strip: [kind][qx][il][lane], shared by the CTA's warps.
    {
        const T *src = a.tabX + (size_t)gx * S::TABX;
        for (int i = threadIdx.y * 32 + lane; i < S::TABX; i += 32 * W) tabXs[i] = src[i];
    }
    __syncthreads();
    if (gy >= g.NSY) return;
    const int ex0 = 32 * gx, ey0 = g.TY * gy;
    const int nsteps = min(g.TY, g.ney - ey0);
    if (nsteps <= 0) return;
    const int ex = ex0 + lane;
    const T *Gstrip = a.G + (size_t)(gx * g.NSY + gy) * g.TY * S::GELEMS;

    if (GEOM == 0) {
        if (lane == 0) {
            for (int i = 0; i < NST; ++i) mbar_init(&wbar[i], 1);
            fence_mbar_init();
        }
        __syncwarp();
        if (lane == 0) {
            for (int s = 0; s < NST && s < nsteps; ++s) {
                mbar_arrive_expect_tx(&wbar[s], S::GBYTES);
                bulk_g2s(Gs + (size_t)s * S::GELEMS, Gstrip + (size_t)s * S::GELEMS, S::GBYTES, &wbar[s]);
            }
        }
    }

    // Control-point rows of x consumed in order k = 0, 1, ... (row ey0 + k).
    const int nrows = nsteps + P;
    auto fetch_row = [&](int k) {
        if (k < nrows) {
            const int R = ey0 + k;
            T *dst = xr + (k % S::XR) * S::XW;
            const bool rv = R < g.n;
            const size_t base = (size_t)(rv ? R : 0) * g.m;
            {
                const int C = ex0 + lane;
                const bool v = rv && C < g.m;
                cp_async_zfill<sizeof(T)>(dst + lane, a.x + base + (v ? C : 0), v);
            }
            if (lane < P) {
                const int C = ex0 + 32 + lane;
                const bool v = rv && C < g.m;
                cp_async_zfill<sizeof(T)>(dst + 32 + lane, a.x + base + (v ? C : 0), v);
            }
        }
        cp_async_commit();
    };
    constexpr int D = S::XR - 1;
    for (int k = 0; k < D; ++k) fetch_row(k);

    // Lane's x-direction column tables live in tabXs[kind][qx][il][lane].
    auto tx = [&](int kind, int qx, int il) -> T { return tabXs[((kind * NQ + qx) * NB + il) * 32 + lane]; };
    // Boundary masking of x (IGA_BC_IDENTITY: x[Dir] is not read).
    unsigned colmask = 0;   // bit il set: column ex+il is a boundary column
    if (a.bc == 1)
        for (int il = 0; il <= P; ++il) {
            const int C = ex + il;
            if (C == 0 || C == g.m - 1) colmask |= 1u << il;
        }

    T xs0[NB][NQ], xs1[NB][NQ];   // x contracted along x with value / derivative tables, rows ey..ey+P
    T acc0[NB][NQ], acc1[NB][NQ]; // y-transposed partial sums for control-point rows ey..ey+P

    auto contract_row = [&](int k, T (&r0)[NQ], T (&r1)[NQ]) {
        cp_async_wait<D - 1>();
        __syncwarp();
        const T *src = xr + (k % S::XR) * S::XW;
        const int R = ey0 + k;
        const bool rowb = (a.bc == 1) && (R == 0 || R == g.n - 1);
        T xv[NB];
#pragma unroll
        for (int il = 0; il < NB; ++il) xv[il] = (rowb || (colmask >> il) & 1u) ? T(0) : src[lane + il];
        __syncwarp();
        fetch_row(k + D);
#pragma unroll
        for (int qx = 0; qx < NQ; ++qx) {
            T s0 = 0, s1 = 0;
#pragma unroll
            for (int il = 0; il < NB; ++il) {
                s0 = fma(tx(0, qx, il), xv[il], s0);
                s1 = fma(tx(1, qx, il), xv[il], s1);
            }
            r0[qx] = s0;
            r1[qx] = s1;
        }
    };

    auto store = [&](int R, int C, T v) {
        const size_t i = (size_t)R * g.m + C;
        const bool bnd = (R == 0 || C == 0 || R == g.n - 1 || C == g.m - 1);
        a.y[i] = bnd ? (a.bc == 1 ? a.x[i] : T(0)) : a.sign * v;
    };
    T *frame = a.frame + (size_t)(gx * g.NSY + gy) * g.FS;
    auto write_row = [&](int lr, const T (&r0)[NQ], const T (&r1)[NQ]) {
        T out[NB];
#pragma unroll
        for (int il = 0; il < NB; ++il) {
            T s = 0;
#pragma unroll
            for (int qx = 0; qx < NQ; ++qx) {
                s = fma(tx(1, qx, il), r0[qx], s);
                s = fma(tx(0, qx, il), r1[qx], s);
            }
            out[il] = s;
        }
        // Column ex0+lane collects out[il] from lane-il; lanes < il receive the
        // wrapped value, which belongs to column ex0+32+lane (spill).
        T tot = out[0], spill = 0;
#pragma unroll
        for (int il = 1; il < NB; ++il) {
            const T v = shfl_idx(out[il], (lane - il) & 31);
            if (lane >= il) tot += v;
            else spill += v;
        }
        const int R = ey0 + lr;
        if (R >= g.n) return;
        int fb;
        const int rc = cover(R, g.TY, g.NSY, P, fb);
        {
            const int C = ex0 + lane;
            if (C < g.m) {
                int fa;
                const int cc = cover(C, 32, g.NSX, P, fa);
                if (rc == 1 && cc == 1) store(R, C, tot);
                else frame[frame_index(lr, lane, P, g.TY)] = tot;
            }
        }
        if (lane < P) {
            const int C = ex0 + 32 + lane;
            if (C < g.m) {
                int fa;
                const int cc = cover(C, 32, g.NSX, P, fa);
                if (rc == 1 && cc == 1) store(R, C, spill);
                else frame[frame_index(lr, 32 + lane, P, g.TY)] = spill;
            }
        }
    };

    // Prologue: rows ey0 .. ey0+P-1.
#pragma unroll
    for (int r = 0; r < P; ++r) contract_row(r, xs0[r], xs1[r]);
#pragma unroll
    for (int r = 0; r < NB; ++r)
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc0[r][q] = acc1[r][q] = 0;

    bool ok = true;
    int failed_step = 0;
    for (int s = 0; s < nsteps; ++s) {
        const int ey = ey0 + s;
        contract_row(s + P, xs0[P], xs1[P]);
        const int slot = s % NST;
        T *Gst = Gs + (size_t)slot * S::GELEMS;
        if (GEOM == 0) {
            if (!mbar_wait_bounded(&wbar[slot], (uint32_t)((s / NST) & 1))) {
                ok = false;
                failed_step = s;
                break;
            }
        } else {
            // Geometry from the control points of this lane's element.
            const bool act = ex < g.nex;
            for (int qy = 0; qy < NQ; ++qy) {
                for (int qx = 0; qx < NQ; ++qx) {
                    T g00 = 0, g01 = 0, g11 = 0;
                    if (act) {
                        double x_xi = 0, x_eta = 0, y_xi = 0, y_eta = 0;
                        for (int jl = 0; jl < NB; ++jl) {
                            const double n2 = (double)a.tabY[((size_t)(ey * 2 + 0) * NQ + qy) * NB + jl];
                            const double d2 = (double)a.tabY[((size_t)(ey * 2 + 1) * NQ + qy) * NB + jl];
                            const double *cp = a.CP + 2 * ((size_t)(ey + jl) * g.m + ex);
                            for (int il = 0; il < NB; ++il) {
                                const double n1 = (double)tx(0, qx, il), d1 = (double)tx(1, qx, il);
                                const double cx = cp[2 * il], cy = cp[2 * il + 1];
                                x_xi += cx * d1 * n2;
                                x_eta += cx * n1 * d2;
                                y_xi += cy * d1 * n2;
                                y_eta += cy * n1 * d2;
                            }
                        }
                        const double det = x_xi * y_eta - x_eta * y_xi;
                        double wgt = (double)a.wq[qy * NQ + qx];
                        if (a.kappa) wgt *= (double)a.kappa[((size_t)ey * g.nex + ex) * S::NQ2 + qy * NQ + qx];
                        const double f = wgt / det;
                        g00 = (T)(f * (x_eta * x_eta + y_eta * y_eta));
                        g01 = (T)(-f * (x_xi * x_eta + y_xi * y_eta));
                        g11 = (T)(f * (x_xi * x_xi + y_xi * y_xi));
                    }
                    const int qp = qy * NQ + qx;
                    Gst[(qp * 3 + 0) * 32 + lane] = g00;
                    Gst[(qp * 3 + 1) * 32 + lane] = g01;
                    Gst[(qp * 3 + 2) * 32 + lane] = g11;
                }
            }
            __syncwarp();
        }
        const T *ty = a.tabY + (size_t)ey * 2 * NQ * NB;
#pragma unroll
        for (int qy = 0; qy < NQ; ++qy) {
            T n2[NB], d2[NB];
#pragma unroll
            for (int jl = 0; jl < NB; ++jl) {
                n2[jl] = __ldg(ty + qy * NB + jl);
                d2[jl] = __ldg(ty + (NQ + qy) * NB + jl);
            }
#pragma unroll
            for (int qx = 0; qx < NQ; ++qx) {
                T uxi = 0, ueta = 0;
#pragma unroll
                for (int jl = 0; jl < NB; ++jl) {
                    uxi = fma(n2[jl], xs1[jl][qx], uxi);
                    ueta = fma(d2[jl], xs0[jl][qx], ueta);
                }
                const int qp = qy * NQ + qx;
                const T g00 = Gst[(qp * 3 + 0) * 32 + lane];
                const T g01 = Gst[(qp * 3 + 1) * 32 + lane];
                const T g11 = Gst[(qp * 3 + 2) * 32 + lane];
                const T vxi = fma(g00, uxi, g01 * ueta);
                const T veta = fma(g01, uxi, g11 * ueta);
#pragma unroll
                for (int jl = 0; jl < NB; ++jl) {
                    acc0[jl][qx] = fma(n2[jl], vxi, acc0[jl][qx]);
                    acc1[jl][qx] = fma(d2[jl], veta, acc1[jl][qx]);
                }
            }
        }
        __syncwarp();
        if (GEOM == 0 && lane == 0 && s + NST < nsteps) {
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&wbar[slot], S::GBYTES);
            bulk_g2s(Gst, Gstrip + (size_t)(s + NST) * S::GELEMS, S::GBYTES, &wbar[slot]);
        }
        write_row(s, acc0[0], acc1[0]);
#pragma unroll
        for (int r = 0; r < P; ++r)
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                xs0[r][q] = xs0[r + 1][q];
                xs1[r][q] = xs1[r + 1][q];
                acc0[r][q] = acc0[r + 1][q];
                acc1[r][q] = acc1[r + 1][q];
            }
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc0[P][q] = acc1[P][q] = 0;
    }
    if (!ok) {
        if (lane == 0) atomicExch(a.err, 8 /* IGA_ERR_TIMEOUT */);
        // Let the copies already issued (steps failed_step .. failed_step+NST-1)
        // land before the CTA's shared memory is released; bounded as well.
        if (GEOM == 0)
            for (int t = failed_step; t < nsteps && t < failed_step + NST; ++t)
                mbar_wait_bounded(&wbar[t % NST], (uint32_t)((t / NST) & 1));
        cp_async_wait<0>();
        return;
    }
    // Rows above the last element row: partial sums for rows ey_last+1 .. ey_last+P.
#pragma unroll
    for (int r = 0; r < P; ++r) {
        write_row(nsteps + r, acc0[0], acc1[0]);
#pragma unroll
        for (int rr = 0; rr < P; ++rr)
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                acc0[rr][q] = acc0[rr + 1][q];
                acc1[rr][q] = acc1[rr + 1][q];
            }
    }
    cp_async_wait<0>();
}

// Sums the frames of the strips covering each seam control point, strip
// (row, then column) in ascending order, and stores sign * sum (boundary
// rules as in apply_kernel).
template <int P, typename T>
__global__ void seam_fixup_kernel(const T *__restrict__ frame, const T *__restrict__ x, T *__restrict__ y,
                                  StripGrid g, T sign, int bc)
{
    const long long nvc = (long long)(g.NSX - 1) * P;   // vertical seam columns
    const long long nV = nvc * g.n;
    const long long nH = (long long)(g.NSY - 1) * P * g.m;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < nV + nH;
         idx += (long long)gridDim.x * blockDim.x) {
        int R, C;
        if (idx < nV) {
            const int cid = (int)(idx % nvc);
            R = (int)(idx / nvc);
            C = 32 * (1 + cid / P) + cid % P;
            if (C >= g.m) continue;
        } else {
            const long long j = idx - nV;
            C = (int)(j % g.m);
            const int rid = (int)(j / g.m);
            R = g.TY * (1 + rid / P) + rid % P;
            if (R >= g.n) continue;
            const int s = C / 32;
            if (C % 32 < P && s >= 1 && s < g.NSX) continue;   // handled as a vertical seam
        }
        int fa, fb;
        const int ca = cover(C, 32, g.NSX, P, fa);
        const int cb = cover(R, g.TY, g.NSY, P, fb);
        T v = 0;
        for (int bi = 0; bi < cb; ++bi) {
            const int b = fb + bi;
            for (int ai = 0; ai < ca; ++ai) {
                const int aa = fa + ai;
                v += frame[(size_t)(aa * g.NSY + b) * g.FS + frame_index(R - g.TY * b, C - 32 * aa, P, g.TY)];
            }
        }
        const size_t i = (size_t)R * g.m + C;
        const bool bnd = (R == 0 || C == 0 || R == g.n - 1 || C == g.m - 1);
        y[i] = bnd ? (bc == 1 ? x[i] : T(0)) : sign * v;
    }
}

}  // namespace iga
