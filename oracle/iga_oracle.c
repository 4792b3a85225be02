/* CPU oracle: plain-C restatement of the reference's matrix-free IGA Poisson
 * operator, load vector, FEM preconditioner and Krylov solve.
 *
 * TEST INFRASTRUCTURE ONLY (see iga_oracle.h): the checker for the CUDA path,
 * never part of it. Every function cites the reference lines it restates,
 * relative to the reference project root. */
#include "iga_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAXP 8
#define ORC_MAXN ((ORC_MAXP + 1) * (ORC_MAXP + 1))

/* ------------------------------------------------------------------ RNG */
static uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static double u53(uint64_t seed, long i)
{
    return (double)(mix64(seed + (uint64_t)(i + 1) * 0x9e3779b97f4a7c15ULL) >> 11) * 0x1.0p-53;
}

void orc_uniform(uint64_t seed, double lo, double hi, double *out, long n)
{
    for (long i = 0; i < n; ++i) out[i] = lo + (hi - lo) * u53(seed, i);
}

void orc_normal(uint64_t seed, double *out, long n)
{
    const double two_pi = 6.283185307179586476925286766559;
    for (long i = 0; i < n; i += 2) {
        const double a = u53(seed, i), b = u53(seed, i + 1);
        const double r = sqrt(-2.0 * log(1.0 - a));
        out[i] = r * cos(two_pi * b);
        if (i + 1 < n) out[i + 1] = r * sin(two_pi * b);
    }
}

/* ------------------------------------------------------------- 1-D pieces */
/* Gauss-Legendre rule on [0,1]; the reference tabulates the same rule to 16
 * digits (matrix_free/src/QuadraturePoint.cpp:3-58). Newton on P_n. */
void orc_gauss01(int n, double *x, double *w)
{
    const double pi = 3.141592653589793238462643383279;
    for (int i = 0; i < n; ++i) {
        double t = cos(pi * (i + 0.75) / (n + 0.5)), dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = t;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * t * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) { p1 = t; p0 = 1.0; }
            dp = n * (t * p1 - p0) / (t * t - 1.0);
            const double dt = p1 / dp;
            t -= dt;
            if (fabs(dt) < 1e-17) break;
        }
        {   /* final derivative at the converged root for the weight */
            double p0 = 1.0, p1 = t;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * t * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) { p1 = t; p0 = 1.0; }
            dp = n * (t * p1 - p0) / (t * t - 1.0);
        }
        /* roots come out descending; store ascending on [0,1] */
        x[n - 1 - i] = 0.5 * (t + 1.0);
        w[n - 1 - i] = 1.0 / ((1.0 - t * t) * dp * dp);
    }
}

/* Bernstein polynomials of degree p on [0,1] and d/dxi
 * (matrix_free/src/BernsteinBasis.cpp:3-146 tabulates the same closed forms). */
void orc_bernstein(int p, double xi, double *B, double *dB)
{
    double lo[ORC_MAXP + 1];
    /* degree p-1 values for the derivative identity dB_k = p (B_{k-1} - B_k) */
    for (int k = 0; k <= p; ++k) B[k] = 0.0;
    B[0] = 1.0;
    for (int d = 1; d <= p; ++d) {
        if (d == p)
            for (int k = 0; k < p; ++k) lo[k] = B[k];
        for (int k = d; k >= 0; --k) B[k] = (k ? xi * B[k - 1] : 0.0) + (k < d ? (1.0 - xi) * B[k] : 0.0);
    }
    if (p == 0) { dB[0] = 0.0; return; }
    for (int k = 0; k <= p; ++k)
        dB[k] = p * ((k ? lo[k - 1] : 0.0) - (k < p ? lo[k] : 0.0));
}

/* Open uniform knot vector of matrix_free/preprocess.cpp:50-56. */
int orc_open_knots(int p, int ne, double L, double *S)
{
    int n = 0;
    const double h = L / ne;
    for (int i = 0; i < p + 1; ++i) S[n++] = 0.0;
    for (int i = 1; i < ne; ++i) S[n++] = i * h;
    for (int i = 0; i < p + 1; ++i) S[n++] = L;
    return n;
}

/* Bezier extraction, Borden et al. 2011 (IJNME 87:15-47) Algorithm 1, as used
 * by matrix_free/src/NURBSExtractionGenerator.cpp:4-82. Written with 1-based
 * knot indices U(i) = S[i-1] as in the paper. C holds one row-major
 * (p+1)x(p+1) block per element. Returns the number of elements. */
int orc_extraction(int p, const double *S, int nS, double *C)
{
#define U(i) S[(i) - 1]
#define CE(e, r, c) C[((e) - 1) * a * a + ((r) - 1) * a + ((c) - 1)]
    const int m = nS, a = p + 1;
    const int maxe = nS - 2 * p - 1;
    double alphas[ORC_MAXP + 2];
    memset(C, 0, sizeof(double) * (size_t)maxe * a * a);
    for (int i = 1; i <= a; ++i) CE(1, i, i) = 1.0;
    int nb = 1, A = p + 1, b = A + 1;
    while (b < m) {
        if (nb + 1 <= maxe)
            for (int i = 1; i <= a; ++i) CE(nb + 1, i, i) = 1.0;
        const int i0 = b;
        while (b < m && U(b + 1) == U(b)) ++b;
        const int mult = b - i0 + 1;
        if (mult < p) {
            const double numer = U(b) - U(A);
            for (int j = p; j > mult; --j) alphas[j - mult] = numer / (U(A + j) - U(A));
            const int r = p - mult;
            for (int j = 1; j <= r; ++j) {
                const int save = r - j + 1, s = mult + j;
                for (int k = p + 1; k > s; --k) {
                    const double al = alphas[k - s];
                    for (int row = 1; row <= a; ++row)
                        CE(nb, row, k) = al * CE(nb, row, k) + (1.0 - al) * CE(nb, row, k - 1);
                }
                if (b < m && nb + 1 <= maxe)
                    for (int o = 0; o <= j; ++o) CE(nb + 1, save + o, save) = CE(nb, p - j + 1 + o, p + 1);
            }
        }
        if (b < m) {
            ++nb;
            A = b;
            ++b;
        }
    }
    return nb;
#undef U
#undef CE
}

/* Greville abscissae (matrix_free/src/AbscissaeGenerator.cpp:27-41). */
void orc_greville(int p, const double *S, int nS, double *g)
{
    const int n = nS - p - 1;
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int j = 1; j <= p; ++j) s += S[i + j];
        g[i] = s / p;
    }
}

/* ------------------------------------------------------- element kernel */
typedef struct {
    int p, q, nq1, nq2;
    double qp1[ORC_MAXP + 1], qw1[ORC_MAXP + 1], qp2[ORC_MAXP + 1], qw2[ORC_MAXP + 1];
    double B1[(ORC_MAXP + 1) * (ORC_MAXP + 1)], dB1[(ORC_MAXP + 1) * (ORC_MAXP + 1)];
    double B2[(ORC_MAXP + 1) * (ORC_MAXP + 1)], dB2[(ORC_MAXP + 1) * (ORC_MAXP + 1)];
} tables;

/* (p+1) Gauss points per direction on [0,1] and Bernstein tables at them
 * (matrix_free/include/LocalAssemblyMF.hpp:17-22). */
static void make_tables(int p, int q, tables *t)
{
    t->p = p;
    t->q = q;
    t->nq1 = p + 1;
    t->nq2 = q + 1;
    orc_gauss01(p + 1, t->qp1, t->qw1);
    orc_gauss01(q + 1, t->qp2, t->qw2);
    for (int i = 0; i < p + 1; ++i) orc_bernstein(p, t->qp1[i], t->B1 + i * (p + 1), t->dB1 + i * (p + 1));
    for (int j = 0; j < q + 1; ++j) orc_bernstein(q, t->qp2[j], t->B2 + j * (q + 1), t->dB2 + j * (q + 1));
}

/* Basis, gradients and JxW at one quadrature point of element (ex, ey):
 * matrix_free/src/ElementMF.cpp:106-207 (N = C B, dN = C dB / h, rational
 * R = N/w, geometry from the element control points, inverse Jacobian,
 * jacobian *= hx*hy), with optional control-point weights W. */
static void element_qp(const orc_patch *P, const tables *t, int ex, int ey, int ii, int jj,
                       double *R, double *dRdx, double *dRdy, double *jxw, double *xq, double *yq)
{
    const int p = P->p, q = P->q, m = P->nex + p;
    const double *e1 = P->C1 + (size_t)ex * (p + 1) * (p + 1);
    const double *e2 = P->C2 + (size_t)ey * (q + 1) * (q + 1);
    const double hx = P->h1[ex], hy = P->h2[ey];
    double N1[ORC_MAXP + 1], dN1[ORC_MAXP + 1], N2[ORC_MAXP + 1], dN2[ORC_MAXP + 1];
    for (int i = 0; i <= p; ++i) {   /* RefElement.cpp:20-57 */
        double s = 0.0, d = 0.0;
        for (int k = 0; k <= p; ++k) {
            s += e1[i * (p + 1) + k] * t->B1[ii * (p + 1) + k];
            d += e1[i * (p + 1) + k] * t->dB1[ii * (p + 1) + k];
        }
        N1[i] = s;
        dN1[i] = d / hx;
    }
    for (int j = 0; j <= q; ++j) {
        double s = 0.0, d = 0.0;
        for (int k = 0; k <= q; ++k) {
            s += e2[j * (q + 1) + k] * t->B2[jj * (q + 1) + k];
            d += e2[j * (q + 1) + k] * t->dB2[jj * (q + 1) + k];
        }
        N2[j] = s;
        dN2[j] = d / hy;
    }
    const int n = (p + 1) * (q + 1);
    double N[ORC_MAXN], Nx[ORC_MAXN], Ny[ORC_MAXN];
    double w = 0.0, wx = 0.0, wy = 0.0;
    for (int j = 0; j <= q; ++j)
        for (int i = 0; i <= p; ++i) {
            const int a = j * (p + 1) + i;
            const double wa = P->W ? P->W[(ey + j) * m + (ex + i)] : 1.0;
            N[a] = wa * N1[i] * N2[j];
            Nx[a] = wa * dN1[i] * N2[j];
            Ny[a] = wa * N1[i] * dN2[j];
            w += N[a];
            wx += Nx[a];
            wy += Ny[a];
        }
    double dRxi[ORC_MAXN], dReta[ORC_MAXN];
    for (int a = 0; a < n; ++a) {
        R[a] = N[a] / w;
        dRxi[a] = (Nx[a] - wx * R[a]) / w;
        dReta[a] = (Ny[a] - wy * R[a]) / w;
    }
    double x = 0, y = 0, x_xi = 0, x_eta = 0, y_xi = 0, y_eta = 0;
    for (int j = 0; j <= q; ++j)
        for (int i = 0; i <= p; ++i) {
            const int a = j * (p + 1) + i;
            const size_t A = (size_t)(ey + j) * m + (ex + i);
            const double cx = P->CP[2 * A], cy = P->CP[2 * A + 1];
            x += cx * R[a];
            y += cy * R[a];
            x_xi += cx * dRxi[a];
            x_eta += cx * dReta[a];
            y_xi += cy * dRxi[a];
            y_eta += cy * dReta[a];
        }
    double jac = x_xi * y_eta - x_eta * y_xi;
    const double xi_x = y_eta / jac, xi_y = -x_eta / jac, eta_x = -y_xi / jac, eta_y = x_xi / jac;
    for (int a = 0; a < n; ++a) {
        dRdx[a] = xi_x * dRxi[a] + eta_x * dReta[a];
        dRdy[a] = xi_y * dRxi[a] + eta_y * dReta[a];
    }
    jac *= hx * hy;
    *jxw = t->qw1[ii] * t->qw2[jj] * jac;   /* ElementMF.cpp:284 */
    if (xq) *xq = x;
    if (yq) *yq = y;
}

static int on_boundary(int i, int j, int m, int n) { return i == 0 || j == 0 || i == m - 1 || j == n - 1; }

/* GlobalAssemblyMF::MatMulMF (matrix_free/src/GlobalAssemblyMF.cpp:141-210)
 * around LocalAssemblyMF::LocalMatMulMF (matrix_free/src/LocalAssemblyMF.cpp:31-67). */
void orc_apply_mf(const orc_patch *P, const double *x, double *y, double sign, int bc)
{
    const int p = P->p, q = P->q, m = P->nex + p, nn = P->ney + q;
    const int n = (p + 1) * (q + 1);
    tables t;
    make_tables(p, q, &t);
    memset(y, 0, sizeof(double) * (size_t)m * nn);
    double R[ORC_MAXN], Rx[ORC_MAXN], Ry[ORC_MAXN], xe[ORC_MAXN], ye[ORC_MAXN];
    for (int ey = 0; ey < P->ney; ++ey)
        for (int ex = 0; ex < P->nex; ++ex) {
            for (int j = 0; j <= q; ++j)
                for (int i = 0; i <= p; ++i) {
                    const int I = ex + i, J = ey + j;
                    xe[j * (p + 1) + i] = (bc == 1 && on_boundary(I, J, m, nn)) ? 0.0 : x[(size_t)J * m + I];
                }
            memset(ye, 0, sizeof(ye));
            for (int jj = 0; jj < t.nq2; ++jj)
                for (int ii = 0; ii < t.nq1; ++ii) {
                    double jxw;
                    element_qp(P, &t, ex, ey, ii, jj, R, Rx, Ry, &jxw, NULL, NULL);
                    if (P->kappa) jxw *= P->kappa[((size_t)ey * P->nex + ex) * t.nq1 * t.nq2 + jj * t.nq1 + ii];
                    double tx = 0.0, ty = 0.0;
                    for (int a = 0; a < n; ++a) {
                        tx += Rx[a] * xe[a];
                        ty += Ry[a] * xe[a];
                    }
                    tx *= sign * jxw;
                    ty *= sign * jxw;
                    for (int a = 0; a < n; ++a) ye[a] += Rx[a] * tx + Ry[a] * ty;
                }
            for (int j = 0; j <= q; ++j)
                for (int i = 0; i <= p; ++i) {
                    const int I = ex + i, J = ey + j;
                    if (bc == 2 || !on_boundary(I, J, m, nn)) y[(size_t)J * m + I] += ye[j * (p + 1) + i];
                }
        }
    for (int J = 0; J < nn; ++J)
        for (int I = 0; I < m; ++I)
            if (bc != 2 && on_boundary(I, J, m, nn)) y[(size_t)J * m + I] = (bc == 1) ? x[(size_t)J * m + I] : 0.0;
}

/* The reference mult_sf: ElementMFSF::GenerateElement (matrix_free/src/ElementMFSF.cpp:237-297:
 * 1-D tables evaluated at the x quadrature points for both directions, per-qp
 * W, J, dW/dx, dW/dy) and the dense Kloc of LocalAssemblyMFSF::LocalMatMulMF
 * (matrix_free/src/LocalAssemblyMFSF.cpp:43-103), then Kloc x_e. Holds for
 * p == q on axis-aligned affine patches, as in the reference. */
void orc_apply_sf(const orc_patch *P, const double *x, double *y, double sign)
{
    const int p = P->p, q = P->q, m = P->nex + p, nn = P->ney + q;
    const int n = (p + 1) * (q + 1), nq1 = p + 1, nq2 = q + 1;
    tables t;
    make_tables(p, q, &t);
    int map[2 * ORC_MAXN];
    {   /* LocalAssemblyMFSF.hpp:24-31 */
        int k = 0;
        for (int i = 0; i < p + 1; ++i)
            for (int j = 0; j < q + 1; ++j) {
                map[2 * k] = j;
                map[2 * k + 1] = i;
                ++k;
            }
    }
    memset(y, 0, sizeof(double) * (size_t)m * nn);
    static double K[ORC_MAXN * ORC_MAXN];
    for (int ey = 0; ey < P->ney; ++ey)
        for (int ex = 0; ex < P->nex; ++ex) {
            const double *e1 = P->C1 + (size_t)ex * (p + 1) * (p + 1);
            const double *e2 = P->C2 + (size_t)ey * (q + 1) * (q + 1);
            const double hx = P->h1[ex], hy = P->h2[ey];
            /* 1-D tables; N2 evaluated at the x points (ElementMFSF.cpp:28-31) */
            double B1[ORC_MAXN], dB1[ORC_MAXN], B2[ORC_MAXN], dB2[ORC_MAXN];
            for (int ii = 0; ii < nq1; ++ii) {
                double Bb[ORC_MAXP + 1], dBb[ORC_MAXP + 1], Bq[ORC_MAXP + 1], dBq[ORC_MAXP + 1];
                orc_bernstein(p, t.qp1[ii], Bb, dBb);
                orc_bernstein(q, t.qp1[ii], Bq, dBq);
                for (int i = 0; i <= p; ++i) {
                    double s = 0, d = 0;
                    for (int k = 0; k <= p; ++k) { s += e1[i * (p + 1) + k] * Bb[k]; d += e1[i * (p + 1) + k] * dBb[k]; }
                    B1[ii * (p + 1) + i] = s;
                    dB1[ii * (p + 1) + i] = d / hx;
                }
                for (int j = 0; j <= q; ++j) {
                    double s = 0, d = 0;
                    for (int k = 0; k <= q; ++k) { s += e2[j * (q + 1) + k] * Bq[k]; d += e2[j * (q + 1) + k] * dBq[k]; }
                    B2[ii * (q + 1) + j] = s;
                    dB2[ii * (q + 1) + j] = d / hy;
                }
            }
            /* per-qp W, J, dW/dx, dW/dy (ElementMFSF.cpp:101-179), index ii*nq2+jj */
            double Wq[ORC_MAXN], Jq[ORC_MAXN], Wx[ORC_MAXN], Wy[ORC_MAXN];
            for (int jj = 0; jj < nq2; ++jj)
                for (int ii = 0; ii < nq1; ++ii) {
                    double w = 0, wxi = 0, weta = 0, x_xi = 0, x_eta = 0, y_xi = 0, y_eta = 0;
                    double Nn[ORC_MAXN], Nxi[ORC_MAXN], Neta[ORC_MAXN];
                    for (int j = 0; j <= q; ++j)
                        for (int i = 0; i <= p; ++i) {
                            const int a = j * (p + 1) + i;
                            Nn[a] = B1[ii * (p + 1) + i] * B2[jj * (q + 1) + j];
                            Nxi[a] = dB1[ii * (p + 1) + i] * B2[jj * (q + 1) + j];
                            Neta[a] = B1[ii * (p + 1) + i] * dB2[jj * (q + 1) + j];
                            w += Nn[a];
                            wxi += Nxi[a];
                            weta += Neta[a];
                        }
                    for (int j = 0; j <= q; ++j)
                        for (int i = 0; i <= p; ++i) {
                            const int a = j * (p + 1) + i;
                            const double Ra = Nn[a] / w;
                            const double Rxi = (Nxi[a] - wxi * Ra) / w, Reta = (Neta[a] - weta * Ra) / w;
                            const size_t A = (size_t)(ey + j) * m + (ex + i);
                            x_xi += P->CP[2 * A] * Rxi;
                            x_eta += P->CP[2 * A] * Reta;
                            y_xi += P->CP[2 * A + 1] * Rxi;
                            y_eta += P->CP[2 * A + 1] * Reta;
                        }
                    const double jac = x_xi * y_eta - x_eta * y_xi;
                    const double xi_x = y_eta / jac, xi_y = -x_eta / jac, eta_x = -y_xi / jac, eta_y = x_xi / jac;
                    const int k = jj * nq1 + ii;   /* push order of ElementMFSF::GenerateElement */
                    Wq[k] = w;
                    Jq[k] = jac * hx * hy;
                    Wx[k] = wxi * xi_x + weta * eta_x;
                    Wy[k] = wxi * xi_y + weta * eta_y;
                }
            memset(K, 0, sizeof(double) * n * n);
            for (int i = 0; i < n; ++i) {
                const int i1 = map[2 * i], i2 = map[2 * i + 1];
                for (int j = 0; j < n; ++j) {
                    const int j1 = map[2 * j], j2 = map[2 * j + 1];
                    for (int ii = 0; ii < nq1; ++ii) {
                        double t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0, t7 = 0;
                        for (int jj = 0; jj < nq2; ++jj) {
                            const int k = ii * nq2 + jj;
                            const double W = Wq[k], J = Jq[k];
                            const double b2i = B2[nq2 * jj + i2], b2j = B2[nq2 * jj + j2];
                            const double d2i = dB2[nq2 * jj + i2], d2j = dB2[nq2 * jj + j2];
                            t1 += t.qw2[jj] * b2i * b2j * J / (W * W);
                            t2 += t.qw2[jj] * d2i * d2j * J / (W * W);
                            t3 += t.qw2[jj] * b2i * b2j * J / (W * W * W) * Wx[k];
                            t4 += t.qw2[jj] * b2i * b2j * J / (W * W * W) * Wx[k];
                            t5 += t.qw2[jj] * b2i * d2j * J / (W * W * W) * Wy[k];
                            t6 += t.qw2[jj] * d2i * b2j * J / (W * W * W) * Wy[k];
                            t7 += t.qw2[jj] * b2i * b2j * (Wx[k] * Wx[k] + Wy[k] * Wy[k]) * J / (W * W);
                        }
                        const double b1i = B1[nq1 * ii + i1], b1j = B1[nq1 * ii + j1];
                        const double d1i = dB1[nq1 * ii + i1], d1j = dB1[nq1 * ii + j1];
                        K[i * n + j] += sign * t.qw1[ii] *
                                        (d1i * d1j * t1 + b1i * b1j * t2 - b1i * d1j * t3 - d1i * b1j * t4 -
                                         b1i * b1j * t5 - b1i * b1j * t6 - b1i * b1j * t7);
                    }
                }
            }
            for (int a = 0; a < n; ++a) {
                const int I = ex + a % (p + 1), J = ey + a / (p + 1);
                if (on_boundary(I, J, m, nn)) continue;
                double s = 0.0;
                for (int b = 0; b < n; ++b) {
                    const int I2 = ex + b % (p + 1), J2 = ey + b / (p + 1);
                    s += K[a * n + b] * x[(size_t)J2 * m + I2];
                }
                y[(size_t)J * m + I] += s;
            }
        }
    for (int J = 0; J < nn; ++J)
        for (int I = 0; I < m; ++I)
            if (on_boundary(I, J, m, nn)) y[(size_t)J * m + I] = 0.0;
}

static double rhs_f(int fkind, double x, double y)
{
    const double pi = 3.141592653589793238462643383279;
    switch (fkind) {
    case 0: return x * (1 - x) * y * (1 - y);   /* LocalAssemblyMF.hpp:52-55 */
    case 1: return 2.0 * pi * pi * sin(pi * x) * sin(pi * y);
    default: {
        const double r = sqrt(x * x + y * y), th = atan2(y, x);
        return (pi * pi * sin(pi * r) - pi * cos(pi * r) / r + 4.0 * sin(pi * r) / (r * r)) * sin(2.0 * th);
    }
    }
}

/* GlobalAssemblyMF::AssemLoad + LocalAssemblyMF::AssemLocalLoad
 * (matrix_free/src/GlobalAssemblyMF.cpp:26-80, matrix_free/src/LocalAssemblyMF.cpp:3-29). */
void orc_rhs(const orc_patch *P, int fkind, double *F)
{
    const int p = P->p, q = P->q, m = P->nex + p, nn = P->ney + q, n = (p + 1) * (q + 1);
    tables t;
    make_tables(p, q, &t);
    memset(F, 0, sizeof(double) * (size_t)m * nn);
    double R[ORC_MAXN], Rx[ORC_MAXN], Ry[ORC_MAXN];
    for (int ey = 0; ey < P->ney; ++ey)
        for (int ex = 0; ex < P->nex; ++ex) {
            double fe[ORC_MAXN] = {0};
            for (int jj = 0; jj < t.nq2; ++jj)
                for (int ii = 0; ii < t.nq1; ++ii) {
                    double jxw, xq, yq;
                    element_qp(P, &t, ex, ey, ii, jj, R, Rx, Ry, &jxw, &xq, &yq);
                    const double f = rhs_f(fkind, xq, yq);
                    for (int a = 0; a < n; ++a) fe[a] += R[a] * f * jxw;
                }
            for (int a = 0; a < n; ++a) {
                const int I = ex + a % (p + 1), J = ey + a / (p + 1);
                if (!on_boundary(I, J, m, nn)) F[(size_t)J * m + I] += fe[a];
            }
        }
}

void orc_qp_points(const orc_patch *P, double *xy, double *jw)
{
    const int p = P->p, q = P->q;
    tables t;
    make_tables(p, q, &t);
    double R[ORC_MAXN], Rx[ORC_MAXN], Ry[ORC_MAXN];
    for (int ey = 0; ey < P->ney; ++ey)
        for (int ex = 0; ex < P->nex; ++ex)
            for (int jj = 0; jj < t.nq2; ++jj)
                for (int ii = 0; ii < t.nq1; ++ii) {
                    const size_t k = ((size_t)ey * P->nex + ex) * t.nq1 * t.nq2 + jj * t.nq1 + ii;
                    double jxw, xq, yq;
                    element_qp(P, &t, ex, ey, ii, jj, R, Rx, Ry, &jxw, &xq, &yq);
                    xy[2 * k] = xq;
                    xy[2 * k + 1] = yq;
                    if (jw) jw[k] = jxw;
                }
}

void orc_eval_qp(const orc_patch *P, const double *u, double *vals)
{
    const int p = P->p, q = P->q, m = P->nex + p, n = (p + 1) * (q + 1);
    tables t;
    make_tables(p, q, &t);
    double R[ORC_MAXN], Rx[ORC_MAXN], Ry[ORC_MAXN];
    for (int ey = 0; ey < P->ney; ++ey)
        for (int ex = 0; ex < P->nex; ++ex)
            for (int jj = 0; jj < t.nq2; ++jj)
                for (int ii = 0; ii < t.nq1; ++ii) {
                    double jxw;
                    element_qp(P, &t, ex, ey, ii, jj, R, Rx, Ry, &jxw, NULL, NULL);
                    double s = 0.0;
                    for (int a = 0; a < n; ++a) s += R[a] * u[(size_t)(ey + a / (p + 1)) * m + (ex + a % (p + 1))];
                    vals[((size_t)ey * P->nex + ex) * t.nq1 * t.nq2 + jj * t.nq1 + ii] = s;
                }
}

void orc_adjoint_grad(const orc_patch *P, const double *u, const double *lam, double *g)
{
    const int p = P->p, q = P->q, m = P->nex + p, n = (p + 1) * (q + 1);
    tables t;
    make_tables(p, q, &t);
    double R[ORC_MAXN], Rx[ORC_MAXN], Ry[ORC_MAXN];
    for (int ey = 0; ey < P->ney; ++ey)
        for (int ex = 0; ex < P->nex; ++ex)
            for (int jj = 0; jj < t.nq2; ++jj)
                for (int ii = 0; ii < t.nq1; ++ii) {
                    double jxw;
                    element_qp(P, &t, ex, ey, ii, jj, R, Rx, Ry, &jxw, NULL, NULL);
                    double ux = 0, uy = 0, lx = 0, ly = 0;
                    for (int a = 0; a < n; ++a) {
                        const size_t A = (size_t)(ey + a / (p + 1)) * m + (ex + a % (p + 1));
                        ux += Rx[a] * u[A];
                        uy += Ry[a] * u[A];
                        lx += Rx[a] * lam[A];
                        ly += Ry[a] * lam[A];
                    }
                    g[((size_t)ey * P->nex + ex) * t.nq1 * t.nq2 + jj * t.nq1 + ii] = -(lx * ux + ly * uy) * jxw;
                }
}

/* --------------------------------------------------- FEM preconditioner */
void orc_fem_nodes(int p, int ne, double L, double *nodes)
{
    if (p >= 3) {   /* matrix_free/preprocess_fem.cpp:38-60 */
        double *S = (double *)malloc(sizeof(double) * (ne + 2 * p + 4));
        const double h = L / (ne + 2);
        int n = 0;
        for (int i = 0; i < p - 1; ++i) S[n++] = 0.0;
        for (int i = 1; i < ne + 2; ++i) S[n++] = i * h;
        for (int i = 0; i < p - 1; ++i) S[n++] = L;
        orc_greville(p - 2, S, n, nodes);
        free(S);
    } else {        /* p == 2: degree-p Greville abscissae of the IGA knots */
        double *S = (double *)malloc(sizeof(double) * (ne + 2 * p + 1));
        const int n = orc_open_knots(p, ne, L, S);
        orc_greville(p, S, n, nodes);
        free(S);
    }
}

/* Bilinear element stiffness with 2x2 Gauss (matrix_free/src/ElementFEM.cpp:3-117,
 * matrix_free/src/LocalAssembly.cpp:42-79), assembled on the node grid
 * (GlobalAssembly::AssemStiffnessLoad(ElementFEM), matrix_free/src/GlobalAssembly.cpp:162-217). */
void orc_fem_matvec(int nfx, int nfy, const double *gx, const double *gy, const double *x, double *y,
                    double sign)
{
    double qp[2], qw[2];
    orc_gauss01(2, qp, qw);
    memset(y, 0, sizeof(double) * (size_t)nfx * nfy);
    for (int ey = 0; ey < nfy - 1; ++ey)
        for (int ex = 0; ex < nfx - 1; ++ex) {
            const double hx = gx[ex + 1] - gx[ex], hy = gy[ey + 1] - gy[ey];
            double K[16] = {0};
            for (int jj = 0; jj < 2; ++jj)
                for (int ii = 0; ii < 2; ++ii) {
                    const double xi = qp[ii], eta = qp[jj];
                    const double N1[2] = {1 - xi, xi}, dN1[2] = {-1, 1}, N2[2] = {1 - eta, eta}, dN2[2] = {-1, 1};
                    const double jac = hx * hy, jxw = qw[ii] * qw[jj] * jac;
                    double Rx[4], Ry[4];
                    for (int j = 0; j < 2; ++j)
                        for (int i = 0; i < 2; ++i) {
                            Rx[j * 2 + i] = dN1[i] * N2[j] / hx;
                            Ry[j * 2 + i] = N1[i] * dN2[j] / hy;
                        }
                    for (int k = 0; k < 4; ++k)
                        for (int l = 0; l < 4; ++l) K[k * 4 + l] += sign * jxw * (Rx[k] * Rx[l] + Ry[k] * Ry[l]);
                }
            int A[4];
            for (int j = 0; j < 2; ++j)
                for (int i = 0; i < 2; ++i) A[j * 2 + i] = (ey + j) * nfx + (ex + i);
            for (int k = 0; k < 4; ++k) {
                const int Ik = A[k] % nfx, Jk = A[k] / nfx;
                if (on_boundary(Ik, Jk, nfx, nfy)) continue;
                double s = 0;
                for (int l = 0; l < 4; ++l) {
                    const int Il = A[l] % nfx, Jl = A[l] / nfx;
                    if (!on_boundary(Il, Jl, nfx, nfy)) s += K[k * 4 + l] * x[A[l]];
                }
                y[A[k]] += s;
            }
        }
    for (int J = 0; J < nfy; ++J)
        for (int I = 0; I < nfx; ++I)
            if (on_boundary(I, J, nfx, nfy)) y[(size_t)J * nfx + I] = x[(size_t)J * nfx + I];
}

static double dot(const double *a, const double *b, long n)
{
    double s = 0.0;
    for (long i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* Inner solve of the PC: CG + Jacobi on the FEM matrix
 * (matrix_free/iteration_number_fempc_mf.cpp:11-17,210-224). */
static void fem_pc_apply(int nfx, int nfy, const double *gx, const double *gy, const double *r,
                         double *z, double rtol, int maxit, double *diag, double *w)
{
    const long N = (long)nfx * nfy;
    double *res = w, *pz = w + N, *pp = w + 2 * N, *ap = w + 3 * N;
    memset(z, 0, sizeof(double) * N);
    memcpy(res, r, sizeof(double) * N);
    const double r0 = sqrt(dot(res, res, N));
    if (r0 == 0.0) return;
    for (long i = 0; i < N; ++i) pz[i] = res[i] / diag[i];
    memcpy(pp, pz, sizeof(double) * N);
    double rz = dot(res, pz, N);
    for (int it = 0; it < maxit; ++it) {
        orc_fem_matvec(nfx, nfy, gx, gy, pp, ap, 1.0);
        const double alpha = rz / dot(pp, ap, N);
        for (long i = 0; i < N; ++i) {
            z[i] += alpha * pp[i];
            res[i] -= alpha * ap[i];
        }
        if (sqrt(dot(res, res, N)) <= rtol * r0) break;
        for (long i = 0; i < N; ++i) pz[i] = res[i] / diag[i];
        const double rz2 = dot(res, pz, N);
        const double beta = rz2 / rz;
        rz = rz2;
        for (long i = 0; i < N; ++i) pp[i] = pz[i] + beta * pp[i];
    }
}

int orc_pcg(const orc_patch *P, const double *gx, const double *gy, const double *b, double *x,
            double rtol, int maxit, double inner_rtol, int inner_maxit, double *relres_out)
{
    const int m = P->nex + P->p, nn = P->ney + P->q;
    const long N = (long)m * nn;
    double *r = calloc(N, sizeof(double)), *z = calloc(N, sizeof(double));
    double *pv = calloc(N, sizeof(double)), *ap = calloc(N, sizeof(double));
    double *diag = calloc(N, sizeof(double)), *w = calloc(4 * N, sizeof(double));
    double *e = calloc(N, sizeof(double));
    /* Jacobi diagonal of the FEM matrix, one unit vector at a time is too slow:
     * assemble it from the 2x2-Gauss element diagonals directly. */
    for (long i = 0; i < N; ++i) {
        const int I = (int)(i % m), J = (int)(i / m);
        if (on_boundary(I, J, m, nn)) { diag[i] = 1.0; continue; }
        double s = 0.0;
        for (int dy = -1; dy <= 0; ++dy)
            for (int dx = -1; dx <= 0; ++dx) {
                const int ex = I + dx, ey = J + dy;
                const double hx = gx[ex + 1] - gx[ex], hy = gy[ey + 1] - gy[ey];
                /* diagonal entry of a bilinear element: hy/(3hx) + hx/(3hy) */
                s += hy / (3.0 * hx) + hx / (3.0 * hy);
            }
        diag[i] = s;
    }
    const double bn = sqrt(dot(b, b, N));
    orc_apply_mf(P, x, ap, 1.0, 1);
    for (long i = 0; i < N; ++i) r[i] = b[i] - ap[i];
    double relres = sqrt(dot(r, r, N)) / bn;
    int it = 0;
    if (relres > rtol) {
        fem_pc_apply(m, nn, gx, gy, r, z, inner_rtol, inner_maxit, diag, w);
        memcpy(pv, z, sizeof(double) * N);
        double rz = dot(r, z, N);
        for (it = 1; it <= maxit; ++it) {
            orc_apply_mf(P, pv, ap, 1.0, 1);
            const double alpha = rz / dot(pv, ap, N);
            for (long i = 0; i < N; ++i) {
                x[i] += alpha * pv[i];
                r[i] -= alpha * ap[i];
            }
            orc_apply_mf(P, x, e, 1.0, 1);   /* true residual */
            double tr = 0.0;
            for (long i = 0; i < N; ++i) tr += (b[i] - e[i]) * (b[i] - e[i]);
            relres = sqrt(tr) / bn;
            if (relres <= rtol) break;
            fem_pc_apply(m, nn, gx, gy, r, z, inner_rtol, inner_maxit, diag, w);
            const double rz2 = dot(r, z, N);
            const double beta = rz2 / rz;
            rz = rz2;
            for (long i = 0; i < N; ++i) pv[i] = z[i] + beta * pv[i];
        }
    }
    if (relres_out) *relres_out = relres;
    free(r); free(z); free(pv); free(ap); free(diag); free(w); free(e);
    return (relres <= rtol) ? it : -it - 1;
}
