#include "iga_host.hpp"

#include <cmath>
#include <cstring>

namespace iga {

void gauss01(int n, double *x, double *w)
{
    const double pi = 3.141592653589793238462643383279;
    for (int i = 0; i < n; ++i) {
        double t = std::cos(pi * (i + 0.75) / (n + 0.5));
        double pn = 0.0, pm = 1.0, dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            pm = 1.0;
            pn = t;
            for (int k = 2; k <= n; ++k) {
                const double pk = ((2.0 * k - 1.0) * t * pn - (k - 1.0) * pm) / k;
                pm = pn;
                pn = pk;
            }
            if (n == 1) { pn = t; pm = 1.0; }
            dp = n * (t * pn - pm) / (t * t - 1.0);
            const double dt = pn / dp;
            t -= dt;
            if (std::fabs(dt) < 1e-17) break;
        }
        pm = 1.0;
        pn = t;
        for (int k = 2; k <= n; ++k) {
            const double pk = ((2.0 * k - 1.0) * t * pn - (k - 1.0) * pm) / k;
            pm = pn;
            pn = pk;
        }
        if (n == 1) { pn = t; pm = 1.0; }
        dp = n * (t * pn - pm) / (t * t - 1.0);
        x[n - 1 - i] = 0.5 * (t + 1.0);
        w[n - 1 - i] = 1.0 / ((1.0 - t * t) * dp * dp);
    }
}

void bernstein(int p, double xi, double *B, double *dB)
{
    // de Casteljau-style build-up of the degree-d values, keeping degree p-1
    // for the derivative identity dB_k = p (B^{p-1}_{k-1} - B^{p-1}_k).
    double prev[16];
    for (int k = 0; k <= p; ++k) B[k] = 0.0;
    B[0] = 1.0;
    for (int d = 1; d <= p; ++d) {
        if (d == p) std::memcpy(prev, B, sizeof(double) * p);
        for (int k = d; k >= 0; --k)
            B[k] = (k > 0 ? xi * B[k - 1] : 0.0) + (k < d ? (1.0 - xi) * B[k] : 0.0);
    }
    for (int k = 0; k <= p; ++k)
        dB[k] = (p == 0) ? 0.0 : p * ((k > 0 ? prev[k - 1] : 0.0) - (k < p ? prev[k] : 0.0));
}

std::vector<double> open_knots(int p, int ne, double L)
{
    std::vector<double> S;
    S.reserve(ne + 2 * p + 1);
    for (int i = 0; i <= p; ++i) S.push_back(0.0);
    for (int i = 1; i < ne; ++i) S.push_back(i * (L / ne));
    for (int i = 0; i <= p; ++i) S.push_back(L);
    return S;
}

std::vector<double> extraction(int p, const std::vector<double> &U)
{
    // Borden et al. 2011, Algorithm 1, with 0-based knot indices: the element
    // being closed starts at knot a, the scan position is b.
    const int nk = (int)U.size(), a1 = p + 1;
    const int maxe = nk - 2 * p - 1;
    std::vector<double> C((size_t)std::max(maxe, 1) * a1 * a1, 0.0);
    auto at = [&](int e, int r, int c) -> double & { return C[((size_t)e * a1 + r) * a1 + c]; };
    for (int i = 0; i < a1; ++i) at(0, i, i) = 1.0;
    int e = 0, a = p, b = p + 1;
    std::vector<double> alpha(p + 2);
    while (b < nk - 1) {
        if (e + 1 < maxe)
            for (int i = 0; i < a1; ++i) at(e + 1, i, i) = 1.0;
        const int b0 = b;
        while (b < nk - 1 && U[b + 1] == U[b]) ++b;
        const int mult = b - b0 + 1;
        if (mult < p) {
            const double numer = U[b] - U[a];
            for (int j = p; j > mult; --j) alpha[j - mult] = numer / (U[a + j] - U[a]);
            const int r = p - mult;
            for (int j = 1; j <= r; ++j) {
                const int save = r - j, s = mult + j;
                for (int k = p; k >= s; --k) {
                    const double al = alpha[k - s + 1];
                    for (int row = 0; row < a1; ++row) at(e, row, k) = al * at(e, row, k) + (1.0 - al) * at(e, row, k - 1);
                }
                if (b < nk - 1 && e + 1 < maxe)
                    for (int o = 0; o <= j; ++o) at(e + 1, save + o, save) = at(e, p - j + o, p);
            }
        }
        if (b < nk - 1) {
            ++e;
            a = b;
            ++b;
        }
    }
    C.resize((size_t)(e + 1) * a1 * a1);
    return C;
}

std::vector<double> greville(int p, const std::vector<double> &U)
{
    const int n = (int)U.size() - p - 1;
    std::vector<double> g(n, 0.0);
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int j = 1; j <= p; ++j) s += U[i + j];
        g[i] = s / p;
    }
    return g;
}

Tables1D tables_1d(int p, int ne, const double *C, const double *wt)
{
    Tables1D t;
    t.p = p;
    t.ne = ne;
    const int nb = p + 1, nq = p + 1;
    t.val.assign((size_t)ne * nq * nb, 0.0);
    t.der.assign((size_t)ne * nq * nb, 0.0);
    std::vector<double> qx(nq), qw(nq), B(nb), dB(nb);
    gauss01(nq, qx.data(), qw.data());
    for (int e = 0; e < ne; ++e) {
        const double *Ce = C + (size_t)e * nb * nb;
        for (int k = 0; k < nq; ++k) {
            bernstein(p, qx[k], B.data(), dB.data());
            double N[16], dN[16];
            for (int i = 0; i < nb; ++i) {   // N = C_e B (matrix_free/src/RefElement.cpp:20-57)
                double s = 0.0, d = 0.0;
                for (int l = 0; l < nb; ++l) {
                    s += Ce[i * nb + l] * B[l];
                    d += Ce[i * nb + l] * dB[l];
                }
                N[i] = s;
                dN[i] = d;
            }
            if (wt) {   // 1-D rational basis R_i = w_i N_i / W
                double W = 0.0, dW = 0.0;
                for (int i = 0; i < nb; ++i) {
                    W += wt[e + i] * N[i];
                    dW += wt[e + i] * dN[i];
                }
                for (int i = 0; i < nb; ++i) {
                    const double R = wt[e + i] * N[i] / W;
                    dN[i] = (wt[e + i] * dN[i] - dW * R) / W;
                    N[i] = R;
                }
            }
            for (int i = 0; i < nb; ++i) {
                t.val[((size_t)e * nq + k) * nb + i] = N[i];
                t.der[((size_t)e * nq + k) * nb + i] = dN[i];
            }
        }
    }
    return t;
}

// ------------------------------------------------------------ NURBS annulus
namespace {
using Hpt = std::vector<double>;   // homogeneous point (w x, w y, w)

// Degree elevation of one Bezier segment: Q_i = i/(p+1) P_{i-1} + (1 - i/(p+1)) P_i.
std::vector<Hpt> bezier_elevate(const std::vector<Hpt> &P)
{
    const int p = (int)P.size() - 1;
    std::vector<Hpt> Q(p + 2, Hpt(P[0].size(), 0.0));
    for (int i = 0; i <= p + 1; ++i) {
        const double a = (double)i / (p + 1);
        for (size_t d = 0; d < P[0].size(); ++d)
            Q[i][d] = (i > 0 ? a * P[i - 1][d] : 0.0) + (i <= p ? (1.0 - a) * P[i][d] : 0.0);
    }
    return Q;
}

// Boehm's single knot insertion of u into a degree-p curve (homogeneous).
void insert_knot(std::vector<Hpt> &P, std::vector<double> &U, int p, double u)
{
    int k = p;
    while (k + 1 < (int)U.size() - p - 1 && U[k + 1] <= u) ++k;   // U[k] <= u < U[k+1]
    std::vector<Hpt> Q(P.size() + 1, Hpt(P[0].size(), 0.0));
    for (int i = 0; i <= k - p; ++i) Q[i] = P[i];
    for (int i = k - p + 1; i <= k; ++i) {
        const double a = (u - U[i]) / (U[i + p] - U[i]);
        for (size_t d = 0; d < P[0].size(); ++d) Q[i][d] = a * P[i][d] + (1.0 - a) * P[i - 1][d];
    }
    for (int i = k + 1; i < (int)Q.size(); ++i) Q[i] = P[i - 1];
    U.insert(U.begin() + k + 1, u);
    P.swap(Q);
}

// Coarse single-segment curve elevated to degree p and refined to ne elements on [0,1].
std::vector<Hpt> elevate_refine(std::vector<Hpt> P, int p, int ne)
{
    while ((int)P.size() - 1 < p) P = bezier_elevate(P);
    std::vector<double> U(p + 1, 0.0);
    U.insert(U.end(), p + 1, 1.0);
    for (int k = 1; k < ne; ++k) insert_knot(P, U, p, (double)k / ne);
    return P;
}
}  // namespace

void quarter_annulus(int p, int ner, int net, double r_in, double r_out, std::vector<double> &CP,
                     std::vector<double> &W, std::vector<double> &C1, std::vector<double> &C2)
{
    // radial: r(xi) = r_in + (r_out - r_in) xi as a linear Bezier segment (weights 1)
    const std::vector<Hpt> rad = elevate_refine({{r_in, 1.0}, {r_out, 1.0}}, p, ner);
    // angular: unit quarter circle, rational quadratic, homogeneous (w x, w y, w)
    const double s2 = std::sqrt(0.5);
    const std::vector<Hpt> ang = elevate_refine({{1.0, 0.0, 1.0}, {s2, s2, s2}, {0.0, 1.0, 1.0}}, p, net);
    const int m = (int)rad.size(), n = (int)ang.size();
    CP.assign(2 * (size_t)m * n, 0.0);
    W.assign((size_t)m * n, 0.0);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            const double r = rad[i][0] / rad[i][1], w = ang[j][2];
            CP[2 * ((size_t)j * m + i)] = r * ang[j][0] / w;
            CP[2 * ((size_t)j * m + i) + 1] = r * ang[j][1] / w;
            W[(size_t)j * m + i] = w;
        }
    C1 = extraction(p, open_knots(p, ner, 1.0));
    C2 = extraction(p, open_knots(p, net, 1.0));
}

static bool factor_weights(const double *w, int m, int n, std::vector<double> &a, std::vector<double> &b)
{
    // w(i,j) = a(i) b(j) with a(0) = 1 (scale-free factorisation).
    a.assign(m, 1.0);
    b.assign(n, 1.0);
    const double w00 = w[0];
    if (!(w00 > 0.0)) return false;
    for (int i = 0; i < m; ++i) a[i] = w[i] / w00;
    for (int j = 0; j < n; ++j) b[j] = w[(size_t)j * m];
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            const double ref = a[i] * b[j], got = w[(size_t)j * m + i];
            if (!(got > 0.0) || std::fabs(got - ref) > 1e-12 * std::fabs(ref)) return false;
        }
    return true;
}

std::string build_patch(const MeshDescView &d, Patch &P)
{
    if (d.p < 1 || d.p > 5) return "p must be in 1..5";
    if (d.q != d.p) return "this library requires p == q";
    if (d.nex < 1 || d.ney < 1) return "nElemX and nElemY must be positive";
    if (!d.CP) return "CP is required";
    P.p = d.p;
    P.q = d.q;
    P.nex = d.nex;
    P.ney = d.ney;
    P.m = d.nex + d.p;
    P.n = d.ney + d.q;
    const long long nf = (long long)P.m * P.n;
    if (nf > (1LL << 31) - 1) return "mesh too large for 32-bit indices";
    P.CP.assign(d.CP, d.CP + 2 * nf);
    const int nb = d.p + 1, nloc = nb * (d.q + 1);
    if (d.C1) P.C1.assign(d.C1, d.C1 + (size_t)d.nex * nb * nb);
    else {
        P.C1 = extraction(d.p, open_knots(d.p, d.nex, 1.0));
        if ((int)(P.C1.size() / (nb * nb)) != d.nex) return "extraction generation failed";
    }
    if (d.C2) P.C2.assign(d.C2, d.C2 + (size_t)d.ney * (d.q + 1) * (d.q + 1));
    else {
        P.C2 = extraction(d.q, open_knots(d.q, d.ney, 1.0));
        if ((int)(P.C2.size() / ((d.q + 1) * (d.q + 1))) != d.ney) return "extraction generation failed";
    }
    if (d.weights) {
        if (!factor_weights(d.weights, P.m, P.n, P.w1, P.w2))
            return "weights must be positive and factor as w(i,j) = a(i) b(j)";
    }
    if (d.IEN) {   // structured connectivity of matrix_free/src/IENGenerator.cpp:68-103
        for (int ey = 0; ey < d.ney; ++ey)
            for (int ex = 0; ex < d.nex; ++ex)
                for (int jl = 0; jl <= d.q; ++jl)
                    for (int il = 0; il <= d.p; ++il) {
                        const long long e = (long long)ey * d.nex + ex;
                        if (d.IEN[e * nloc + jl * nb + il] != (ey + jl) * P.m + ex + il)
                            return "IEN is not the structured single-patch connectivity";
                    }
    }
    auto bnd = [&](long long A) {
        const int i = (int)(A % P.m), j = (int)(A / P.m);
        return i == 0 || j == 0 || i == P.m - 1 || j == P.n - 1;
    };
    if (d.ID) {
        for (long long A = 0; A < nf; ++A) {
            const int expect = bnd(A) ? -1 : (int)A;
            if (d.ID[A] != expect) return "ID must be -1 on the boundary ring and the identity elsewhere";
        }
    }
    if (d.Dir) {
        long long k = 0;
        for (long long A = 0; A < nf; ++A)
            if (bnd(A)) {
                if (k >= d.nDir || d.Dir[k] != A) return "Dir must list the boundary ring in ascending order";
                ++k;
            }
        if (k != d.nDir) return "Dir must list the boundary ring in ascending order";
    }
    if (d.kappa) P.kappa.assign(d.kappa, d.kappa + (size_t)d.nex * d.ney * nloc);
    return "";
}

}  // namespace iga
