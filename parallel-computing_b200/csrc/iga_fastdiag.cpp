// Generalised eigenpairs of a symmetric tridiagonal pencil (K, M), M SPD:
// K v = lambda M v with V^T M V = I. Used to invert the tensor-product FEM
// preconditioner matrix K_fem = Kx (x) My + Mx (x) Ky exactly ("fast
// diagonalisation"): K_fem^-1 = (Vy (x) Vx) (I (x) Lx + Ly (x) I)^-1 (Vy (x) Vx)^T.
//
// Eigenvalues: bisection on Sylvester inertia counts of K - s M (the number
// of negative pivots of its LDL^T factorisation equals the number of
// eigenvalues below s). Eigenvectors: inverse iteration with a tridiagonal
// LU factorisation with partial pivoting, M-normalised.
#include "iga_fastdiag.hpp"

#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

namespace iga {

static int count_below(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo, double s)
{
    int neg = 0;
    double d = 1.0;
    for (int i = 0; i < n; ++i) {
        const double a = Kd[i] - s * Md[i];
        const double b = i > 0 ? (Ko[i - 1] - s * Mo[i - 1]) : 0.0;
        d = a - (i > 0 ? b * b / d : 0.0);
        if (d == 0.0) d = -1e-300;
        if (d < 0.0) ++neg;
    }
    return neg;
}

// Solve (K - s M) x = rhs for a tridiagonal matrix, LU with partial pivoting.
// Pivots smaller than `floor` (s is an eigenvalue to machine precision, and
// may make the matrix exactly singular) are raised to it, as in classical
// inverse iteration: the solution then grows like 1/floor along the
// eigenvector instead of overflowing.
static void tri_solve_pivot(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo, double s,
                            const double *rhs, double *x, std::vector<double> &w, double floor)
{
    // rows: sub l[i] (i,i-1), diag d[i], sup u[i] (i,i+1), second sup u2[i] (fill-in)
    w.resize(5 * (size_t)n);
    double *l = w.data(), *d = l + n, *u = d + n, *u2 = u + n, *y = u2 + n;
    for (int i = 0; i < n; ++i) {
        d[i] = Kd[i] - s * Md[i];
        u[i] = i + 1 < n ? Ko[i] - s * Mo[i] : 0.0;
        l[i] = i > 0 ? Ko[i - 1] - s * Mo[i - 1] : 0.0;
        u2[i] = 0.0;
        y[i] = rhs[i];
    }
    // Gaussian elimination with row interchanges between rows i and i+1.
    for (int i = 0; i + 1 < n; ++i) {
        if (std::fabs(l[i + 1]) > std::fabs(d[i])) {
            // swap rows i and i+1 (row i+1 has entries l[i+1] at col i, d[i+1] at i+1, u[i+1] at i+2)
            std::swap(d[i], l[i + 1]);
            std::swap(u[i], d[i + 1]);
            std::swap(u2[i], u[i + 1]);
            std::swap(y[i], y[i + 1]);
        }
        if (std::fabs(d[i]) < floor) d[i] = d[i] < 0.0 ? -floor : floor;
        const double f = l[i + 1] / d[i];
        l[i + 1] = 0.0;
        d[i + 1] -= f * u[i];
        u[i + 1] -= f * u2[i];
        y[i + 1] -= f * y[i];
    }
    if (std::fabs(d[n - 1]) < floor) d[n - 1] = d[n - 1] < 0.0 ? -floor : floor;
    for (int i = n - 1; i >= 0; --i) {
        double v = y[i];
        if (i + 1 < n) v -= u[i] * x[i + 1];
        if (i + 2 < n) v -= u2[i] * x[i + 2];
        x[i] = v / d[i];
    }
}

// Eigenvalues by bisection on inertia counts (ascending), `threads` host
// threads over the eigenvalues.
void pencil_eigvals(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo, double *lam,
                    int threads)
{
    if (n <= 0) return;
    const double hi0 = pencil_upper_bound(n, Kd, Ko, Md, Mo);
    const unsigned nt = (unsigned)std::max(1, std::min(threads, n));
    std::vector<std::thread> pool;
    auto work = [=](unsigned t) {
        for (int k = (int)t; k < n; k += (int)nt) {
            double lo = 0.0, hi = hi0;
            for (int it = 0; it < 200 && hi - lo > 4e-16 * hi; ++it) {
                const double mid = 0.5 * (lo + hi);
                if (count_below(n, Kd, Ko, Md, Mo, mid) > k) hi = mid;
                else lo = mid;
            }
            lam[k] = 0.5 * (lo + hi);
        }
    };
    if (nt == 1) work(0);
    else {
        for (unsigned t = 0; t < nt; ++t) pool.emplace_back(work, t);
        for (auto &th : pool) th.join();
    }
}

// Eigenvectors for given eigenvalues: inverse iteration with a tridiagonal
// LU factorisation with partial pivoting, M-normalised, the largest
// component positive; eigenvalues that coincide to working precision (e.g.
// two modes localised at the two ends of a symmetric grid, which give inverse
// iteration no way to tell their vectors apart) are handled cluster by
// cluster, each vector M-orthogonalised against the cluster's earlier ones
// after every solve.
void pencil_eigvecs(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo, const double *lam,
                    double *V, int threads)
{
    if (n <= 0) return;
    double kmax = 0.0, mmax = 0.0;
    for (int i = 0; i < n; ++i) {
        const double ko = (i > 0 ? std::fabs(Ko[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(Ko[i]) : 0.0);
        const double mo = (i > 0 ? std::fabs(Mo[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(Mo[i]) : 0.0);
        kmax = std::max(kmax, std::fabs(Kd[i]) + ko);
        mmax = std::max(mmax, Md[i] + mo);
    }
    const unsigned nt = (unsigned)std::max(1, std::min(threads, n));
    auto work = [=](unsigned t) {
        std::vector<double> w, v(n), x(n), mv(n);
        for (int k = (int)t; k < n; k += (int)nt) {
            const double s0 = lam[k];
            const double floor = 4e-16 * (kmax + s0 * mmax);
            bool ok = false;
            for (int attempt = 0; attempt < 4 && !ok; ++attempt) {
                // shift perturbed on retries only
                const double s = s0 * (1.0 + (attempt ? 1e-13 * attempt : 0.0));
                for (int i = 0; i < n; ++i) v[i] = 1.0 + 0.5 * std::sin(0.7 * (i + 1) + 1.3 * (k + 1) + attempt);
                ok = true;
                for (int it = 0; it < 3 && ok; ++it) {
                    for (int i = 0; i < n; ++i) {   // M v
                        double a = Md[i] * v[i];
                        if (i > 0) a += Mo[i - 1] * v[i - 1];
                        if (i + 1 < n) a += Mo[i] * v[i + 1];
                        mv[i] = a;
                    }
                    tri_solve_pivot(n, Kd, Ko, Md, Mo, s, mv.data(), x.data(), w, floor);
                    double nrm = 0.0;
                    for (int i = 0; i < n; ++i) {
                        double a = Md[i] * x[i];
                        if (i > 0) a += Mo[i - 1] * x[i - 1];
                        if (i + 1 < n) a += Mo[i] * x[i + 1];
                        nrm += a * x[i];
                    }
                    if (!(nrm > 0.0) || !std::isfinite(nrm)) {
                        ok = false;
                        break;
                    }
                    nrm = std::sqrt(nrm);
                    for (int i = 0; i < n; ++i) v[i] = x[i] / nrm;
                }
            }
            int imax = 0;
            for (int i = 1; i < n; ++i)
                if (std::fabs(v[i]) > std::fabs(v[imax])) imax = i;
            const double sg = v[imax] < 0 ? -1.0 : 1.0;
            for (int i = 0; i < n; ++i) V[(size_t)k * n + i] = sg * v[i];
        }
    };
    if (nt == 1) work(0);
    else {
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nt; ++t) pool.emplace_back(work, t);
        for (auto &th : pool) th.join();
    }

    const double ctol = 1e-5 * lam[n - 1];
    std::vector<double> w, v(n), x(n), mv(n);
    auto mdot = [&](const double *a, const double *b) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) {
            double t = Md[i] * b[i];
            if (i > 0) t += Mo[i - 1] * b[i - 1];
            if (i + 1 < n) t += Mo[i] * b[i + 1];
            s += a[i] * t;
        }
        return s;
    };
    for (int k0 = 0; k0 < n;) {
        int k1 = k0;
        while (k1 + 1 < n && lam[k1 + 1] - lam[k1] < ctol) ++k1;
        for (int k = k0 + 1; k <= k1; ++k) {
            const double floor = 4e-16 * (kmax + lam[k] * mmax);
            for (int i = 0; i < n; ++i) v[i] = 1.0 + 0.5 * std::cos(0.37 * (i + 1) + 2.1 * (k + 1));
            for (int it = 0; it < 4; ++it) {
                for (int i = 0; i < n; ++i) {
                    double a = Md[i] * v[i];
                    if (i > 0) a += Mo[i - 1] * v[i - 1];
                    if (i + 1 < n) a += Mo[i] * v[i + 1];
                    mv[i] = a;
                }
                tri_solve_pivot(n, Kd, Ko, Md, Mo, lam[k], mv.data(), x.data(), w, floor);
                for (int pass = 0; pass < 2; ++pass)
                    for (int j = k0; j < k; ++j) {
                        const double *u = V + (size_t)j * n;
                        const double c = mdot(u, x.data());
                        for (int i = 0; i < n; ++i) x[i] -= c * u[i];
                    }
                const double nrm = std::sqrt(std::max(mdot(x.data(), x.data()), 1e-300));
                for (int i = 0; i < n; ++i) v[i] = x[i] / nrm;
            }
            for (int i = 0; i < n; ++i) V[(size_t)k * n + i] = v[i];
        }
        k0 = k1 + 1;
    }
}

void pencil_eig(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo, double *lam, double *V)
{
    const int nt = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    pencil_eigvals(n, Kd, Ko, Md, Mo, lam, nt);
    pencil_eigvecs(n, Kd, Ko, Md, Mo, lam, V, nt);
}

bool pencil_centrosymmetric(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo)
{
    if (n < 2) return false;
    auto sym = [](const double *v, int len) {
        double mx = 0.0, dif = 0.0;
        for (int i = 0; i < len; ++i) {
            mx = std::max(mx, std::fabs(v[i]));
            dif = std::max(dif, std::fabs(v[i] - v[len - 1 - i]));
        }
        return dif <= 1e-12 * mx;
    };
    return sym(Kd, n) && sym(Md, n) && sym(Ko, n - 1) && sym(Mo, n - 1);
}

void pencil_fold(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo, int parity,
                 std::vector<double> &kd, std::vector<double> &ko, std::vector<double> &md, std::vector<double> &mo)
{
    const int fo = n / 2, fe = n - fo, h = parity == 0 ? fe : fo;
    kd.assign(Kd, Kd + h);
    md.assign(Md, Md + h);
    ko.assign(h, 0.0);
    mo.assign(h, 0.0);
    for (int i = 0; i + 1 < h; ++i) {
        ko[i] = Ko[i];
        mo[i] = Mo[i];
    }
    if (h == 0) return;
    if (n % 2 == 0) {
        const double sg = parity == 0 ? 1.0 : -1.0;
        kd[h - 1] += sg * Ko[h - 1];
        md[h - 1] += sg * Mo[h - 1];
    } else if (parity == 0) {
        kd[h - 1] *= 0.5;
        md[h - 1] *= 0.5;
    }
}

}  // namespace iga
