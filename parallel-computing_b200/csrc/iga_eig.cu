// Eigenvalues of many symmetric tridiagonal pencils (K, M), M SPD, on the
// device: bisection on Sylvester inertia counts of K - s M, one thread per
// eigenvalue (interface in iga_fastdiag.hpp). The host version of the same
// bisection (iga_fastdiag.cpp) costs O(n^2) dependent divisions per pencil
// and dominated the set-up of batches and of large plans; here every
// eigenvalue of every pencil is an independent thread.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "iga_fastdiag.hpp"
#include "iga_plan.hpp"

namespace iga {

namespace {

struct EigSet {
    long long off;   // first entry of the pencil's arrays (and of its eigenvalues)
    long long voff;  // first entry of its eigenvectors (n x n)
    int n;
    double hi;       // upper bound of the spectrum (Gershgorin)
    double kmax, mmax;   // row-sum bounds of K and M (pivot floor of inverse iteration)
};

__device__ int find_set(const EigSet *__restrict__ sets, int nsets, long long t)
{
    int lo_s = 0, hi_s = nsets - 1;
    while (lo_s < hi_s) {
        const int mid = (lo_s + hi_s + 1) / 2;
        if (sets[mid].off <= t) lo_s = mid;
        else hi_s = mid - 1;
    }
    return lo_s;
}

// Number of eigenvalues of (K, M) below s: the negative pivots of the
// LDL^T factorisation of K - s M (zero pivots taken as a tiny negative).
__device__ int count_below_dev(const double *__restrict__ Kd, const double *__restrict__ Ko,
                               const double *__restrict__ Md, const double *__restrict__ Mo, int n, double s)
{
    int neg = 0;
    double d = 1.0;
    for (int i = 0; i < n; ++i) {
        const double a = Kd[i] - s * Md[i];
        const double b = i > 0 ? (Ko[i - 1] - s * Mo[i - 1]) : 0.0;
        d = a - (i > 0 ? b * b / d : 0.0);
        if (d == 0.0) d = -1e-300;
        neg += d < 0.0;
    }
    return neg;
}

// Thread t: eigenvalue k = t - off of the set whose range holds t (sets in
// ascending offset order; found by binary search over the few sets).
__global__ void eig_bisect_kernel(const EigSet *__restrict__ sets, int nsets, long long total,
                                  const double *__restrict__ Kd, const double *__restrict__ Ko,
                                  const double *__restrict__ Md, const double *__restrict__ Mo,
                                  double *__restrict__ lam)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    const EigSet S = sets[find_set(sets, nsets, t)];
    const int k = (int)(t - S.off);
    const double *kd = Kd + S.off, *ko = Ko + S.off, *md = Md + S.off, *mo = Mo + S.off;
    double lo = 0.0, hi = S.hi;
    for (int it = 0; it < 200 && hi - lo > 4e-16 * hi; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (count_below_dev(kd, ko, md, mo, S.n, mid) > k) hi = mid;
        else lo = mid;
    }
    lam[t] = 0.5 * (lo + hi);
}

// Eigenvector of eigenvalue t (thread t, as above): inverse iteration, three
// solves of (K - s M) x = M v with a tridiagonal LU factorisation with
// partial pivoting (pivots below `floor` raised to it), M-normalised, the
// largest component positive; up to four attempts with a perturbed shift
// and start vector if a solve breaks down. The same method as the host's
// pencil_eigvecs (without its handling of coincident eigenvalues, which the
// caller does on the host). Per-thread work arrays in `w`, entry i of array
// j of thread t at (j n_max + i) total + t (coalesced over the threads).
__global__ void eig_vec_kernel(const EigSet *__restrict__ sets, int nsets, long long total, int nmax,
                               const double *__restrict__ Kd, const double *__restrict__ Ko,
                               const double *__restrict__ Md, const double *__restrict__ Mo,
                               const double *__restrict__ lam, double *__restrict__ w, double *__restrict__ V)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    const EigSet S = sets[find_set(sets, nsets, t)];
    const int k = (int)(t - S.off), n = S.n;
    const double *kd = Kd + S.off, *ko = Ko + S.off, *md = Md + S.off, *mo = Mo + S.off;
    auto at = [&](int j, int i) -> double & { return w[((long long)j * nmax + i) * total + t]; };
    // arrays: 0 l, 1 d, 2 u, 3 u2, 4 y, 5 x, 6 v, 7 mv
    const double s0 = lam[t];
    const double floor = 4e-16 * (S.kmax + s0 * S.mmax);
    bool ok = false;
    for (int attempt = 0; attempt < 4 && !ok; ++attempt) {
        const double s = s0 * (1.0 + (attempt ? 1e-13 * attempt : 0.0));
        for (int i = 0; i < n; ++i) at(6, i) = 1.0 + 0.5 * sin(0.7 * (i + 1) + 1.3 * (k + 1) + attempt);
        ok = true;
        for (int it = 0; it < 3 && ok; ++it) {
            for (int i = 0; i < n; ++i) {   // mv = M v, and the factors of K - s M
                double a = md[i] * at(6, i);
                if (i > 0) a += mo[i - 1] * at(6, i - 1);
                if (i + 1 < n) a += mo[i] * at(6, i + 1);
                at(4, i) = a;
                at(1, i) = kd[i] - s * md[i];
                at(2, i) = i + 1 < n ? ko[i] - s * mo[i] : 0.0;
                at(0, i) = i > 0 ? ko[i - 1] - s * mo[i - 1] : 0.0;
                at(3, i) = 0.0;
            }
            for (int i = 0; i + 1 < n; ++i) {   // elimination with row interchanges of rows i, i+1
                double di = at(1, i), ui = at(2, i), u2i = at(3, i), yi = at(4, i);
                double l1 = at(0, i + 1), d1 = at(1, i + 1), u1 = at(2, i + 1), y1 = at(4, i + 1);
                if (fabs(l1) > fabs(di)) {
                    double tmp = di; di = l1; l1 = tmp;
                    tmp = ui; ui = d1; d1 = tmp;
                    tmp = u2i; u2i = u1; u1 = tmp;
                    tmp = yi; yi = y1; y1 = tmp;
                }
                if (fabs(di) < floor) di = di < 0.0 ? -floor : floor;
                const double f = l1 / di;
                d1 -= f * ui;
                u1 -= f * u2i;
                y1 -= f * yi;
                at(1, i) = di; at(2, i) = ui; at(3, i) = u2i; at(4, i) = yi;
                at(0, i + 1) = 0.0; at(1, i + 1) = d1; at(2, i + 1) = u1; at(4, i + 1) = y1;
            }
            if (fabs(at(1, n - 1)) < floor) at(1, n - 1) = at(1, n - 1) < 0.0 ? -floor : floor;
            for (int i = n - 1; i >= 0; --i) {   // back substitution into x
                double v = at(4, i);
                if (i + 1 < n) v -= at(2, i) * at(5, i + 1);
                if (i + 2 < n) v -= at(3, i) * at(5, i + 2);
                at(5, i) = v / at(1, i);
            }
            double nrm = 0.0;
            for (int i = 0; i < n; ++i) {
                double a = md[i] * at(5, i);
                if (i > 0) a += mo[i - 1] * at(5, i - 1);
                if (i + 1 < n) a += mo[i] * at(5, i + 1);
                nrm += a * at(5, i);
            }
            if (!(nrm > 0.0) || !isfinite(nrm)) {
                ok = false;
                break;
            }
            const double inv = 1.0 / sqrt(nrm);
            for (int i = 0; i < n; ++i) at(6, i) = at(5, i) * inv;
        }
    }
    int imax = 0;
    for (int i = 1; i < n; ++i)
        if (fabs(at(6, i)) > fabs(at(6, imax))) imax = i;
    const double sg = at(6, imax) < 0 ? -1.0 : 1.0;
    double *out = V + S.voff + (long long)k * n;
    for (int i = 0; i < n; ++i) out[i] = sg * at(6, i);
}

}  // namespace

double pencil_upper_bound(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo)
{
    double kmax = 0.0, mmin = 1e300;
    for (int i = 0; i < n; ++i) {
        const double ko = (i > 0 ? std::fabs(Ko[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(Ko[i]) : 0.0);
        const double mo = (i > 0 ? std::fabs(Mo[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(Mo[i]) : 0.0);
        kmax = std::max(kmax, std::fabs(Kd[i]) + ko);
        mmin = std::min(mmin, Md[i] - mo);
    }
    return kmax / std::max(mmin, 1e-300) * 1.01 + 1e-300;
}

int pencil_eig_device(int device, const std::vector<PencilRef> &P, std::vector<std::vector<double>> &lam,
                      std::vector<std::vector<double>> *vec, double **dvec, std::vector<long long> *voff)
{
    if (dvec) {
        *dvec = nullptr;
        vec = nullptr;
        if (voff) voff->assign(P.size(), -1);
    }
    lam.assign(P.size(), {});
    if (vec) vec->assign(P.size(), {});
    std::vector<EigSet> sets;
    long long total = 0, vtotal = 0;
    int nmax = 1;
    for (const PencilRef &p : P) {
        if (p.n <= 0) continue;
        double kmax = 0.0, mmax = 0.0;
        for (int i = 0; i < p.n; ++i) {
            const double ko = (i > 0 ? std::fabs(p.Ko[i - 1]) : 0.0) + (i + 1 < p.n ? std::fabs(p.Ko[i]) : 0.0);
            const double mo = (i > 0 ? std::fabs(p.Mo[i - 1]) : 0.0) + (i + 1 < p.n ? std::fabs(p.Mo[i]) : 0.0);
            kmax = std::max(kmax, std::fabs(p.Kd[i]) + ko);
            mmax = std::max(mmax, p.Md[i] + mo);
        }
        sets.push_back(EigSet{total, vtotal, p.n, pencil_upper_bound(p.n, p.Kd, p.Ko, p.Md, p.Mo), kmax, mmax});
        total += p.n;
        vtotal += (long long)p.n * p.n;
        nmax = std::max(nmax, p.n);
    }
    if (total == 0) return IGA_OK;
    // one host block: Kd | Ko | Md | Mo, each `total` long (off-diagonals padded to n per pencil)
    std::vector<double> h((size_t)total * 4, 0.0);
    {
        size_t q = 0;
        for (const PencilRef &p : P) {
            if (p.n <= 0) continue;
            for (int i = 0; i < p.n; ++i) {
                h[q + i] = p.Kd[i];
                h[(size_t)total + q + i] = i + 1 < p.n ? p.Ko[i] : 0.0;
                h[2 * (size_t)total + q + i] = p.Md[i];
                h[3 * (size_t)total + q + i] = i + 1 < p.n ? p.Mo[i] : 0.0;
            }
            q += p.n;
        }
    }
    int prev = 0;
    cudaGetDevice(&prev);
    double *d = nullptr, *dw = nullptr, *dv = nullptr;
    EigSet *ds = nullptr;
    auto release = [&]() {
        for (void *q : {(void *)d, (void *)dw, (void *)dv, (void *)ds})
            if (q) cudaFree(q);
        cudaSetDevice(prev);
    };
    auto fail = [&](cudaError_t e) {
        release();
        set_error(std::string("device eigenpairs: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? IGA_ERR_NOMEM : IGA_ERR_CUDA;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(e);
    if ((e = cudaMalloc((void **)&d, sizeof(double) * (size_t)total * 5)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc((void **)&ds, sizeof(EigSet) * sets.size())) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(d, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(ds, sets.data(), sizeof(EigSet) * sets.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e);
    double *dl = d + 4 * (size_t)total;
    const int threads = 128;
    const unsigned blocks = (unsigned)((total + threads - 1) / threads);
    eig_bisect_kernel<<<blocks, threads>>>(ds, (int)sets.size(), total, d, d + total, d + 2 * total, d + 3 * total, dl);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
    std::vector<double> hv;
    if (vec || dvec) {
        if ((e = cudaMalloc((void **)&dw, sizeof(double) * 8 * (size_t)nmax * (size_t)total)) != cudaSuccess ||
            (e = cudaMalloc((void **)&dv, sizeof(double) * (size_t)vtotal)) != cudaSuccess)
            return fail(e);
        eig_vec_kernel<<<blocks, threads>>>(ds, (int)sets.size(), total, nmax, d, d + total, d + 2 * total,
                                            d + 3 * total, dl, dw, dv);
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
        if (vec) {
            hv.resize((size_t)vtotal);
            if ((e = cudaMemcpy(hv.data(), dv, sizeof(double) * (size_t)vtotal, cudaMemcpyDeviceToHost)) != cudaSuccess)
                return fail(e);
        }
    }
    std::vector<double> hl((size_t)total);
    if ((e = cudaMemcpy(hl.data(), dl, sizeof(double) * (size_t)total, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return fail(e);
    double *keep = nullptr;
    if (dvec) {   // the caller takes the vectors' buffer
        keep = dv;
        dv = nullptr;
    }
    release();
    size_t q = 0, qv = 0;
    for (size_t k = 0; k < P.size(); ++k) {
        const int n = P[k].n;
        if (n <= 0) continue;
        lam[k].assign(hl.begin() + q, hl.begin() + q + n);
        q += n;
        if (dvec) {
            if (voff) (*voff)[k] = (long long)qv;
            const double ctol = 1e-5 * lam[k][n - 1];
            bool cluster = false;
            for (int a = 0; a + 1 < n && !cluster; ++a) cluster = lam[k][a + 1] - lam[k][a] < ctol;
            if (cluster) {   // as below, then over the device copy
                std::vector<double> V((size_t)n * n);
                pencil_eigvecs(n, P[k].Kd, P[k].Ko, P[k].Md, P[k].Mo, lam[k].data(), V.data(), 1);
                cudaSetDevice(device);
                e = cudaMemcpy(keep + qv, V.data(), sizeof(double) * V.size(), cudaMemcpyHostToDevice);
                cudaSetDevice(prev);
                if (e != cudaSuccess) {
                    cudaFree(keep);
                    set_error(std::string("device eigenpairs: ") + cudaGetErrorString(e));
                    return IGA_ERR_CUDA;
                }
            }
            qv += (size_t)n * n;
        }
        if (vec) {
            std::vector<double> &V = (*vec)[k];
            V.assign(hv.begin() + qv, hv.begin() + qv + (size_t)n * n);
            qv += (size_t)n * n;
            // eigenvalues that coincide to working precision: inverse iteration
            // cannot tell their vectors apart; redo this pencil's vectors on the
            // host, which orthogonalises within such clusters
            const double ctol = 1e-5 * lam[k][n - 1];
            bool cluster = false;
            for (int a = 0; a + 1 < n && !cluster; ++a) cluster = lam[k][a + 1] - lam[k][a] < ctol;
            if (cluster) pencil_eigvecs(n, P[k].Kd, P[k].Ko, P[k].Md, P[k].Mo, lam[k].data(), V.data(), 1);
        }
    }
    if (dvec) *dvec = keep;
    return IGA_OK;
}

int pencil_eigvals_device(int device, const std::vector<PencilRef> &P, std::vector<std::vector<double>> &lam)
{
    return pencil_eig_device(device, P, lam, nullptr, nullptr, nullptr);
}

}  // namespace iga
