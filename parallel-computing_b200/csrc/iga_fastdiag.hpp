// Generalised eigenpairs of symmetric tridiagonal pencils (see iga_fastdiag.cpp).
#pragma once
#include <vector>

namespace iga {

// K = tridiag(Ko, Kd, Ko), M = tridiag(Mo, Md, Mo) of size n (off arrays hold
// entry (i, i+1) at index i). Outputs ascending eigenvalues lam[n] and
// M-normalised eigenvectors, column-major: V[k*n + i] = component i of vector k.
void pencil_eig(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo, double *lam, double *V);

// The two steps of pencil_eig: ascending eigenvalues by bisection, and the
// M-normalised eigenvectors of given eigenvalues by inverse iteration (host
// threads over the eigenpairs).
void pencil_eigvals(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo, double *lam,
                    int threads);
void pencil_eigvecs(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo, const double *lam,
                    double *V, int threads);
// Upper bound of the pencil's spectrum (Gershgorin, with a margin).
double pencil_upper_bound(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo);

// A pencil for the batched device bisection.
struct PencilRef {
    int n = 0;
    const double *Kd = nullptr, *Ko = nullptr, *Md = nullptr, *Mo = nullptr;
};
// Ascending eigenvalues of every pencil, computed on `device` (one thread
// per eigenvalue, the same bisection as pencil_eigvals); synchronous, host
// in and out. Returns IGA_OK or an IGA_ERR_* status.
int pencil_eigvals_device(int device, const std::vector<PencilRef> &P, std::vector<std::vector<double>> &lam);
// Eigenvalues and, when vec is set, M-normalised eigenvectors ((*vec)[k]:
// component i of vector a at a n + i), both computed on `device` (inverse
// iteration one thread per eigenpair; pencils with coincident eigenvalues
// get their vectors from pencil_eigvecs on the host).
// With dvec set, the vectors stay on the device instead: *dvec receives the
// buffer (all pencils' n x n blocks, the caller frees it) and (*voff)[k] the
// offset of pencil k's block; vec is then ignored.
int pencil_eig_device(int device, const std::vector<PencilRef> &P, std::vector<std::vector<double>> &lam,
                      std::vector<std::vector<double>> *vec, double **dvec = nullptr,
                      std::vector<long long> *voff = nullptr);

// Parity split of a centrosymmetric pencil (entry i equals entry n-1-i, to
// rounding): every eigenvector is symmetric (v[i] = v[n-1-i]) or
// antisymmetric, and each class is the eigenproblem of a half-size symmetric
// tridiagonal pencil in u = v[0 .. h-1], h = ceil(n/2) (parity 0) or
// floor(n/2) (parity 1):
//   n = 2h:   rows 0 .. h-1, the last diagonal entry plus (symmetric) or
//             minus (antisymmetric) the coupling (h-1, h);
//   n = 2h+1: symmetric: rows 0 .. h with the middle row's diagonal halved
//             (its row equation divided by 2, which makes the half pencil
//             symmetric); antisymmetric: rows 0 .. h-1 (the middle entry is 0).
// v^T M v = 2 u^T M_half u, so M_half-normalised half vectors are divided by
// sqrt 2 to give M-normalised full ones.
bool pencil_centrosymmetric(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo);
void pencil_fold(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo, int parity,
                 std::vector<double> &kd, std::vector<double> &ko, std::vector<double> &md, std::vector<double> &mo);

}  // namespace iga
