// Generalised eigenpairs of symmetric tridiagonal pencils (see iga_fastdiag.cpp).
#pragma once

namespace iga {

// K = tridiag(Ko, Kd, Ko), M = tridiag(Mo, Md, Mo) of size n (off arrays hold
// entry (i, i+1) at index i). Outputs ascending eigenvalues lam[n] and
// M-normalised eigenvectors, column-major: V[k*n + i] = component i of vector k.
void pencil_eig(int n, const double *Kd, const double *Ko, const double *Md, const double *Mo, double *lam, double *V);

}  // namespace iga
