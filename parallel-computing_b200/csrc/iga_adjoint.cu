// Variable coefficient kappa and the adjoint gradient dJ/dkappa
// (no counterpart in the reference, whose operator has kappa = 1).
//
// For -div(kappa grad u) = f discretised with kappa at the quadrature points,
// K(kappa) = sum_q kappa_q K_q, and for J(u(kappa)) with K lambda = dJ/du
// (lambda = 0 on the boundary):
//     dJ/dkappa_q = -lambda^T K_q u = -(grad lambda . grad u)(x_q) * JxW_q.
// K is symmetric, so the adjoint solve is the forward solver with another
// right-hand side.
#include <cuda_runtime.h>

#include <string>

#include "../../include/iga_solve.h"
#include "iga_plan.hpp"

namespace iga {

// One thread per (element, quadrature point): gradients of u and lambda in
// reference coordinates, geometry from the control points, no kappa.
__global__ void adjoint_grad_kernel(const double *__restrict__ u, const double *__restrict__ lam,
                                    double *__restrict__ g, const double *__restrict__ tabX64,
                                    const double *__restrict__ tabY64, const double *__restrict__ CP,
                                    const double *__restrict__ qw, StripGrid sg)
{
    const int P = sg.P, NB = P + 1, NQ = P + 1, NQ2 = NQ * NQ;
    const long long total = (long long)sg.nex * sg.ney * NQ2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int qp = (int)(t % NQ2);
        const long long e = t / NQ2;
        const int ex = (int)(e % sg.nex), ey = (int)(e / sg.nex);
        const int qx = qp % NQ, qy = qp / NQ;
        double x_xi = 0, x_eta = 0, y_xi = 0, y_eta = 0, u_xi = 0, u_eta = 0, l_xi = 0, l_eta = 0;
        for (int jl = 0; jl < NB; ++jl) {
            const double n2 = tabY64[((size_t)(ey * 2 + 0) * NQ + qy) * NB + jl];
            const double d2 = tabY64[((size_t)(ey * 2 + 1) * NQ + qy) * NB + jl];
            for (int il = 0; il < NB; ++il) {
                const double n1 = tabX64[((size_t)(ex * 2 + 0) * NQ + qx) * NB + il];
                const double d1 = tabX64[((size_t)(ex * 2 + 1) * NQ + qx) * NB + il];
                const size_t A = (size_t)(ey + jl) * sg.m + (ex + il);
                const double a_xi = d1 * n2, a_eta = n1 * d2;
                x_xi += CP[2 * A] * a_xi;
                x_eta += CP[2 * A] * a_eta;
                y_xi += CP[2 * A + 1] * a_xi;
                y_eta += CP[2 * A + 1] * a_eta;
                u_xi += u[A] * a_xi;
                u_eta += u[A] * a_eta;
                l_xi += lam[A] * a_xi;
                l_eta += lam[A] * a_eta;
            }
        }
        const double det = x_xi * y_eta - x_eta * y_xi;
        const double f = qw[qx] * qw[qy] / det;
        const double g00 = f * (x_eta * x_eta + y_eta * y_eta);
        const double g01 = -f * (x_xi * x_eta + y_xi * y_eta);
        const double g11 = f * (x_xi * x_xi + y_xi * y_xi);
        g[t] = -(l_xi * (g00 * u_xi + g01 * u_eta) + l_eta * (g01 * u_xi + g11 * u_eta));
    }
}

}  // namespace iga

using namespace iga;

extern "C" {

int iga_adjoint_grad(iga_plan *pl, const double *u, const double *lam, double *g, void *stream)
{
    if (!pl || !u || !lam || !g) return IGA_ERR_ARG;
    adjoint_grad_kernel<<<4 * 148, 256, 0, (cudaStream_t)stream>>>(u, lam, g, pl->tabX64, pl->tabY64, pl->CP, pl->qw,
                                                                  pl->grid);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("iga_adjoint_grad: ") + cudaGetErrorString(e));
        return IGA_ERR_CUDA;
    }
    return IGA_OK;
}

}  // extern "C"
