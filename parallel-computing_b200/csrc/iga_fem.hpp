// 1-D ingredients of the bilinear FEM preconditioner grid, shared by the
// single-patch and the batched solvers.
#pragma once
#include <vector>

#include "iga_host.hpp"

namespace iga {

// Linear-element stiffness (kd diagonal, ko[i] = K(i, i+1)) and mass (md, mo)
// matrices of the 1-D node set g.
void fem_1d(const std::vector<double> &g, std::vector<double> &kd, std::vector<double> &ko, std::vector<double> &md,
            std::vector<double> &mo);

// 1-D FEM nodes (one per IGA control point) on [0, L]: degree p-2 Greville
// abscissae of the shortened knot vector (matrix_free/preprocess_fem.cpp:38-60)
// for p >= 3, the degree-2 Greville abscissae of the IGA knots for p = 2.
std::vector<double> fem_nodes_1d(int p, int ne, double L);

// Mean polyline lengths of the control net's rows (Lx) and columns (Ly).
void net_lengths(const Patch &P, double &Lx, double &Ly);

// The pencil (K, M) of fem_1d restricted to the free nodes 1 .. n-2.
void interior_pencil(const std::vector<double> &g, std::vector<double> &Kd, std::vector<double> &Ko,
                     std::vector<double> &Md, std::vector<double> &Mo);

}  // namespace iga
