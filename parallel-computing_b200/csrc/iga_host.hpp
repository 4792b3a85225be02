// Host-side 1-D ingredients of the IGA patch: quadrature, Bernstein basis,
// knot vectors, Bezier extraction, Greville abscissae, and the per-element
// 1-D basis tables the device kernels consume.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace iga {

// Gauss-Legendre rule with n points on [0,1] (the reference tabulates the same
// rule: matrix_free/src/QuadraturePoint.cpp:3-58).
void gauss01(int n, double *x, double *w);

// Bernstein polynomials of degree p at xi in [0,1] and their xi-derivative
// (matrix_free/src/BernsteinBasis.cpp:3-146).
void bernstein(int p, double xi, double *B, double *dB);

// Open uniform knot vector on [0, L] (matrix_free/preprocess.cpp:50-56).
std::vector<double> open_knots(int p, int ne, double L);

// Bezier extraction operators, one row-major (p+1)^2 block per element
// (Borden et al. 2011, Algorithm 1; matrix_free/src/NURBSExtractionGenerator.cpp:4-82).
std::vector<double> extraction(int p, const std::vector<double> &knots);

// Greville abscissae of degree p (matrix_free/src/AbscissaeGenerator.cpp:27-41).
std::vector<double> greville(int p, const std::vector<double> &knots);

// 1-D basis tables of one parametric direction: for every element e and
// quadrature point k, value[e][k][i] and d/dxi[e][k][i] (reference element
// coordinate xi in [0,1], no division by the element size) of the p+1
// functions supported on e. With 1-D weights wt (NULL = polynomial) the
// functions are the rational R_i = wt_i N_i / sum_j wt_j N_j.
struct Tables1D {
    int p = 0, ne = 0;
    std::vector<double> val, der;  // [ne][p+1][p+1]
};
Tables1D tables_1d(int p, int ne, const double *C /* ne*(p+1)^2 */, const double *wt /* ne+p or null */);

// Exact quarter annulus r in [r_in, r_out], theta in [0, pi/2] as a NURBS
// patch: radial direction (x-fastest index) linear, angular direction the
// rational quadratic arc (weights 1, sqrt(2)/2, 1), both degree-elevated to p
// and refined by uniform knot insertion to ner x net elements. Outputs the
// control points (x, y interleaved), one weight per control point, and the
// (open uniform) knot vectors' extraction operators.
void quarter_annulus(int p, int ner, int net, double r_in, double r_out, std::vector<double> &CP,
                     std::vector<double> &W, std::vector<double> &C1, std::vector<double> &C2);

// Host description of a validated patch.
struct Patch {
    int p = 0, q = 0, nex = 0, ney = 0, m = 0, n = 0;
    std::vector<double> CP;       // 2*m*n
    std::vector<double> C1, C2;   // extraction operators
    std::vector<double> w1, w2;   // 1-D weight factors (empty: polynomial)
    std::vector<double> kappa;    // per quadrature point (empty: 1)
};

// Validates the reference-layout description and fills a Patch. Returns an
// error message (empty on success).
struct MeshDescView {
    int p, q, nex, ney;
    const double *CP, *weights, *C1, *C2;
    const int *IEN, *ID, *Dir;
    int nDir;
    const double *kappa;
};
std::string build_patch(const MeshDescView &d, Patch &out);

}  // namespace iga
