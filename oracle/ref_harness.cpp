// Test-infrastructure harness around the reference's own PETSc-free element code.
//
// This file is ORACLE code: it is compiled together with the unmodified
// reference sources (matrix_free/src/*.cpp, read in place by oracle/Makefile)
// into oracle/_ref/libigaref.so. Only tests/, tests/golden/make_golden.py,
// __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm load it.
// The shipped CUDA path never links or calls it.
//
// The reference's global layer (GlobalAssemblyMF / GlobalAssembly) needs PETSc,
// which is absent, so the loops below restate only that PETSc glue with plain
// arrays, line for line in the order the reference runs it:
//   * MatMulMF (MF and MFSF overloads): matrix_free/src/GlobalAssemblyMF.cpp:141-281
//     element loop jj (y) outer, ii (x) inner; x gathered through IEN; y
//     scattered through ID with negative indices ignored (VEC_IGNORE_NEGATIVE_INDICES,
//     matrix_free/iteration_number_fempc_mf.cpp:67); then y[Dir] = 0.
//   * AssemLoad: matrix_free/src/GlobalAssemblyMF.cpp:26-80, F[Dir] = 0 (:283-290).
//   * AssemStiffnessLoad + DirichletBC: matrix_free/src/GlobalAssembly.cpp:103-217;
//     PETSc drops rows/columns with negative indices, Dir diagonal gets +1.
//   * Mesh generation: matrix_free/preprocess.cpp:37-87 and
//     matrix_free/preprocess_fem.cpp:38-73, serial partition
//     (matrix_free/src/Partition.cpp:73-109: with one part old_to_new is the
//     identity, ID = index for free DOFs and -1 on the boundary, Dir = the
//     boundary indices in ascending order).
//   * Control points: ControlPointGenerator needs Eigen (absent); its output
//     for the linear parameterisation equals the degree-p Greville abscissae,
//     which are computed here with the reference's AbscissaeGenerator.
//   * Partitioned meshes: matrix_free/preprocess.cpp:16-87 drives the
//     reference's own Partition + FileManager (compiled unmodified) to write
//     info.txt and <base>_<rank>.txt; the partitioned MatMulMF restates the
//     glue of matrix_free/src/GlobalAssemblyMF.cpp:141-210 with the PETSc
//     ghosted vector replaced by arrays: local form = owned entries (the
//     part's contiguous range of the partition numbering) then the ghosts
//     (ghostID), y scattered to global indices ID >= 0, then y[Dir] = 0.
#include <cstring>
#include <string>
#include <cmath>
#include <thread>
#include <vector>

#include "AbscissaeGenerator.hpp"
#include "BSplineBasis.hpp"
#include "Element.hpp"
#include "ElementFEM.hpp"
#include "ElementMF.hpp"
#include "ElementMFSF.hpp"
#include "FileManager.hpp"
#include "IDGenerator.hpp"
#include "IENGenerator.hpp"
#include "LocalAssembly.hpp"
#include "LocalAssemblyMF.hpp"
#include "LocalAssemblyMFSF.hpp"
#include "NURBSExtractionGenerator.hpp"
#include "Partition.hpp"
#include "QuadraturePoint.hpp"

namespace {

std::vector<double> open_knots(int p, int ne, double L)
{
    // matrix_free/preprocess.cpp:50-56
    std::vector<double> S;
    const double h = L / ne;
    for (int i = 0; i < p + 1; ++i) S.push_back(0.0);
    for (int i = 1; i < ne; ++i) S.push_back(i * h);
    for (int i = 0; i < p + 1; ++i) S.push_back(L);
    return S;
}

struct Mesh {
    int p, q, nex, ney, nfx, nfy;
    const double *CP;
    const int *IEN, *ID, *Dir;
    int nDir;
    const double *C1, *C2, *h1, *h2;
};

Mesh make_mesh(int p, int q, int nex, int ney, const double *CP, const int *IEN,
               const int *ID, const int *Dir, int nDir, const double *C1,
               const double *C2, const double *h1, const double *h2)
{
    Mesh m{p, q, nex, ney, nex + p, ney + q, CP, IEN, ID, Dir, nDir, C1, C2, h1, h2};
    return m;
}

// One element of MatMulMF's loop body (GlobalAssemblyMF.cpp:168-193) for an
// element-row block [jy0, jy1), accumulating into y (private per thread).
template <class LA, class EL>
void mult_block(const Mesh &m, LA *la, EL *el, const double *x, double *y, int jy0, int jy1)
{
    const int nloc = (m.p + 1) * (m.q + 1);
    const int pp = m.p + 1, qq = m.q + 1;
    std::vector<double> eCP(2 * nloc), e1(pp * pp), e2(qq * qq);
    for (int jj = jy0; jj < jy1; ++jj) {
        for (int ii = 0; ii < m.nex; ++ii) {
            const int e = jj * m.nex + ii;
            for (int j = 0; j < nloc; ++j) {
                const int A = m.IEN[e * nloc + j];
                eCP[2 * j] = m.CP[2 * A];
                eCP[2 * j + 1] = m.CP[2 * A + 1];
                la->Floc_in[j] = x[A];
            }
            std::copy(m.C1 + ii * pp * pp, m.C1 + (ii + 1) * pp * pp, e1.begin());
            std::copy(m.C2 + jj * qq * qq, m.C2 + (jj + 1) * qq * qq, e2.begin());
            el->SetElement(e1, e2, m.h1[ii], m.h2[jj]);
            la->LocalMatMulMF(el, eCP);
            for (int j = 0; j < nloc; ++j) {
                const int r = m.ID[m.IEN[e * nloc + j]];
                if (r >= 0) y[r] += la->Floc_out[j];
            }
        }
    }
}

template <class LA, class EL>
void mult_threads(const Mesh &m, const double *x, double *y, int nthreads)
{
    const int nf = m.nfx * m.nfy;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > m.ney) nthreads = m.ney;
    std::vector<std::vector<double>> part(nthreads, std::vector<double>(nf, 0.0));
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) {
        const int jy0 = (int)((long long)m.ney * t / nthreads);
        const int jy1 = (int)((long long)m.ney * (t + 1) / nthreads);
        pool.emplace_back([&, t, jy0, jy1]() {
            LA la(m.p, m.q);
            EL el(m.p, m.q);
            mult_block(m, &la, &el, x, part[t].data(), jy0, jy1);
        });
    }
    for (auto &th : pool) th.join();
    // Fixed-order sum of the per-thread partial vectors (thread 0 first), the
    // host-core analogue of the reference's per-rank VecAssembly.
    for (int i = 0; i < nf; ++i) {
        double s = 0.0;
        for (int t = 0; t < nthreads; ++t) s += part[t][i];
        y[i] = s;
    }
    for (int d = 0; d < m.nDir; ++d) y[m.Dir[d]] = 0.0;  // GlobalAssemblyMF.cpp:201-205
}

}  // namespace

extern "C" {

// Gauss points/weights on [0,1] and Bernstein B, dB at them
// (QuadraturePoint.cpp:3-58, BernsteinBasis.hpp:13-25).
int ref_tables(int p, double *qp, double *qw, double *B, double *dB)
{
    QuadraturePoint quad(p + 1, 0, 1);
    BernsteinBasis bern(p);
    bern.GenerateBernsteinBasis(&quad);
    const auto x = quad.GetQuadraturePoint();
    const auto w = quad.GetWeight();
    for (int i = 0; i < p + 1; ++i) { qp[i] = x[i]; qw[i] = w[i]; }
    const auto &b = bern.GetBernsteinBasis();
    const auto &db = bern.GetBernsteinBasisDerivative();
    std::memcpy(B, b.data(), sizeof(double) * b.size());
    std::memcpy(dB, db.data(), sizeof(double) * db.size());
    return 0;
}

// Bezier extraction operators for an arbitrary knot vector (NURBSExtractionGenerator.cpp:4-82).
int ref_extraction(int p, const double *knots, int nknots, double *C)
{
    std::vector<double> S(knots, knots + nknots);
    BSplineBasis b(p, S);
    NURBSExtractionGenerator g;
    const auto c = g.GenerateExtraction1D(&b);
    std::memcpy(C, c.data(), sizeof(double) * c.size());
    return (int)c.size();
}

// Greville abscissae of degree p (AbscissaeGenerator.cpp:27-41).
int ref_greville(int p, const double *knots, int nknots, double *out)
{
    std::vector<double> S(knots, knots + nknots);
    AbscissaeGenerator a;
    const auto g = a.GrevilleAbscissae(S, p);
    std::memcpy(out, g.data(), sizeof(double) * g.size());
    return (int)g.size();
}

// IGA mesh of matrix_free/preprocess.cpp with the serial partition.
int ref_mesh(int p, int q, int nex, int ney, double Lx, double Ly, double *CP, int *IEN,
             int *ID, int *Dir, int *nDir, double *C1, double *C2, double *h1, double *h2)
{
    const std::vector<double> S = open_knots(p, nex, Lx), T = open_knots(q, ney, Ly);
    BSplineBasis b1(p, S), b2(q, T);
    IENGenerator ig;
    IDGenerator idg;
    NURBSExtractionGenerator ng;
    AbscissaeGenerator ag;
    const auto ien = ig.GenerateIEN2D(&b1, &b2);
    const auto id = idg.GenerateID2D(&b1, &b2);
    const auto g1 = ag.GrevilleAbscissae(S, p), g2 = ag.GrevilleAbscissae(T, q);
    const auto c1 = ng.GenerateExtraction1D(&b1), c2 = ng.GenerateExtraction1D(&b2);
    const int m = nex + p, n = ney + q;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            CP[2 * (j * m + i)] = g1[i];
            CP[2 * (j * m + i) + 1] = g2[j];
        }
    std::memcpy(IEN, ien.data(), sizeof(int) * ien.size());
    int nd = 0;
    for (int A = 0; A < m * n; ++A) {
        ID[A] = (id[A] == -1) ? -1 : A;
        if (id[A] == -1) Dir[nd++] = A;
    }
    *nDir = nd;
    std::memcpy(C1, c1.data(), sizeof(double) * c1.size());
    std::memcpy(C2, c2.data(), sizeof(double) * c2.size());
    for (int i = 0; i < nex; ++i) h1[i] = Lx / nex;
    for (int j = 0; j < ney; ++j) h2[j] = Ly / ney;
    return 0;
}

// y = A_ref x through LocalAssemblyMF/ElementMF (the mult_mf path).
int ref_apply_mf(int p, int q, int nex, int ney, const double *CP, const int *IEN, const int *ID,
                 const int *Dir, int nDir, const double *C1, const double *C2, const double *h1,
                 const double *h2, const double *x, double *y, int nthreads)
{
    const Mesh m = make_mesh(p, q, nex, ney, CP, IEN, ID, Dir, nDir, C1, C2, h1, h2);
    mult_threads<LocalAssemblyMF, ElementMF>(m, x, y, nthreads);
    return 0;
}

// y = A_ref x through LocalAssemblyMFSF/ElementMFSF (the mult_sf path; the
// reference's formula holds for p == q on axis-aligned affine patches).
int ref_apply_sf(int p, int q, int nex, int ney, const double *CP, const int *IEN, const int *ID,
                 const int *Dir, int nDir, const double *C1, const double *C2, const double *h1,
                 const double *h2, const double *x, double *y, int nthreads)
{
    const Mesh m = make_mesh(p, q, nex, ney, CP, IEN, ID, Dir, nDir, C1, C2, h1, h2);
    mult_threads<LocalAssemblyMFSF, ElementMFSF>(m, x, y, nthreads);
    return 0;
}

// F = int R f (f = x(1-x)y(1-y), hard-coded in the reference), F[Dir] = 0.
int ref_rhs(int p, int q, int nex, int ney, const double *CP, const int *IEN, const int *ID,
            const int *Dir, int nDir, const double *C1, const double *C2, const double *h1,
            const double *h2, double *F)
{
    const Mesh m = make_mesh(p, q, nex, ney, CP, IEN, ID, Dir, nDir, C1, C2, h1, h2);
    const int nloc = (p + 1) * (q + 1), pp = p + 1, qq = q + 1;
    LocalAssemblyMF la(p, q);
    ElementMF el(p, q);
    std::vector<double> eCP(2 * nloc), e1(pp * pp), e2(qq * qq);
    std::fill(F, F + m.nfx * m.nfy, 0.0);
    for (int jj = 0; jj < ney; ++jj)
        for (int ii = 0; ii < nex; ++ii) {
            const int e = jj * nex + ii;
            for (int j = 0; j < nloc; ++j) {
                const int A = IEN[e * nloc + j];
                eCP[2 * j] = CP[2 * A];
                eCP[2 * j + 1] = CP[2 * A + 1];
            }
            std::copy(C1 + ii * pp * pp, C1 + (ii + 1) * pp * pp, e1.begin());
            std::copy(C2 + jj * qq * qq, C2 + (jj + 1) * qq * qq, e2.begin());
            el.SetElement(e1, e2, h1[ii], h2[jj]);
            la.AssemLocalLoad(&el, eCP);
            for (int j = 0; j < nloc; ++j) {
                const int r = ID[IEN[e * nloc + j]];
                if (r >= 0) F[r] += la.Floc[j];
            }
        }
    for (int d = 0; d < nDir; ++d) F[Dir[d]] = 0.0;
    return 0;
}

// y = K_ref x for the ASSEMBLED IGA stiffness (Element + LocalAssembly), with
// the PETSc rules: entries whose row or column index is negative are dropped
// and each Dirichlet diagonal gets +1 (GlobalAssembly.cpp:204-217).
int ref_assembled_matvec(int p, int q, int nex, int ney, const double *CP, const int *IEN,
                         const int *ID, const int *Dir, int nDir, const double *C1,
                         const double *C2, const double *h1, const double *h2, const double *x,
                         double *y)
{
    const int nloc = (p + 1) * (q + 1), pp = p + 1, qq = q + 1;
    LocalAssembly la(p, q);
    Element el(p, q);
    std::vector<double> eCP(2 * nloc), e1(pp * pp), e2(qq * qq);
    std::vector<int> eID(nloc);
    std::fill(y, y + (nex + p) * (ney + q), 0.0);
    for (int jj = 0; jj < ney; ++jj)
        for (int ii = 0; ii < nex; ++ii) {
            const int e = jj * nex + ii;
            for (int j = 0; j < nloc; ++j) {
                const int A = IEN[e * nloc + j];
                eID[j] = ID[A];
                eCP[2 * j] = CP[2 * A];
                eCP[2 * j + 1] = CP[2 * A + 1];
            }
            std::copy(C1 + ii * pp * pp, C1 + (ii + 1) * pp * pp, e1.begin());
            std::copy(C2 + jj * qq * qq, C2 + (jj + 1) * qq * qq, e2.begin());
            el.SetElement(e1, e2, h1[ii], h2[jj]);
            la.AssemLocalStiffnessLoad(&el, eCP);
            for (int k = 0; k < nloc; ++k) {
                if (eID[k] < 0) continue;
                double s = 0.0;
                for (int l = 0; l < nloc; ++l)
                    if (eID[l] >= 0) s += la.Kloc[k * nloc + l] * x[eID[l]];
                y[eID[k]] += s;
            }
        }
    for (int d = 0; d < nDir; ++d) y[Dir[d]] += x[Dir[d]];
    return 0;
}

// Bilinear FEM preconditioner grid of matrix_free/preprocess_fem.cpp:38-73
// (nodes = degree p-2 Greville abscissae of the shortened knot vector; the
// reference divides by p-2, so p = 2 yields NaN nodes, reproduced here).
int ref_fem_mesh(int p, int q, int nex, int ney, double Lx, double Ly, double *CP, int *IEN,
                 int *ID, int *Dir, int *nDir)
{
    const double hx = Lx / (nex + 2), hy = Ly / (ney + 2);
    const int nfx = p + nex, nfy = q + ney;
    std::vector<double> S, T;
    for (int i = 0; i < p - 1; ++i) S.push_back(0.0);
    for (int i = 1; i < nex + 2; ++i) S.push_back(i * hx);
    for (int i = 0; i < p - 1; ++i) S.push_back(Lx);
    for (int i = 0; i < q - 1; ++i) T.push_back(0.0);
    for (int i = 1; i < ney + 2; ++i) T.push_back(i * hy);
    for (int i = 0; i < q - 1; ++i) T.push_back(Ly);
    AbscissaeGenerator ag;
    const auto cp = ag.GenerateAbscissae2D(S, T, p - 2, q - 2);
    std::memcpy(CP, cp.data(), sizeof(double) * cp.size());
    IENGenerator ig;
    IDGenerator idg;
    const auto ien = ig.GenerateIEN2D(nfx - 1, nfy - 1);
    const auto id = idg.GenerateID2D(nfx, nfy);
    std::memcpy(IEN, ien.data(), sizeof(int) * ien.size());
    int nd = 0;
    for (int A = 0; A < nfx * nfy; ++A) {
        ID[A] = (id[A] == -1) ? -1 : A;
        if (id[A] == -1) Dir[nd++] = A;
    }
    *nDir = nd;
    return (int)(cp.size() / 2);
}

// y = K_fem x (ElementFEM + LocalAssembly(1,1), 2x2 Gauss), same PETSc rules.
int ref_fem_matvec(int nfx, int nfy, const double *CP, const int *IEN, const int *ID,
                   const int *Dir, int nDir, const double *x, double *y)
{
    ElementFEM el(1, 1);
    LocalAssembly la(1, 1);
    std::vector<double> eCP(8);
    std::vector<int> eID(4);
    std::fill(y, y + nfx * nfy, 0.0);
    const int nex = nfx - 1, ney = nfy - 1;
    for (int jj = 0; jj < ney; ++jj)
        for (int ii = 0; ii < nex; ++ii) {
            const int e = jj * nex + ii;
            for (int j = 0; j < 4; ++j) {
                const int A = IEN[e * 4 + j];
                eID[j] = ID[A];
                eCP[2 * j] = CP[2 * A];
                eCP[2 * j + 1] = CP[2 * A + 1];
            }
            la.AssemLocalStiffnessLoad(&el, eCP);
            for (int k = 0; k < 4; ++k) {
                if (eID[k] < 0) continue;
                double s = 0.0;
                for (int l = 0; l < 4; ++l)
                    if (eID[l] >= 0) s += la.Kloc[k * 4 + l] * x[eID[l]];
                y[eID[k]] += s;
            }
        }
    for (int d = 0; d < nDir; ++d) y[Dir[d]] += x[Dir[d]];
    return 0;
}

// info.txt and the partition files of matrix_free/preprocess.cpp, written by
// the reference's Partition / FileManager into dir (files dir/<base>_<rank>.txt).
int ref_write_partition(int p, int q, int nex, int ney, double Lx, double Ly, int part_num_1d, const char *dir,
                        const char *base)
{
    const std::vector<double> S = open_knots(p, nex, Lx), T = open_knots(q, ney, Ly);
    BSplineBasis b1(p, S), b2(q, T);
    IENGenerator ig;
    IDGenerator idg;
    NURBSExtractionGenerator ng;
    AbscissaeGenerator ag;
    const auto ien = ig.GenerateIEN2D(&b1, &b2);
    const auto id = idg.GenerateID2D(&b1, &b2);
    const auto g1 = ag.GrevilleAbscissae(S, p), g2 = ag.GrevilleAbscissae(T, q);
    const auto c1 = ng.GenerateExtraction1D(&b1), c2 = ng.GenerateExtraction1D(&b2);
    const int m = nex + p, n = ney + q;
    std::vector<double> CP(2 * m * n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            CP[2 * (j * m + i)] = g1[i];
            CP[2 * (j * m + i) + 1] = g2[j];
        }
    const std::string d(dir), bn(base);
    FileManager fm;
    fm.WritePreprocessInfo(d + "/info.txt", p, q, Lx, Ly, nex, ney, part_num_1d, 2, bn);
    Partition part(part_num_1d, part_num_1d, 2, d + "/" + bn);
    part.GeneratePartition(&b1, &b2, CP, ien, id, c1, c2);
    return 0;
}

// y = A_ref x over all parts of a partitioned mesh (x, y in the partition
// numbering, length nfunc): per part, the MatMulMF element loop on its local
// form, scattering to the global rows ID >= 0; then every part's Dir rows = 0.
int ref_apply_partitioned(const char *dir, const char *base, int p, int q, int nparts, const double *x, double *y,
                          int nfunc)
{
    std::fill(y, y + nfunc, 0.0);
    FileManager fm;
    const int nloc = (p + 1) * (q + 1), pp = p + 1, qq = q + 1;
    LocalAssemblyMF la(p, q);
    ElementMF el(p, q);
    std::vector<std::vector<int>> dirs;
    int offset = 0;
    for (int r = 0; r < nparts; ++r) {
        int nlf = 0, nlx = 0, nly = 0;
        std::vector<double> h1, h2, CP, C1, C2;
        std::vector<int> ID, ghost, Dir, IEN;
        fm.ReadPartition(fm.GetPartitionFilename(std::string(dir) + "/" + base, r), nlf, nlx, nly, h1, h2, CP, ID,
                         ghost, Dir, IEN, C1, C2);
        std::vector<double> xl(nlf + ghost.size());
        for (int k = 0; k < nlf; ++k) xl[k] = x[offset + k];
        for (size_t g = 0; g < ghost.size(); ++g) xl[nlf + g] = x[ghost[g]];
        std::vector<double> eCP(2 * nloc), e1(pp * pp), e2(qq * qq);
        for (int jj = 0; jj < nly; ++jj)
            for (int ii = 0; ii < nlx; ++ii) {
                const int e = jj * nlx + ii;
                for (int j = 0; j < nloc; ++j) {
                    const int A = IEN[e * nloc + j];
                    eCP[2 * j] = CP[2 * A];
                    eCP[2 * j + 1] = CP[2 * A + 1];
                    la.Floc_in[j] = xl[A];
                }
                std::copy(C1.begin() + ii * pp * pp, C1.begin() + (ii + 1) * pp * pp, e1.begin());
                std::copy(C2.begin() + jj * qq * qq, C2.begin() + (jj + 1) * qq * qq, e2.begin());
                el.SetElement(e1, e2, h1[ii], h2[jj]);
                la.LocalMatMulMF(&el, eCP);
                for (int j = 0; j < nloc; ++j) {
                    const int row = ID[IEN[e * nloc + j]];
                    if (row >= 0) y[row] += la.Floc_out[j];
                }
            }
        dirs.push_back(Dir);
        offset += nlf;
    }
    for (const auto &D : dirs)
        for (int d : D) y[d] = 0.0;
    return offset;
}

}  // extern "C"
