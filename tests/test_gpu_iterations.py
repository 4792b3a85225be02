"""Solver iteration counts against the reference's own records.

The reference records p = 3 FEM-preconditioned matrix-free solves on one rank
(matrix_free/data/fempc_mf.txt:1-36): 35, 33 and 28 outer iterations at
32^2, 64^2 and 128^2 elements, with its load x(1-x)y(1-y)
(matrix_free/include/LocalAssemblyMF.hpp:52-55), the outer KSP from options
(PETSc's default: GMRES restarted every 30 iterations, left-preconditioned;
no run script for this driver is recorded) preconditioned by an inner
Jacobi-CG on the bilinear FEM matrix, and rtol = abstol = 1e-10 on the
PRECONDITIONED residual norm (matrix_free/iteration_number_fempc_mf.cpp:
199-224). PETSc stops when ||M^-1 r|| <= max(rtol ||M^-1 b||, abstol): at
these sizes abstol dominates, so the solve ends at a preconditioned residual
reduction of about 1e-9, not 1e-10.

Two checks:
  * a restarted GMRES(30) restated here with exactly that stopping rule, over
    this library's MatMult and its inner-CG preconditioner (iga_pc_apply),
    must take the recorded counts within GMRES_TOL iterations. The operator,
    load, preconditioner and stopping rule are the reference's; what differs
    is rounding (PETSc's classical Gram-Schmidt, its inner CG's own stopping
    rule on the preconditioned residual), which moves a count by a few
    iterations near the abstol threshold;
  * the device solver (flexible PCG with the same preconditioner) run to the
    relative true residual that GMRES reached when it stopped must take the
    GMRES count within PCG_TOL (CG minimises the energy norm where GMRES
    minimises the preconditioned residual: for this SPD pair the counts stay
    close at equal accuracy). The device solver's own default stop, a
    relative TRUE residual of 1e-10, is a stricter target than the
    reference's and takes about twice the iterations (printed).
"""
import numpy as np
import pytest

from iga_testlib import load_binding

pytestmark = pytest.mark.gpu

REFERENCE_COUNTS = {32: 35, 64: 33, 128: 28}   # matrix_free/data/fempc_mf.txt:12,24,36
GMRES_TOL = 4
PCG_TOL = 4


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def gmres_left(torch, A, M, b, rtol=1e-10, abstol=1e-10, restart=30, maxit=2000):
    """Left-preconditioned restarted GMRES with PETSc's default test: stop
    when the preconditioned residual norm (the Arnoldi least-squares
    estimate) is <= max(rtol * ||M^-1 b||, abstol), x0 = 0. Returns the
    iterations taken and the solution."""
    x = torch.zeros_like(b)
    z = M(b)
    target = max(rtol * float(z.norm()), abstol)
    its = 0
    while its < maxit:
        beta = float(z.norm())
        if beta <= target:
            return its, x
        V = [z / beta]
        H = np.zeros((restart + 1, restart))
        cs, sn = np.zeros(restart), np.zeros(restart)
        g = np.zeros(restart + 1)
        g[0] = beta
        k = 0
        for j in range(restart):
            w = M(A(V[j]))
            for i in range(j + 1):   # modified Gram-Schmidt
                H[i, j] = float(torch.dot(w, V[i]))
                w = w - H[i, j] * V[i]
            H[j + 1, j] = float(w.norm())
            V.append(w / H[j + 1, j] if H[j + 1, j] > 0 else w)
            for i in range(j):   # earlier rotations on the new column
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            r = np.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = H[j, j] / r, H[j + 1, j] / r
            H[j, j], H[j + 1, j] = r, 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            its += 1
            k = j + 1
            if abs(g[j + 1]) <= target:
                break
        y = np.linalg.solve(np.triu(H[:k, :k]), g[:k])
        for i in range(k):
            x = x + float(y[i]) * V[i]
        if abs(g[k]) <= target:
            return its, x
        z = M(b - A(x))
    return its, x


@pytest.mark.parametrize("ne", sorted(REFERENCE_COUNTS))
def test_iteration_counts_match_reference_records(torch_cuda, ne):
    torch = torch_cuda
    ib = load_binding()
    plan = ib.Plan(ib.unit_square(3, ne), sign=ib.SIGN_SPD, bc=ib.BC_IDENTITY)
    b = torch.empty(plan.nfunc, dtype=torch.float64, device="cuda")
    plan.rhs(b, ib.F_REFERENCE)

    def A(v):
        y = torch.empty_like(v)
        plan.apply(v, y)
        return y

    def M(v):
        z = torch.empty_like(v)
        plan.pc_apply(v, z, pc=ib.PC_FEM_CG, precision=ib.FP64, pc_rtol=1e-10, pc_max_it=10000)
        return z

    its_gmres, xg = gmres_left(torch, A, M, b)
    rel_gmres = float((b - A(xg)).norm() / b.norm())
    x = torch.zeros_like(b)
    st = plan.solve(b, x, pc=ib.PC_FEM_CG, rtol=rel_gmres)
    x2 = torch.zeros_like(b)
    st2 = plan.solve(b, x2, pc=ib.PC_FEM_CG, rtol=1e-10)
    ref = REFERENCE_COUNTS[ne]
    print(f"p=3 {ne}^2: reference {ref}, GMRES(30) restatement {its_gmres} (true residual {rel_gmres:.2e}), "
          f"device PCG to that residual {st.iterations}, device PCG to 1e-10 {st2.iterations}")
    assert abs(its_gmres - ref) <= GMRES_TOL
    assert abs(st.iterations - its_gmres) <= PCG_TOL
    assert st.relres <= rel_gmres and st2.relres <= 1e-10
    plan.close()
