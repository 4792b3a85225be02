"""Device PCG with the bilinear-FEM preconditioner (include/iga_solve.h).

The FEM matrix is checked against the reference's own FEM assembly (golden
vectors from ElementFEM + LocalAssembly); the solve against the oracle's CPU
PCG (same preconditioner, inner Jacobi-CG to 1e-10). Solutions of two solvers
that both reach a relative residual of 1e-10 agree to about cond(K) * 1e-10,
so they are compared at 1e-7 relative on these small meshes.
"""
import numpy as np
import pytest

from iga_testlib import boundary_mask, distorted, load_binding, splitmix_normal, splitmix_uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def ib():
    return load_binding()


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def csr_matvec(rp, col, val, x):
    y = np.zeros(len(rp) - 1)
    for i in range(len(rp) - 1):
        y[i] = np.dot(val[rp[i]:rp[i + 1]], x[col[rp[i]:rp[i + 1]]])
    return y


@pytest.mark.parametrize("p,ne", [(3, 16), (4, 10)])
def test_fem_csr_matches_reference_assembly(torch_cuda, ib, orc, gold, p, ne):
    plan = ib.Plan(ib.unit_square(p, ne))
    gx, gy = plan.fem_nodes()
    assert np.abs(gx - gold[f"fem_p{p}_nodes"]).max() < 1e-14
    rp, col, val = plan.fem_csr(sign=-1)
    assert np.all(np.diff(rp) >= 1)
    for i in range(len(rp) - 1):   # sorted, unique columns per row
        assert np.all(np.diff(col[rp[i]:rp[i + 1]]) > 0)
    y = csr_matvec(rp, col, val, gold[f"fem_p{p}_x"])
    assert rel(y, gold[f"fem_p{p}_y"]) < 1e-13


def test_fem_nodes_p2_replacement(torch_cuda, ib, orc):
    plan = ib.Plan(ib.unit_square(2, 6))
    gx, _ = plan.fem_nodes()
    assert np.abs(gx - orc.fem_nodes(2, 6)).max() < 1e-14


@pytest.mark.parametrize("p", [2, 3, 4])
def test_matrix_free_fem_equals_csr(torch_cuda, ib, orc, p):
    torch = torch_cuda
    plan = ib.Plan(ib.unit_square(p, 37, 21), precision=ib.MIXED)
    rp, col, val = plan.fem_csr(sign=1)
    x = splitmix_uniform(3, -1.0, 1.0, plan.nfunc)
    ref = csr_matvec(rp, col, val, x)
    gx, gy = plan.fem_nodes()
    assert rel(ref, orc.fem_matvec(gx, gy, x, 1.0)) < 1e-13
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    plan.fem_apply(xd, yd, precision=ib.FP64)
    y32 = torch.empty_like(xd, dtype=torch.float32)
    plan.fem_apply(xd.float(), y32, precision=ib.FP32)
    torch.cuda.synchronize()
    assert rel(yd.cpu().numpy(), ref) < 1e-13
    assert rel(y32.double().cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("p,ne", [(2, 16), (3, 12), (4, 10)])
def test_pcg_matches_oracle_pcg(torch_cuda, ib, orc, p, ne):
    torch = torch_cuda
    mesh = ib.unit_square(p, ne)
    plan = ib.Plan(mesh)
    b = orc.rhs(mesh, 1)
    x_ref, it_ref, rr_ref = orc.pcg(mesh, b, rtol=1e-10)
    assert it_ref > 0
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros_like(bd)
    st = plan.solve(bd, xd, pc=ib.PC_FEM_CG, rtol=1e-10)
    x = xd.cpu().numpy()
    assert st.status == 0 and st.relres <= 1e-10
    assert abs(st.iterations - it_ref) <= 2
    assert rel(x, x_ref) < 1e-7
    # the solution satisfies the SPD system on the CPU oracle too
    r = b - orc.apply_mf(mesh, x, sign=1.0, bc=1)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 2e-10


def test_pcg_distorted_geometry_and_no_pc(torch_cuda, ib, orc):
    torch = torch_cuda
    mesh = distorted(ib.unit_square(3, 20, 14))
    plan = ib.Plan(mesh)
    b = orc.rhs(mesh, 1)
    bd = torch.from_numpy(b).cuda()
    for pc in (ib.PC_NONE, ib.PC_FEM_CG):
        xd = torch.zeros_like(bd)
        st = plan.solve(bd, xd, pc=pc, rtol=1e-10)
        assert st.status == 0 and st.relres <= 1e-10
        r = b - orc.apply_mf(mesh, xd.cpu().numpy(), sign=1.0, bc=1)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 2e-10


@pytest.mark.parametrize("pc", [0, 1])
def test_mixed_precision_refinement(torch_cuda, ib, orc, pc):
    torch = torch_cuda
    mesh = ib.unit_square(3, 40)
    plan = ib.Plan(mesh, precision=ib.MIXED)
    b = splitmix_normal(2, plan.nfunc)
    b[boundary_mask(43, 43)] = 0.0
    bd = torch.from_numpy(b).cuda()
    x64 = torch.zeros_like(bd)
    s64 = plan.solve(bd, x64, pc=pc, rtol=1e-10)
    x32 = torch.zeros_like(bd)
    smx = plan.solve(bd, x32, pc=pc, rtol=1e-10, precision=ib.MIXED, pc_rtol=1e-4)
    assert s64.status == 0 and smx.status == 0
    assert smx.relres <= 1e-10 and smx.sweeps >= 2
    assert rel(x32.cpu().numpy(), x64.cpu().numpy()) < 1e-7
    r = b - orc.apply_mf(mesh, x32.cpu().numpy(), sign=1.0, bc=1)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 2e-10


@pytest.mark.parametrize("pc,kappa", [(1, False), (2, False), (2, True)])
def test_fp64_pcg_with_fp32_preconditioner(torch_cuda, ib, orc, pc, kappa):
    """IGA_MIXED_PC: FP64 flexible PCG whose preconditioner runs in FP32 reaches the
    FP64 tolerance on an FP64-only plan and agrees with the FP64 solve."""
    torch = torch_cuda
    mesh = distorted(ib.unit_square(3, 40, 33))
    plan = ib.Plan(mesh)
    if kappa:
        nq = 40 * 33 * 16
        k = 1.0 + 0.5 * splitmix_uniform(5, -1, 1, nq)
        plan.set_kappa(torch.from_numpy(k).cuda())
    b = splitmix_normal(2, plan.nfunc)
    b[boundary_mask(43, 36)] = 0.0
    bd = torch.from_numpy(b).cuda()
    x64, xpc = torch.zeros_like(bd), torch.zeros_like(bd)
    s64 = plan.solve(bd, x64, pc=pc, rtol=1e-10, pc_rtol=1e-6)
    spc = plan.solve(bd, xpc, pc=pc, rtol=1e-10, pc_rtol=1e-6, precision=ib.MIXED_PC)
    assert s64.status == 0 and spc.status == 0 and spc.relres <= 1e-10 and spc.sweeps == 0
    assert spc.iterations <= 2 * s64.iterations + 5
    assert rel(xpc.cpu().numpy(), x64.cpu().numpy()) < 1e-7
    if not kappa:
        r = b - orc.apply_mf(mesh, xpc.cpu().numpy(), sign=1.0, bc=1)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 2e-10
    # an unknown solve precision is an argument error
    with pytest.raises(ib.IgaError):
        plan.solve(bd, xpc, precision=7)


def test_solver_failure_modes(torch_cuda, ib):
    torch = torch_cuda
    plan = ib.Plan(ib.unit_square(2, 16))
    n = plan.nfunc
    b = torch.from_numpy(splitmix_uniform(4, -1, 1, n)).cuda()
    b[torch.from_numpy(boundary_mask(18, 18)).cuda()] = 0
    x = torch.zeros_like(b)
    st = plan.solve(b, x, check=False, max_it=1, pc=ib.PC_NONE)
    assert st.status == 5          # IGA_ERR_NOT_CONVERGED
    bad = b.clone()
    bad[n // 2] = float("nan")
    st = plan.solve(bad, x, check=False)
    assert st.status == 7          # IGA_ERR_NONFINITE
    zero = torch.zeros_like(b)
    st = plan.solve(zero, x, check=False)
    assert st.status == 0 and float(x.abs().max()) == 0.0
    # the solver reuses its state: a second solve gives the same answer bitwise
    x1, x2 = torch.zeros_like(b), torch.zeros_like(b)
    plan.solve(b, x1)
    plan.solve(b, x2)
    torch.cuda.synchronize()
    assert torch.equal(x1, x2)


@pytest.mark.parametrize("pc,prec,tol", [(2, 0, 1e-10), (2, 1, 2e-2), (1, 0, 1e-9), (1, 1, 1e-3)])
def test_preconditioner_inverts_fem_matrix(torch_cuda, ib, pc, prec, tol):
    """K_fem (M^-1 r) = r for the exact inverse and the inner CG (FP64 and FP32/TF32)."""
    torch = torch_cuda
    plan = ib.Plan(distorted(ib.unit_square(3, 45, 30)), precision=ib.MIXED)
    dt = torch.float64 if prec == 0 else torch.float32
    r = torch.from_numpy(splitmix_uniform(8, -1, 1, plan.nfunc)).to(device="cuda", dtype=dt)
    r[torch.from_numpy(boundary_mask(48, 33)).cuda()] = 0
    z = torch.empty_like(r)
    plan.pc_apply(r, z, pc=pc, precision=prec, pc_rtol=1e-10 if prec == 0 else 1e-5)
    y = torch.empty_like(r)
    plan.fem_apply(z, y, precision=prec)
    torch.cuda.synchronize()
    assert float((y - r).norm() / r.norm()) < tol


@pytest.mark.parametrize("nex,ney", [(300, 260), (130, 517), (517, 130)])
def test_exact_pc_multi_tile_transforms(torch_cuda, ib, nex, ney):
    """The exact inverse's two transform GEMMs over many 128 x 128 output tiles
    with ragged edges (the library's own DMMA tiles in FP64, the TMA-fed
    tcgen05 TF32 tiles in FP32): FP64 K_fem z = r to 1e-10; the FP32 z close
    to the FP64 one (TF32 operands: about 1e-3 relative)."""
    torch = torch_cuda
    mesh = distorted(ib.unit_square(3, nex, ney))
    plan = ib.Plan(mesh, precision=ib.MIXED)
    m, n = nex + 3, ney + 3
    r = torch.from_numpy(splitmix_uniform(12, -1, 1, plan.nfunc)).cuda()
    r[torch.from_numpy(boundary_mask(m, n)).cuda()] = 0
    z = torch.empty_like(r)
    plan.pc_apply(r, z, pc=ib.PC_FEM_EXACT, precision=ib.FP64)
    y = torch.empty_like(r)
    plan.fem_apply(z, y, precision=ib.FP64)
    r32 = r.float()
    z32 = torch.empty_like(r32)
    plan.pc_apply(r32, z32, pc=ib.PC_FEM_EXACT, precision=ib.FP32)
    torch.cuda.synchronize()
    assert plan.device_status() == 0
    assert float((y - r).norm() / r.norm()) < 1e-10
    assert float((z32.double() - z).norm() / z.norm()) < 1e-2
    plan.close()


@pytest.mark.parametrize("p,nex,ney", [(3, 300, 260), (3, 517, 130), (2, 16, 20), (4, 5, 7), (2, 1, 9)])
def test_exact_pc_parity_split_equals_full_transforms(torch_cuda, ib, p, nex, ney):
    """The exact inverse's x transforms split by parity (the FEM nodes are
    symmetric about the patch middle: even/odd folds of r, half-size
    eigenvector blocks, GEMM tiles over one block's k range, unfold into z)
    give the same z as the full transforms: FP64 to 1e-12, and the FP32 (TF32)
    forms both within 1e-2 of the FP64 z. Odd and even numbers of free x
    nodes (301, 518, 16, 7) and one free x node (no split possible)."""
    torch = torch_cuda
    mesh = distorted(ib.unit_square(p, nex, ney)) if nex > 1 else ib.unit_square(p, nex, ney)
    plan = ib.Plan(mesh, precision=ib.MIXED)
    m, n = nex + p, ney + p
    r = torch.from_numpy(splitmix_uniform(21, -1, 1, plan.nfunc)).cuda()
    r[torch.from_numpy(boundary_mask(m, n)).cuda()] = 0
    out = {}
    for split in (1, 0):
        plan.set_pc_split(split)
        z = torch.empty_like(r)
        plan.pc_apply(r, z, pc=ib.PC_FEM_EXACT, precision=ib.FP64)
        z32 = torch.empty_like(r.float())
        plan.pc_apply(r.float(), z32, pc=ib.PC_FEM_EXACT, precision=ib.FP32)
        torch.cuda.synchronize()
        assert plan.device_status() == 0
        out[split] = (z.clone(), z32.double())
    y = torch.empty_like(r)
    plan.fem_apply(out[1][0], y, precision=ib.FP64)
    torch.cuda.synchronize()
    assert float((y - r).norm() / r.norm()) < 1e-10
    z1, z0 = out[1][0], out[0][0]
    assert float((z1 - z0).norm() / z0.norm()) < 1e-12
    for s in (1, 0):
        assert float((out[s][1] - z0).norm() / z0.norm()) < 1e-2
    plan.close()


@pytest.mark.parametrize("ney", [9700, 19400, 95])
def test_exact_pc_long_columns(torch_cuda, ib, ney):
    """Tall meshes: the y tridiagonal solves of the exact inverse run on columns of
    ney + 1 free rows, past the shared-memory staging limits (9642 FP64 / 19285 FP32
    entries) where the kernel works in place, and just below a lane-segment edge.
    FP64: K_fem z = r. FP32: z close to the FP64 z (a residual check means nothing
    in FP32 here: the y systems' condition numbers reach ney^2)."""
    torch = torch_cuda
    mesh = ib.unit_square(2, 9, ney)
    plan = ib.Plan(mesh, precision=ib.MIXED)
    m, n = 11, ney + 2
    r = torch.from_numpy(splitmix_uniform(9, -1, 1, plan.nfunc)).cuda()
    r[torch.from_numpy(boundary_mask(m, n)).cuda()] = 0
    z = torch.empty_like(r)
    plan.pc_apply(r, z, pc=ib.PC_FEM_EXACT, precision=ib.FP64)
    y = torch.empty_like(r)
    plan.fem_apply(z, y, precision=ib.FP64)
    r32 = r.float()
    z32 = torch.empty_like(r32)
    plan.pc_apply(r32, z32, pc=ib.PC_FEM_EXACT, precision=ib.FP32)
    torch.cuda.synchronize()
    assert float((y - r).norm() / r.norm()) < 1e-9
    assert float((z32.double() - z).norm() / z.norm()) < 1e-2


@pytest.mark.parametrize("p,ne", [(2, 16), (3, 40), (4, 24), (3, 510), (3, 512), (5, 20)])
def test_exact_pc_solve_matches_inner_cg_solve(torch_cuda, ib, orc, p, ne):
    torch = torch_cuda
    mesh = ib.unit_square(p, ne)
    plan = ib.Plan(mesh, precision=ib.MIXED)
    b = torch.from_numpy(orc.rhs(mesh, 1)).cuda()
    xa, xb, xc = torch.zeros_like(b), torch.zeros_like(b), torch.zeros_like(b)
    sa = plan.solve(b, xa, pc=ib.PC_FEM_CG)
    sb = plan.solve(b, xb, pc=ib.PC_FEM_EXACT)
    sc = plan.solve(b, xc, pc=ib.PC_FEM_EXACT, precision=ib.MIXED)
    assert sb.relres <= 1e-10 and sc.relres <= 1e-10
    # the inner CG stops at 1e-10, the exact inverse is exact: same PCG up to a few iterations
    assert abs(sa.iterations - sb.iterations) <= max(2, 0.1 * sa.iterations)
    ref = xa.cpu().numpy()
    assert rel(xb.cpu().numpy(), ref) < 1e-7
    assert rel(xc.cpu().numpy(), ref) < 1e-7


@pytest.mark.parametrize("precision", [0, 2])
def test_large_solve_runs_as_one_conditional_graph(torch_cuda, ib, precision):
    """p=3 1536^2: the PCG loop graph (with the preconditioner's tensor-core
    GEMMs and programmatic dependencies between its kernels) instantiates, so
    no fallback message is left behind, and the solve converges."""
    torch = torch_cuda
    plan = ib.Plan(ib.unit_square(3, 1536), precision=ib.MIXED)
    b = torch.empty(plan.nfunc, dtype=torch.float64, device="cuda")
    plan.rhs(b, ib.F_SINSIN)
    x = torch.zeros_like(b)
    kw = dict(pc=ib.PC_FEM_EXACT, precision=precision)
    if precision == ib.MIXED:
        kw["sweep_rtol"] = 1e-3
    st = plan.solve(b, x, **kw)
    torch.cuda.synchronize()
    assert st.status == 0 and st.relres <= 1e-10
    assert "PCG loop" not in ib._lib().iga_last_error().decode()
    plan.close()
