"""Batched solves (include/iga_batch.h): many independent problems in one
graph launch.

The batch has no reference implementation; it is checked against this
library's single-problem path (the same strip kernel must give bit-identical
operator results at the same tile shape), against the single-problem exact
preconditioner (the single plan's own GEMMs), and against the oracle's CPU PCG and operator
(every solution's residual is recomputed on the CPU).
"""
import numpy as np
import pytest

from iga_testlib import boundary_mask, distorted, load_binding, splitmix_normal, splitmix_uniform

pytestmark = pytest.mark.gpu

SHAPES = [(2, 8, 8), (3, 9, 6), (3, 40, 17), (2, 33, 70), (3, 64, 64), (2, 17, 5), (1, 12, 9), (4, 20, 26),
          (3, 130, 45), (2, 96, 128)]


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


def meshes_of(ib, shapes):
    return [ib.unit_square(p, nex, ney) for p, nex, ney in shapes]


def test_batch_apply_matches_single_plans_bitwise(torch_cuda, ib):
    torch = torch_cuda
    meshes = meshes_of(ib, SHAPES)
    meshes[2] = distorted(meshes[2])   # one non-affine patch
    batch = ib.Batch(meshes, precision=ib.MIXED)
    x = torch.from_numpy(splitmix_uniform(11, -1, 1, batch.ntot)).cuda()
    y = torch.empty_like(x)
    batch.apply(x, y)
    y32 = torch.empty_like(x, dtype=torch.float32)
    batch.apply(x.float(), y32, precision=ib.FP32)
    torch.cuda.synchronize()
    for i, m in enumerate(meshes):
        a, b = batch.offsets[i], batch.offsets[i + 1]
        ty, _ = batch.shape(i)
        plan = ib.Plan(m, precision=ib.MIXED, sign=ib.SIGN_SPD, bc=ib.BC_IDENTITY, rows_per_strip=ty)
        ys = torch.empty(b - a, dtype=torch.float64, device="cuda")
        plan.apply(x[a:b], ys, precision=ib.FP64)
        ys32 = torch.empty(b - a, dtype=torch.float32, device="cuda")
        plan.apply(x[a:b].float(), ys32, precision=ib.FP32)
        torch.cuda.synchronize()
        assert torch.equal(ys, y[a:b]), f"problem {i}"
        assert torch.equal(ys32, y32[a:b]), f"problem {i} (FP32)"


def test_batch_apply_matches_oracle(torch_cuda, ib, orc):
    torch = torch_cuda
    meshes = meshes_of(ib, SHAPES[:6])
    batch = ib.Batch(meshes)
    x = splitmix_uniform(12, -1, 1, batch.ntot)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    batch.apply(xd, yd)
    y = yd.cpu().numpy()
    for i, m in enumerate(meshes):
        a, b = batch.offsets[i], batch.offsets[i + 1]
        assert rel(y[a:b], orc.apply_mf(m, x[a:b], sign=1.0, bc=1)) < 1e-12


# FP64 GEMMs (DMMA) match the single-problem DMMA GEMMs to rounding; the FP32
# preconditioner runs its GEMMs on TF32 operands (10-bit mantissa).
@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-2)])
def test_batch_preconditioner_matches_single(torch_cuda, ib, prec, tol):
    torch = torch_cuda
    meshes = meshes_of(ib, SHAPES)
    batch = ib.Batch(meshes, precision=ib.MIXED)
    dt = torch.float64 if prec == 0 else torch.float32
    r = torch.from_numpy(splitmix_uniform(13, -1, 1, batch.ntot)).to(device="cuda", dtype=dt)
    z = torch.empty_like(r)
    batch.pc_apply(r, z, precision=prec)
    zn = torch.empty_like(r)
    batch.pc_apply(r, zn, pc=ib.PC_NONE, precision=prec)
    torch.cuda.synchronize()
    assert torch.equal(zn, r)
    for i, m in enumerate(meshes):
        a, b = batch.offsets[i], batch.offsets[i + 1]
        plan = ib.Plan(m, precision=ib.MIXED)
        zs = torch.empty(b - a, dtype=torch.float64, device="cuda")
        plan.pc_apply(r[a:b].double(), zs, pc=ib.PC_FEM_EXACT, precision=ib.FP64)
        torch.cuda.synchronize()
        assert rel(z[a:b].double().cpu().numpy(), zs.cpu().numpy()) < tol, f"problem {i}"


def residuals(orc, meshes, offsets, b, x):
    out = []
    for i, m in enumerate(meshes):
        s, e = offsets[i], offsets[i + 1]
        r = b[s:e] - orc.apply_mf(m, x[s:e], sign=1.0, bc=1)
        out.append(np.linalg.norm(r) / max(np.linalg.norm(b[s:e]), 1e-300))
    return np.array(out)


@pytest.mark.parametrize("prec", [0, 2])
def test_batch_solve_matches_oracle(torch_cuda, ib, orc, prec):
    torch = torch_cuda
    meshes = meshes_of(ib, SHAPES)
    batch = ib.Batch(meshes, precision=prec)
    b = ib.batch_rhs(SHAPES, seed=2)
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros_like(bd)
    st, its, relres = batch.solve(bd, xd, rtol=1e-10)
    x = xd.cpu().numpy()
    assert st.status == 0 and st.converged == len(meshes)
    assert np.all(relres <= 1e-10) and st.max_relres <= 1e-10
    assert np.all(residuals(orc, meshes, batch.offsets, b, x) < 1.5e-10)
    if prec == 2:
        assert st.max_sweeps >= 2
    # the oracle's own CPU PCG on the small problems
    for i in (0, 1, 5):
        s, e = batch.offsets[i], batch.offsets[i + 1]
        x_ref, it_ref, _ = orc.pcg(meshes[i], b[s:e], rtol=1e-10)
        assert rel(x[s:e], x_ref) < 1e-7


def test_batch_solve_matches_single_solves(torch_cuda, ib):
    torch = torch_cuda
    shapes = SHAPES[2:6]
    meshes = meshes_of(ib, shapes)
    batch = ib.Batch(meshes)
    b = ib.batch_rhs(shapes, seed=5)
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros_like(bd)
    st, its, _ = batch.solve(bd, xd)
    for i, m in enumerate(meshes):
        s, e = batch.offsets[i], batch.offsets[i + 1]
        plan = ib.Plan(m)
        xs = torch.zeros(e - s, dtype=torch.float64, device="cuda")
        ss = plan.solve(bd[s:e].contiguous(), xs, pc=ib.PC_FEM_EXACT)
        torch.cuda.synchronize()
        assert abs(ss.iterations - its[i]) <= 2
        assert rel(xd[s:e].cpu().numpy(), xs.cpu().numpy()) < 1e-8


def test_batch_edge_cases(torch_cuda, ib, orc):
    torch = torch_cuda
    shapes = [(3, 12, 12), (2, 30, 9), (3, 7, 40)]
    meshes = meshes_of(ib, shapes)
    batch = ib.Batch(meshes, precision=ib.MIXED)
    b = ib.batch_rhs(shapes, seed=7)
    s1, e1 = batch.offsets[1], batch.offsets[2]
    b[s1:e1] = 0.0                      # a zero right-hand side: x = 0, no iterations
    bd = torch.from_numpy(b).cuda()
    for prec_kw in ({}, {"pc": ib.PC_NONE}):
        xd = torch.full_like(bd, 3.0)   # ignored: x0 = 0 unless x0_nonzero
        st, its, relres = batch.solve(bd, xd, **prec_kw)
        x = xd.cpu().numpy()
        assert st.status == 0 and its[1] == 0 and np.all(x[s1:e1] == 0.0)
        assert np.all(residuals(orc, meshes, batch.offsets, b, x) < 1.5e-10)
    # restarting from the solution converges at once
    st2, its2, _ = batch.solve(bd, xd, x0_nonzero=1)
    assert st2.status == 0 and its2.max() <= 1
    # a solve that cannot converge reports it per problem
    st3, its3, relres3 = batch.solve(bd, torch.zeros_like(bd), check=False, max_it=1, max_sweeps=1, pc=ib.PC_NONE)
    assert st3.status == 5 and st3.converged == 1      # only the zero problem
    # a single problem and repeated solves give identical results
    one = ib.Batch(meshes[:1])
    x1, x2 = torch.zeros(one.ntot, dtype=torch.float64, device="cuda"), torch.zeros(one.ntot, dtype=torch.float64,
                                                                                      device="cuda")
    one.solve(bd[:one.ntot].contiguous(), x1)
    one.solve(bd[:one.ntot].contiguous(), x2)
    torch.cuda.synchronize()
    assert torch.equal(x1, x2)


def test_batch_nonfinite_problem_is_isolated(torch_cuda, ib):
    torch = torch_cuda
    shapes = [(2, 16, 16), (3, 20, 12)]
    batch = ib.Batch(meshes_of(ib, shapes))
    b = ib.batch_rhs(shapes, seed=9)
    b[batch.offsets[0] + 40] = np.nan
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros_like(bd)
    st, its, relres = batch.solve(bd, xd, check=False)
    assert st.status == 7 and st.converged == 1 and relres[1] <= 1e-10


def test_autotune_writes_table_and_batch_uses_it(torch_cuda, ib, tmp_path):
    shapes = [(3, 48, 48), (3, 64, 40), (2, 128, 128), (2, 120, 100), (3, 200, 180)]
    meshes = meshes_of(ib, shapes)
    path = str(tmp_path / "tune.json")
    ib.batch_autotune(meshes, path, precision=ib.FP64)
    import json
    t = json.load(open(path))
    assert t["format"] == "iga-batch-tune-1" and t["rows"] and t["warps"]
    batch = ib.Batch(meshes, tune_file=path)
    for i, (p, nex, ney) in enumerate(shapes):
        rows, warps = ib.tune_lookup(path, p, ib.FP64, nex, ney)
        assert rows > 0 and warps > 0
        assert batch.shape(i) == (max(rows, p), warps)


def test_full_size_batch_converges(torch_cuda, ib):
    """256 problems, p in {2, 3}, 32..256 elements per direction (seed 2): every
    problem reaches 1e-10 in FP64 and in mixed precision."""
    torch = torch_cuda
    shapes = ib.batch_problems(256, seed=2)
    meshes = meshes_of(ib, shapes)
    b = torch.from_numpy(ib.batch_rhs(shapes, seed=2)).cuda()
    for prec in (ib.FP64, ib.MIXED):
        batch = ib.Batch(meshes, precision=prec)
        x = torch.zeros_like(b)
        st, its, relres = batch.solve(b, x)
        assert st.status == 0 and st.converged == 256 and relres.max() <= 1e-10
        # the residual seen from the single-problem path
        for i in (0, 100, 255):
            s, e = batch.offsets[i], batch.offsets[i + 1]
            plan = ib.Plan(meshes[i], sign=ib.SIGN_SPD, bc=ib.BC_IDENTITY)
            q = torch.empty(e - s, dtype=torch.float64, device="cuda")
            plan.apply(x[s:e], q)
            torch.cuda.synchronize()
            assert float((b[s:e] - q).norm() / b[s:e].norm()) <= 1.5e-10
        batch.close()
