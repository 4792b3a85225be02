"""NURBS geometry: the exact quarter annulus (the mixed-precision configuration).

The reference has no rational geometry, so parity here is against the oracle's
restatement of the reference element algorithm extended with control-point
weights (R = w N / sum w N, the reference's own rational formulas with w = 1
generalised): parity unpinned with respect to the reference itself.
"""
import numpy as np
import pytest

from iga_testlib import load_binding, splitmix_uniform

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


def test_annulus_geometry_is_exact(ib, orc):
    """Every quadrature point lies at radius 1 + xi (linear radial map), inside the
    first quadrant, and the quadrature of the Jacobian gives the area 3 pi / 4."""
    p, ne = 4, 12
    M = ib.quarter_annulus(p, ne, ne + 3)
    xy, jw = orc.qp_points(M)
    qx, _ = orc.gauss01(p + 1)
    ex = np.repeat(np.tile(np.arange(M["nex"]), M["ney"]), (p + 1) ** 2)
    qi = np.tile(np.arange((p + 1) ** 2), M["nex"] * M["ney"]) % (p + 1)
    r = np.hypot(xy[:, 0], xy[:, 1])
    assert np.abs(r - (1.0 + (ex + qx[qi]) / M["nex"])).max() < 1e-14
    assert xy.min() > 0.0
    assert abs(jw.sum() - 0.75 * np.pi) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("p", [2, 3, 4])
@pytest.mark.parametrize("geom", [0, 1])
def test_annulus_apply_matches_oracle(torch_cuda, ib, orc, p, geom):
    torch = torch_cuda
    M = ib.quarter_annulus(p, 37, 21)
    x = splitmix_uniform(p + 40, -1.0, 1.0, (37 + p) * (21 + p))
    ref = orc.apply_mf(M, x)
    for prec, tol in ((ib.FP64, 1e-12), (ib.FP32, 2e-5)):
        plan = ib.Plan(M, precision=prec, geometry=geom)
        dt = torch.float64 if prec == ib.FP64 else torch.float32
        xd = torch.from_numpy(x).to(device="cuda", dtype=dt)
        yd = torch.empty_like(xd)
        plan.apply(xd, yd)
        torch.cuda.synchronize()
        assert rel(yd.double().cpu().numpy(), ref) < tol
        plan.close()


@pytest.mark.gpu
def test_annulus_load_vector(torch_cuda, ib, orc):
    torch = torch_cuda
    M = ib.quarter_annulus(4, 20, 26)
    plan = ib.Plan(M)
    F = torch.empty(plan.nfunc, dtype=torch.float64, device="cuda")
    plan.rhs(F, ib.F_ANNULUS)
    torch.cuda.synchronize()
    assert rel(F.cpu().numpy(), orc.rhs(M, 2)) < 1e-12


@pytest.mark.gpu
def test_annulus_mixed_precision_solve(torch_cuda, ib, orc):
    """FP32 operator + FP32 PCG sweeps with FP64 refinement reach 1e-10 and agree
    with the FP64 solve; the solution approximates u = sin(pi r) sin(2 theta)."""
    torch = torch_cuda
    M = ib.quarter_annulus(4, 24, 24)
    plan = ib.Plan(M, precision=ib.MIXED)
    b = torch.empty(plan.nfunc, dtype=torch.float64, device="cuda")
    plan.rhs(b, ib.F_ANNULUS)
    x64, x32 = torch.zeros_like(b), torch.zeros_like(b)
    s64 = plan.solve(b, x64, pc=ib.PC_FEM_EXACT)
    smx = plan.solve(b, x32, pc=ib.PC_FEM_EXACT, precision=ib.MIXED)
    assert s64.relres <= 1e-10 and smx.relres <= 1e-10 and smx.sweeps >= 2
    u64 = x64.cpu().numpy()
    assert rel(x32.cpu().numpy(), u64) < 1e-8
    # residual of the SPD system with the oracle operator
    r = b.cpu().numpy() - orc.apply_mf(M, u64, sign=1.0, bc=1)
    assert np.linalg.norm(r) / np.linalg.norm(b.cpu().numpy()) < 2e-10
    # discretisation error at the quadrature points
    xy, jw = orc.qp_points(M)
    rr, th = np.hypot(xy[:, 0], xy[:, 1]), np.arctan2(xy[:, 1], xy[:, 0])
    uex = np.sin(np.pi * rr) * np.sin(2 * th)
    uh = orc.eval_qp(M, u64)
    err = np.sqrt(np.sum(jw * (uh - uex) ** 2) / np.sum(jw * uex ** 2))
    assert err < 1e-5
