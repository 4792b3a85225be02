"""Variable coefficient kappa and the adjoint gradient dJ/dkappa (no counterpart
in the reference: checked against the oracle's FP64 CPU gradient and by
central finite differences)."""
import numpy as np
import pytest

from iga_testlib import boundary_mask, distorted, load_binding, splitmix_uniform

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


def test_adjoint_grad_kernel_matches_oracle(torch_cuda, ib, orc):
    torch = torch_cuda
    M = distorted(ib.unit_square(3, 30, 22))
    plan = ib.Plan(M)
    n = plan.nfunc
    u = splitmix_uniform(1, -1, 1, n)
    lam = splitmix_uniform(2, -1, 1, n)
    g = torch.empty(30 * 22 * 16, dtype=torch.float64, device="cuda")
    plan.adjoint_grad(torch.from_numpy(u).cuda(), torch.from_numpy(lam).cuda(), g)
    torch.cuda.synchronize()
    assert rel(g.cpu().numpy(), orc.adjoint_grad(M, u, lam)) < 1e-12


@pytest.mark.parametrize("geom", [0, 1])
def test_set_kappa_equals_plan_kappa(torch_cuda, ib, orc, geom):
    torch = torch_cuda
    M = ib.unit_square(3, 40, 36)
    kappa = np.exp(ib.grf_qp(M, seed=5))
    Mk = dict(M, kappa=kappa)
    x = splitmix_uniform(3, -1, 1, 43 * 39)
    ref = orc.apply_mf(Mk, x)
    xd = torch.from_numpy(x).cuda()
    p1 = ib.Plan(Mk, geometry=geom)
    p2 = ib.Plan(M, geometry=geom)
    p2.set_kappa(torch.from_numpy(kappa).cuda())
    y1, y2 = torch.empty_like(xd), torch.empty_like(xd)
    p1.apply(xd, y1)
    p2.apply(xd, y2)
    torch.cuda.synchronize()
    assert rel(y1.cpu().numpy(), ref) < 1e-12
    assert torch.equal(y1, y2)


def test_grf_statistics(ib):
    M = ib.unit_square(3, 64)
    g = ib.grf_qp(M, sigma=1.0, ell=0.1, seed=3)
    assert abs(g.mean()) < 0.3 and 0.6 < g.std() < 1.4
    g2 = ib.grf_qp(M, sigma=1.0, ell=0.1, seed=3)
    assert np.array_equal(g, g2)


@pytest.fixture(scope="module")
def adjoint_problem(torch_cuda, ib):
    """p=3, 24x24: kappa = exp(g), u_obs = u(exp(0.8 g)) + 1% noise, J = |u - u_obs|^2 / 2."""
    torch = torch_cuda
    M = ib.unit_square(3, 24)
    g = ib.grf_qp(M, seed=3)
    plan = ib.Plan(M)
    n = plan.nfunc
    F = torch.empty(n, dtype=torch.float64, device="cuda")
    plan.rhs(F, ib.F_SINSIN)
    bmask = torch.from_numpy(boundary_mask(27, 27)).cuda()
    kw = dict(pc=ib.PC_FEM_EXACT, rtol=1e-13)
    KS = ib.kappa_solve_function()
    with torch.no_grad():
        u_true = KS.apply(torch.from_numpy(np.exp(0.8 * g)).cuda(), plan, F, bmask, kw)
    noise = torch.from_numpy(ib.splitmix_normal(3, n, offset=10 ** 7)).cuda()
    u_obs = u_true + 0.01 * float(u_true.abs().max()) * noise
    u_obs[bmask] = 0.0
    return dict(M=M, g=g, plan=plan, F=F, bmask=bmask, kw=kw, KS=KS, u_obs=u_obs)


def J_of(torch, P, kappa):
    u = P["KS"].apply(kappa, P["plan"], P["F"], P["bmask"], P["kw"])
    return 0.5 * ((u - P["u_obs"]) ** 2).sum()


def test_adjoint_gradient_vs_finite_differences(torch_cuda, ib, adjoint_problem):
    torch = torch_cuda
    P = adjoint_problem
    kappa = torch.from_numpy(np.exp(P["g"])).cuda().requires_grad_(True)
    J = J_of(torch, P, kappa)
    J.backward()
    grad = kappa.grad.clone()
    eps = 1e-6
    worst = 0.0
    for k in range(16):
        d = torch.from_numpy(ib.splitmix_normal(100 + k, kappa.numel())).cuda()
        with torch.no_grad():
            jp = J_of(torch, P, kappa + eps * d)
            jm = J_of(torch, P, kappa - eps * d)
        fd = float((jp - jm) / (2 * eps))
        ad = float((grad * d).sum())
        worst = max(worst, abs(fd - ad) / max(abs(ad), 1e-300))
    assert worst < 1e-5


def test_adjoint_gradient_vs_cpu_fp64(torch_cuda, ib, orc, adjoint_problem):
    """The same gradient from the oracle: CPU PCG forward and adjoint solves and
    the CPU gradient formula."""
    torch = torch_cuda
    P = adjoint_problem
    M = P["M"]
    kappa = np.exp(P["g"])
    kt = torch.from_numpy(kappa).cuda().requires_grad_(True)
    J = J_of(torch, P, kt)
    J.backward()
    Mk = dict(M, kappa=kappa)
    F = P["F"].cpu().numpy()
    u, it1, rr1 = orc.pcg(Mk, F, rtol=1e-12, maxit=5000)
    rhs = u - P["u_obs"].cpu().numpy()
    rhs[P["bmask"].cpu().numpy()] = 0.0
    lam, it2, rr2 = orc.pcg(Mk, rhs, rtol=1e-12, maxit=5000)
    assert it1 > 0 and it2 > 0
    g_cpu = orc.adjoint_grad(Mk, u, lam)
    assert rel(kt.grad.cpu().numpy(), g_cpu) < 1e-6
