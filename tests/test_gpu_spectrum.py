"""Spectral estimates (iga_spectrum_estimate): Lanczos extremes of K and of
the FEM-preconditioned M^-1 K against dense eigen-solves of the oracle's
operator and the assembled FEM matrix, and the h-independence of the
preconditioned condition number (the property the reference's
eigenvalue_problem/ study measures)."""
import numpy as np
import pytest

from iga_testlib import boundary_mask, load_binding

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


def dense_interior(orc, mesh, plan):
    m, n = mesh["nex"] + mesh["p"], mesh["ney"] + mesh["p"]
    free = ~boundary_mask(m, n)
    idx = np.nonzero(free)[0]
    K = np.empty((len(idx), len(idx)))
    for c, j in enumerate(idx):
        e = np.zeros(m * n)
        e[j] = 1.0
        K[:, c] = orc.apply_mf(mesh, e, sign=1.0, bc=1)[idx]
    rp, col, val = plan.fem_csr(sign=1)
    F = np.zeros((m * n, m * n))
    for i in range(m * n):
        F[i, col[rp[i]:rp[i + 1]]] = val[rp[i]:rp[i + 1]]
    return 0.5 * (K + K.T), F[np.ix_(idx, idx)]


@pytest.mark.parametrize("p,nex,ney", [(3, 12, 10), (2, 14, 9), (4, 9, 9)])
def test_lanczos_extremes_match_dense(torch_cuda, ib, orc, p, nex, ney):
    import scipy.linalg
    mesh = ib.unit_square(p, nex, ney)
    plan = ib.Plan(mesh)
    K, F = dense_interior(orc, mesh, plan)
    ek = np.linalg.eigvalsh(K)
    ep = scipy.linalg.eigh(K, F, eigvals_only=True)
    n = K.shape[0]
    # the largest Ritz value converges first and to rounding; the smallest to
    # 1e-4 (p = 2 has a tight cluster at the bottom of the preconditioned spectrum)
    lo, hi, k = plan.spectrum(pc=ib.PC_NONE, steps=n + 20)
    assert abs(lo / ek[0] - 1) < 1e-4 and abs(hi / ek[-1] - 1) < 1e-8
    for pc in (ib.PC_FEM_EXACT, ib.PC_FEM_CG):
        lo, hi, k = plan.spectrum(pc=pc, steps=n + 20)
        assert abs(lo / ep[0] - 1) < 1e-4 and abs(hi / ep[-1] - 1) < 1e-6, (pc, lo, hi, ep[0], ep[-1])


def test_preconditioned_condition_number_is_mesh_independent(torch_cuda, ib):
    kap_k, kap_p = [], []
    for ne in (32, 64, 128):
        plan = ib.Plan(ib.unit_square(3, ne))
        lo, hi, _ = plan.spectrum(pc=ib.PC_NONE, steps=400)
        kap_k.append(hi / lo)
        lo, hi, _ = plan.spectrum(pc=ib.PC_FEM_EXACT, steps=200)
        kap_p.append(hi / lo)
    # K: about 4x per refinement (kappa ~ h^-2); M^-1 K: bounded
    assert 3.0 < kap_k[1] / kap_k[0] < 4.5 and 3.0 < kap_k[2] / kap_k[1] < 4.5
    assert max(kap_p) / min(kap_p) < 1.2 and max(kap_p) < 200
