"""Parity of the CUDA matrix-free operator (through the C ABI) with the reference.

Bar: FP64 results within 1e-12 relative (max-norm, relative to the largest
entry) of the reference's own element code (golden vectors) and of the oracle;
FP32 within 2e-5 relative. Repeated applies are bitwise identical.
"""
import ctypes
import os

import numpy as np
import pytest

from iga_testlib import (REF_CPU_LIB, _p, distorted, golden_mesh, load_binding, splitmix_uniform, unit_square_mesh,
                         window, window_rows)

pytestmark = pytest.mark.gpu
TOL64 = 1e-12
TOL32 = 2e-5
GOLD_CASES = ["c1", "p3_16", "p4_12", "p3_12x7"]


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


def run(torch, plan, x, dtype=None, precision=None):
    dt = dtype or (torch.float32 if plan.precision == 1 else torch.float64)
    xd = torch.from_numpy(np.asarray(x)).to(device="cuda", dtype=dt)
    yd = torch.full_like(xd, float("nan"))
    plan.apply(xd, yd, precision=precision)
    torch.cuda.synchronize()
    return yd.double().cpu().numpy()


@pytest.mark.parametrize("name", GOLD_CASES)
@pytest.mark.parametrize("geom", [0, 1])
def test_apply_matches_reference_golden(torch_cuda, ib, gold, name, geom):
    M = golden_mesh(gold, name)
    plan = ib.Plan(M, geometry=geom, IEN=gold[f"{name}_IEN"], ID=gold[f"{name}_ID"], Dir=gold[f"{name}_Dir"])
    y = run(torch_cuda, plan, gold[f"{name}_x"])
    assert rel(y, gold[f"{name}_y_mf"]) < TOL64
    assert rel(y, gold[f"{name}_y_sf"]) < TOL64


@pytest.mark.parametrize("name", GOLD_CASES)
def test_apply_equals_assembled_with_zero_dirichlet(torch_cuda, ib, gold, name):
    M = golden_mesh(gold, name)
    plan = ib.Plan(M)
    x = gold[f"{name}_x"].copy()
    x[gold[f"{name}_Dir"]] = 0.0
    assert rel(run(torch_cuda, plan, x), gold[f"{name}_y_assembled_x0"]) < TOL64


@pytest.mark.parametrize("p,nex,ney,ty", [(1, 35, 12, 4), (2, 40, 20, 8), (3, 70, 33, 16), (3, 33, 70, 5),
                                          (4, 64, 31, 12), (5, 37, 21, 7), (3, 96, 96, 0), (2, 130, 17, 0)])
@pytest.mark.parametrize("geom", [0, 1])
@pytest.mark.parametrize("bc,sign", [(0, -1), (1, 1)])
def test_apply_matches_oracle_distorted(torch_cuda, ib, orc, p, nex, ney, ty, geom, bc, sign):
    M = distorted(ib.unit_square(p, nex, ney))
    plan = ib.Plan(M, geometry=geom, bc=bc, sign=sign, rows_per_strip=ty)
    x = splitmix_uniform(p * 1000 + nex, -1.0, 1.0, plan.nfunc)
    assert rel(run(torch_cuda, plan, x), orc.apply_mf(M, x, sign=float(sign), bc=bc)) < TOL64


@pytest.mark.parametrize("geom", [0, 1])
def test_apply_with_kappa(torch_cuda, ib, orc, geom):
    M = distorted(ib.unit_square(3, 40, 36))
    M["kappa"] = np.exp(splitmix_uniform(9, -1.0, 1.0, 40 * 36 * 16))
    plan = ib.Plan(M, geometry=geom)
    x = splitmix_uniform(10, -1.0, 1.0, plan.nfunc)
    assert rel(run(torch_cuda, plan, x), orc.apply_mf(M, x)) < TOL64


@pytest.mark.parametrize("p", [2, 3, 4])
@pytest.mark.parametrize("geom", [0, 1])
def test_fp32_operator(torch_cuda, ib, orc, p, geom):
    M = distorted(ib.unit_square(p, 48, 40))
    plan = ib.Plan(M, precision=ib.FP32, geometry=geom)
    x = splitmix_uniform(p, -1.0, 1.0, plan.nfunc)
    assert rel(run(torch_cuda, plan, x), orc.apply_mf(M, x)) < TOL32


def test_mixed_plan_has_both_precisions(torch_cuda, ib, orc):
    M = ib.unit_square(3, 50, 50)
    plan = ib.Plan(M, precision=ib.MIXED)
    x = splitmix_uniform(4, -1.0, 1.0, plan.nfunc)
    ref = orc.apply_mf(M, x)
    assert rel(run(torch_cuda, plan, x, dtype=torch_cuda.float64, precision=ib.FP64), ref) < TOL64
    assert rel(run(torch_cuda, plan, x, dtype=torch_cuda.float32, precision=ib.FP32), ref) < TOL32


@pytest.mark.parametrize("geom", [0, 1])
def test_bitwise_reproducible(torch_cuda, ib, geom):
    torch = torch_cuda
    M = distorted(ib.unit_square(3, 200, 150))
    plan = ib.Plan(M, geometry=geom)
    x = torch.from_numpy(splitmix_uniform(5, -1.0, 1.0, plan.nfunc)).cuda()
    ys = []
    for _ in range(3):
        y = torch.empty_like(x)
        plan.apply(x, y)
        ys.append(y)
    torch.cuda.synchronize()
    assert torch.equal(ys[0], ys[1]) and torch.equal(ys[0], ys[2])


@pytest.mark.parametrize("p,geom,precision", [(3, 0, 0), (3, 1, 0), (4, 0, 1), (2, 0, 0)])
def test_apply_captures_into_cuda_graph(torch_cuda, ib, p, geom, precision):
    """iga_apply is stream-ordered and capturable: the MatMult captured into a
    CUDA graph (torch.cuda.graph) and replayed on new inputs in the same
    buffers gives the eager results bitwise."""
    torch = torch_cuda
    plan = ib.Plan(distorted(ib.unit_square(p, 96, 80)), geometry=geom, precision=precision)
    dt = torch.float32 if precision == ib.FP32 else torch.float64
    x = torch.from_numpy(splitmix_uniform(31, -1.0, 1.0, plan.nfunc)).to(device="cuda", dtype=dt)
    x2 = torch.from_numpy(splitmix_uniform(32, -1.0, 1.0, plan.nfunc)).to(device="cuda", dtype=dt)
    y1, y2, y = torch.empty_like(x), torch.empty_like(x), torch.empty_like(x)
    plan.apply(x, y1)
    plan.apply(x2, y2)
    xin = x.clone()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        plan.apply(xin, y, stream=torch.cuda.current_stream())
    y.fill_(float("nan"))
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(y, y1)
    xin.copy_(x2)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(y, y2)
    del g
    plan.close()


@pytest.mark.parametrize("p,nex,ney,geom,bc,ty", [(3, 64, 64, 0, 0, 0), (3, 200, 150, 0, 0, 0), (2, 90, 333, 0, 1, 0),
                                                  (4, 70, 45, 0, 0, 0), (3, 48, 200, 1, 0, 0), (3, 40, 37, 0, 1, 37),
                                                  (2, 33, 500, 1, 2, 16)])
def test_host_buffer_apply_equals_device_apply(torch_cuda, ib, p, nex, ney, geom, bc, ty):
    """iga_apply_host uploads x, applies and downloads y slab by slab on three
    streams; every point is computed as by the device apply: bitwise equal,
    for either geometry mode, every boundary rule and one-slab patches."""
    M = distorted(ib.unit_square(p, nex, ney))
    plan = ib.Plan(M, geometry=geom, bc=bc, rows_per_strip=ty)
    x = splitmix_uniform(6, -1.0, 1.0, plan.nfunc)
    ref = run(torch_cuda, plan, x)
    assert np.array_equal(plan.apply_host(x), ref)
    assert np.array_equal(plan.apply_host(x), ref)   # the pipeline's streams and events reused


def test_reference_shaped_entry_point(torch_cuda, ib, gold):
    """iga_MatrixFreeMatMultCUDA takes the reference's device-pointer argument list."""
    torch = torch_cuda
    name = "p3_16"
    M = golden_mesh(gold, name)
    dev = {k: torch.from_numpy(np.asarray(gold[f"{name}_{k}"])).cuda() for k in ("CP", "C1", "C2", "h1", "h2",
                                                                                  "IEN", "ID")}
    x = torch.from_numpy(gold[f"{name}_x"]).cuda()
    y = torch.zeros_like(x)
    L = ib.lib()
    st = L.iga_MatrixFreeMatMultCUDA(3, 3, M["nex"], M["ney"], None, None, None, None, dev["C1"].data_ptr(),
                                     dev["C2"].data_ptr(), dev["h1"].data_ptr(), dev["h2"].data_ptr(),
                                     dev["IEN"].data_ptr(), dev["ID"].data_ptr(), dev["CP"].data_ptr(), None, None,
                                     x.data_ptr(), y.data_ptr())
    assert st == 0
    torch.cuda.synchronize()
    assert rel(y.cpu().numpy(), gold[f"{name}_y_mf"]) < TOL64
    assert L.iga_MatrixFreeMatMultCUDA_release() == 0


def test_full_size_c2_properties(torch_cuda, ib, orc):
    """p=3, 2048x2048 elements (4.2M DOFs): sf == mf, windowed parity with the
    oracle at corner, edge and interior windows, linear reproduction."""
    torch = torch_cuda
    M = ib.unit_square(3, 2048, 2048)
    x = splitmix_uniform(1, -1.0, 1.0, (2051) ** 2)
    xd = torch.from_numpy(x).cuda()
    ys = {}
    for geom in (0, 1):
        plan = ib.Plan(M, geometry=geom)
        y = torch.empty_like(xd)
        plan.apply(xd, y)
        torch.cuda.synchronize()
        ys[geom] = y.cpu().numpy()
        plan.close()
    assert rel(ys[0], ys[1]) < TOL64
    Y = ys[0].reshape(2051, 2051)
    for (ea, eb, fa, fb) in [(0, 40, 0, 40), (2008, 2048, 2008, 2048), (1000, 1040, 0, 30), (700, 760, 1500, 1530),
                             (0, 33, 1017, 1090)]:
        Wm = window(M, ea, eb, fa, fb)
        r0, r1, c0, c1 = window_rows(M, ea, eb, fa, fb)
        xw = x.reshape(2051, 2051)[fa:fb + 3, ea:eb + 3].ravel()
        yw = orc.apply_mf(Wm, xw).reshape(fb - fa + 3, eb - ea + 3)
        got = Y[r0:r1, c0:c1]
        ref = yw[r0 - fa:r1 - fa, c0 - ea:c1 - ea]
        assert np.abs(got - ref).max() <= TOL64 * np.abs(ys[0]).max()
    # Coefficients of a linear function: -Laplace(u) = 0, so every row vanishes.
    cp = M["CP"].reshape(-1, 2)
    lin = torch.from_numpy(0.3 * cp[:, 0] - 0.7 * cp[:, 1] + 0.1).cuda()
    plan = ib.Plan(M)
    y = torch.empty_like(lin)
    plan.apply(lin, y)
    torch.cuda.synchronize()
    assert float(y.abs().max()) < 1e-12


def test_c1_hundred_matmults_equal_assembled_matvec(torch_cuda, ib, orc, gold):
    """p = 2, 64x64 elements: 100 matrix-free MatMults (the reference's
    MatMulMF, matrix_free/mult_mf.cpp:75) on seeded x with the Dirichlet
    entries zeroed, each against the assembled-matrix MatMult. The reference's own
    assembled matvec (ref_assembled_matvec of its compiled element code) is
    the checker where that library is present, the oracle everywhere; the 100
    applies run back to back on one plan and one stream."""
    torch = torch_cuda
    name = "c1"
    M = golden_mesh(gold, name)
    Dir = gold[f"{name}_Dir"]
    plan = ib.Plan(M, IEN=gold[f"{name}_IEN"], ID=gold[f"{name}_ID"], Dir=Dir)
    nf = plan.nfunc
    X = np.stack([splitmix_uniform(k, -1.0, 1.0, nf) for k in range(100)])
    X[:, Dir] = 0.0
    xd = torch.from_numpy(X).cuda()
    yd = torch.full_like(xd, float("nan"))
    for k in range(100):
        plan.apply(xd[k], yd[k])
    torch.cuda.synchronize()
    Y = yd.cpu().numpy()
    ref_lib = ctypes.CDLL(REF_CPU_LIB) if os.path.exists(REF_CPU_LIB) else None
    Mr = {k: np.ascontiguousarray(gold[f"{name}_{k}"]) for k in ("CP", "IEN", "ID", "Dir", "C1", "C2", "h1", "h2")}
    for k in range(100):
        assert rel(Y[k], orc.apply_mf(M, X[k])) < TOL64
        if ref_lib is not None:
            yk = np.zeros(nf)
            ref_lib.ref_assembled_matvec(M["p"], M["q"], M["nex"], M["ney"], _p(Mr["CP"]), _p(Mr["IEN"]),
                                         _p(Mr["ID"]), _p(Mr["Dir"]), len(Mr["Dir"]), _p(Mr["C1"]), _p(Mr["C2"]),
                                         _p(Mr["h1"]), _p(Mr["h2"]), _p(X[k]), _p(yk))
            assert rel(Y[k], yk) < TOL64
    plan.close()
