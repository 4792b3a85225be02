"""The allocation-free MatMult entry point (iga_MatrixFreeMatMultCUDA_noalloc).

It exists for callers that cannot allocate device memory when they need a
MatMult (their memory pool owns the GPU, or a cudaMalloc/cudaFree device
synchronisation inside a solver loop is not acceptable); its scratch is a
fixed device array inside the library. Checked here against the existing
reference-shaped entry point (iga_MatrixFreeMatMultCUDA) on two calls in a row,
through the C ABI, within the FP64 tolerance of the other operator tests.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import numpy as np
import pytest

from iga_testlib import distorted, golden_mesh, load_binding, splitmix_uniform

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def bernstein_tables(orc, p):
    qx, qw = orc.gauss01(p + 1)
    B = np.concatenate([orc.bernstein(p, t)[0] for t in qx])
    dB = np.concatenate([orc.bernstein(p, t)[1] for t in qx])
    return B, dB, qw


def device_args(torch, orc, mesh):
    """Device copies of the reference-layout arrays; the x- and y-direction
    tables (B1/B2, dB1/dB2, qw1/qw2) are separate buffers, so that a mix-up
    of the two directions' arguments would show."""
    p = mesh["p"]
    B, dB, qw = bernstein_tables(orc, p)
    d = {k: torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64)).cuda()
         for k, v in dict(B1=B, dB1=dB, qw1=qw, B2=B.copy(), dB2=dB.copy(), qw2=qw.copy(), C1=mesh["C1"],
                          C2=mesh["C2"], CP=mesh["CP"], h1=np.full(mesh["nex"], 1.0 / mesh["nex"]),
                          h2=np.full(mesh["ney"], 1.0 / mesh["ney"])).items()}
    return d


def call_both(torch, ib, mesh, d, x_host):
    L = ib.lib()
    p, nex, ney = mesh["p"], mesh["nex"], mesh["ney"]
    x = torch.from_numpy(x_host).cuda()
    y_new = torch.full_like(x, float("nan"))
    y_old = torch.full_like(x, float("nan"))
    ptr = {k: v.data_ptr() for k, v in d.items()}
    st = L.iga_MatrixFreeMatMultCUDA_noalloc(p, p, nex, ney, ptr["B1"], ptr["B2"], ptr["dB1"], ptr["dB2"], ptr["C1"],
                                             ptr["C2"], ptr["h1"], ptr["h2"], None, None, ptr["CP"], ptr["qw1"],
                                             ptr["qw2"], x.data_ptr(), y_new.data_ptr(), None)
    assert st == 0, ib.lib().iga_last_error()
    st = L.iga_MatrixFreeMatMultCUDA(p, p, nex, ney, ptr["B1"], ptr["B2"], ptr["dB1"], ptr["dB2"], ptr["C1"],
                                     ptr["C2"], ptr["h1"], ptr["h2"], None, None, ptr["CP"], ptr["qw1"], ptr["qw2"],
                                     x.data_ptr(), y_old.data_ptr())
    assert st == 0, ib.lib().iga_last_error()
    torch.cuda.synchronize()
    return y_new.cpu().numpy(), y_old.cpu().numpy()


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("case", ["golden_p3_16", "p1_77x40", "p2_130x17", "p3_300x200", "p4_70x45", "p5_50x37"])
def test_noalloc_matches_existing_entry_point_twice(torch_cuda, orc, gold, case):
    ib = load_binding()
    if case == "golden_p3_16":
        mesh = golden_mesh(gold, "p3_16")
    else:
        p, dims = case.split("_")
        nex, ney = (int(v) for v in dims.split("x"))
        mesh = distorted(ib.unit_square(int(p[1]), nex, ney))
    d = device_args(torch_cuda, orc, mesh)
    n = (mesh["nex"] + mesh["p"]) * (mesh["ney"] + mesh["p"])
    for seed in (21, 22):   # two calls in a row: the shared scratch keeps the previous call's contents
        x = splitmix_uniform(seed, -1.0, 1.0, n)
        y_new, y_old = call_both(torch_cuda, ib, mesh, d, x)
        assert np.isfinite(y_new).all()
        assert rel(y_new, y_old) < TOL64
    if case == "golden_p3_16":   # and against the compiled reference's own MatMult
        x = np.asarray(gold["p3_16_x"])
        y_new, _ = call_both(torch_cuda, ib, mesh, d, x)
        assert rel(y_new, gold["p3_16_y_mf"]) < TOL64
    assert ib.lib().iga_MatrixFreeMatMultCUDA_release() == 0


def test_noalloc_refuses_misaligned_arrays_before_any_launch(torch_cuda, orc):
    """d_CP is read as 16-byte (x, y) pairs: an array 8 bytes into a larger
    buffer is refused with IGA_ERR_ARG on the host (nothing is launched, y
    keeps its contents); so are double arrays off an 8-byte boundary."""
    torch = torch_cuda
    ib = load_binding()
    L = ib.lib()
    mesh = ib.unit_square(3, 20, 12)
    d = device_args(torch, orc, mesh)
    n = (20 + 3) * (12 + 3)
    cp_buf = torch.zeros(2 * n + 1, dtype=torch.float64, device="cuda")
    cp_buf[1:] = d["CP"]
    x = torch.from_numpy(splitmix_uniform(5, -1.0, 1.0, n)).cuda()
    y = torch.full_like(x, 3.0)
    ptr = {k: v.data_ptr() for k, v in d.items()}

    def call(cp, xin):
        return L.iga_MatrixFreeMatMultCUDA_noalloc(3, 3, 20, 12, ptr["B1"], ptr["B2"], ptr["dB1"], ptr["dB2"],
                                                   ptr["C1"], ptr["C2"], None, None, None, None, cp, ptr["qw1"],
                                                   ptr["qw2"], xin, y.data_ptr(), None)

    assert call(cp_buf.data_ptr() + 8, x.data_ptr()) == 1
    assert b"16-byte" in L.iga_last_error()
    assert call(ptr["CP"], x.data_ptr() + 4) == 1
    torch.cuda.synchronize()
    assert bool((y == 3.0).all())
    assert call(ptr["CP"], x.data_ptr()) == 0   # the aligned call still works
    torch.cuda.synchronize()
    assert np.isfinite(y.cpu().numpy()).all()


def test_noalloc_rejects_meshes_beyond_its_scratch(torch_cuda):
    ib = load_binding()
    L = ib.lib()
    dummy = torch_cuda.zeros(16, dtype=torch_cuda.float64, device="cuda").data_ptr()
    # p = 3 with 8192 x 8192 elements needs far more than the fixed scratch.
    st = L.iga_MatrixFreeMatMultCUDA_noalloc(3, 3, 8192, 8192, *([dummy] * 8), None, None, dummy, dummy, dummy,
                                             dummy, dummy, None)
    assert st == 2
    assert b"16 MiB" in L.iga_last_error()
    st = L.iga_MatrixFreeMatMultCUDA_noalloc(3, 2, 8, 8, *([dummy] * 8), None, None, dummy, dummy, dummy, dummy,
                                             dummy, None)
    assert st == 2
    # a degree the entry point does not handle is "unsupported", not a bad argument
    st = L.iga_MatrixFreeMatMultCUDA_noalloc(6, 6, 8, 8, *([dummy] * 8), None, None, dummy, dummy, dummy, dummy,
                                             dummy, None)
    assert st == 2
    st = L.iga_MatrixFreeMatMultCUDA_noalloc(0, 0, 8, 8, *([dummy] * 8), None, None, dummy, dummy, dummy, dummy,
                                             dummy, None)
    assert st == 1
