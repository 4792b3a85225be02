"""The reference-shaped MatMult entry point (iga_MatrixFreeMatMultCUDA) against
the reference's own GPU kernel (matrix_free_gpu/src/mult.cu, built for sm_100a
into oracle/_ref) on equation numberings other than the serial one, its checks
of the caller's IEN / ID / Bernstein tables, the load vector against the
reference's AssemLoad (golden vectors), and the bounded-wait timeout path of
the MatMult kernel with the plan status query."""
import numpy as np
import pytest

from iga_testlib import RefGpuKernel, golden_mesh, load_binding, splitmix_uniform

pytestmark = pytest.mark.gpu
TOL64 = 1e-12
ERR_ARG, ERR_UNSUPPORTED, ERR_TIMEOUT = 1, 2, 8


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


def serial_id(m, n):
    """The reference's serial numbering (matrix_free/src/Partition.cpp:102-108)."""
    A = np.arange(m * n, dtype=np.int32).reshape(n, m)
    A[0, :] = A[-1, :] = A[:, 0] = A[:, -1] = -1
    return A.ravel()


def numbering(kind, m, n):
    ID = serial_id(m, n).reshape(n, m)
    if kind == "top_side_free":   # the top side is not Dirichlet: its control points keep their rows
        ID[-1, :] = np.arange((n - 1) * m, n * m)
        ID[-1, 0] = ID[-1, -1] = -1
    elif kind == "reversed":       # free control points numbered backwards
        free = ID >= 0
        ID[free] = m * n - 1 - ID[free]
    elif kind == "compressed":     # free control points numbered 0, 1, 2, ... (a PETSc-style global vector)
        free = ID >= 0
        ID[free] = np.arange(int(free.sum()))
    return ID.ravel()


def device(torch, arrays):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in arrays.items() if v is not None}


def call_cached(L, p, nex, ney, d, x, y, with_tables=True):
    ptr = lambda k: d[k].data_ptr() if k in d else None  # noqa: E731
    B, dB, qw = (ptr("B"), ptr("dB"), ptr("qw")) if with_tables else (None, None, None)
    return L.iga_MatrixFreeMatMultCUDA(p, p, nex, ney, B, B, dB, dB, ptr("C1"), ptr("C2"), ptr("h1"), ptr("h2"),
                                       ptr("IEN"), ptr("ID"), ptr("CP"), qw, qw, x.data_ptr(), y.data_ptr())


def call_noalloc(L, p, nex, ney, d, x, y):
    ptr = lambda k: d[k].data_ptr() if k in d else None  # noqa: E731
    return L.iga_MatrixFreeMatMultCUDA_noalloc(p, p, nex, ney, ptr("B"), ptr("B"), ptr("dB"), ptr("dB"), ptr("C1"),
                                               ptr("C2"), ptr("h1"), ptr("h2"), ptr("IEN"), ptr("ID"), ptr("CP"),
                                               ptr("qw"), ptr("qw"), x.data_ptr(), y.data_ptr(), None)


@pytest.mark.parametrize("kind", ["serial", "top_side_free", "reversed", "compressed"])
@pytest.mark.parametrize("entry", ["cached", "noalloc"])
def test_reference_entry_honours_ID_like_the_reference_kernel(torch_cuda, ib, kind, entry):
    """Rows go to y[ID[A]] (none for ID < 0), as in the reference kernel's
    scatter (matrix_free_gpu/src/mult.cu:455-460); y is zeroed first, as the
    reference caller does (GlobalAssemblyMF.cu:210)."""
    torch = torch_cuda
    if not RefGpuKernel.available():
        pytest.skip("oracle/_ref/libigaref_gpu.so not built (needs the reference tree)")
    nex, ney, p = 64, 48, 3
    m, n = nex + p, ney + p
    ID = numbering(kind, m, n)
    ref = RefGpuKernel(nex, ney, ID=ID)
    d = device(torch, ref.arrays)
    L = ib.lib()
    for seed in (31, 32):
        x = torch.from_numpy(splitmix_uniform(seed, -1.0, 1.0, m * n)).cuda()
        y_ref, y = torch.zeros_like(x), torch.zeros_like(x)
        ref.apply(x.data_ptr(), y_ref.data_ptr())
        st = (call_cached if entry == "cached" else call_noalloc)(L, p, nex, ney, d, x, y)
        assert st == 0, L.iga_last_error()
        torch.cuda.synchronize()
        a, b = y.cpu().numpy(), y_ref.cpu().numpy()
        assert rel(a, b) < TOL64
        assert np.array_equal(a == 0, b == 0)   # the same rows receive nothing
    ref.close()
    assert L.iga_MatrixFreeMatMultCUDA_release() == 0


@pytest.mark.parametrize("entry", ["cached", "noalloc"])
@pytest.mark.parametrize("bad", ["IEN_swapped", "ID_twice", "ID_range"])
def test_reference_entry_refuses_arrays_it_cannot_honour(torch_cuda, ib, gold, entry, bad):
    torch = torch_cuda
    name = "p3_16"
    M = golden_mesh(gold, name)
    p, nex, ney = 3, M["nex"], M["ney"]
    N = (nex + p) * (ney + p)
    IEN = np.array(gold[f"{name}_IEN"], np.int32)
    ID = np.array(gold[f"{name}_ID"], np.int32)
    if bad == "IEN_swapped":
        IEN[[5, 6]] = IEN[[6, 5]]
    elif bad == "ID_twice":
        ID[N // 2 + 1] = ID[N // 2]
    else:
        ID[N // 2] = N
    qx, qw = gold["tab_p3_qp"], gold["tab_p3_qw"]
    d = device(torch, dict(CP=M["CP"], C1=M["C1"], C2=M["C2"], h1=M["h1"], h2=M["h2"], IEN=IEN, ID=ID,
                           B=gold["tab_p3_B"], dB=gold["tab_p3_dB"], qw=qw))
    assert len(qx) == 4
    x = torch.from_numpy(gold[f"{name}_x"]).cuda()
    y = torch.full_like(x, 7.0)
    L = ib.lib()
    st = (call_cached if entry == "cached" else call_noalloc)(L, p, nex, ney, d, x, y)
    assert st == ERR_UNSUPPORTED
    assert L.iga_last_error()
    torch.cuda.synchronize()
    assert bool((y == 7.0).all())   # refused before y is touched
    assert L.iga_MatrixFreeMatMultCUDA_release() == 0


def test_reference_entry_checks_the_callers_rule_tables(torch_cuda, ib, gold):
    """The reference's own Bernstein tables and Gauss weights are accepted;
    tables of another rule are refused (the plan integrates with its own)."""
    torch = torch_cuda
    name = "p3_16"
    M = golden_mesh(gold, name)
    base = dict(CP=M["CP"], C1=M["C1"], C2=M["C2"], h1=M["h1"], h2=M["h2"], IEN=gold[f"{name}_IEN"],
                ID=gold[f"{name}_ID"], B=gold["tab_p3_B"], dB=gold["tab_p3_dB"], qw=gold["tab_p3_qw"])
    x = torch.from_numpy(gold[f"{name}_x"]).cuda()
    L = ib.lib()
    y = torch.zeros_like(x)
    d_base = device(torch, base)   # kept alive: a freed array's address may be reused by the next one
    assert call_cached(L, 3, M["nex"], M["ney"], d_base, x, y) == 0
    torch.cuda.synchronize()
    assert rel(y.cpu().numpy(), gold[f"{name}_y_mf"]) < TOL64
    d_other = dict(d_base)
    d_other["qw"] = torch.full((4,), 0.25, dtype=torch.float64, device="cuda")   # equal weights: not Gauss
    assert call_cached(L, 3, M["nex"], M["ney"], d_other, x, y) == ERR_UNSUPPORTED
    assert L.iga_MatrixFreeMatMultCUDA_release() == 0


def test_reference_entry_rejects_misaligned_vectors(torch_cuda, ib, gold):
    torch = torch_cuda
    M = golden_mesh(gold, "p3_16")
    d = device(torch, dict(CP=M["CP"], C1=M["C1"], C2=M["C2"]))
    N = (M["nex"] + 3) * (M["ney"] + 3)
    buf = torch.zeros(N + 1, dtype=torch.float64, device="cuda")
    L = ib.lib()
    ptr = buf.data_ptr() + 4   # not a multiple of 8: refused on the host, nothing launched
    st = L.iga_MatrixFreeMatMultCUDA(3, 3, M["nex"], M["ney"], None, None, None, None, d["C1"].data_ptr(),
                                     d["C2"].data_ptr(), None, None, None, None, d["CP"].data_ptr(), None, None, ptr,
                                     buf.data_ptr())
    assert st == ERR_ARG


@pytest.mark.parametrize("name", ["c1", "p3_16", "p4_12", "p3_12x7"])
def test_load_vector_matches_reference_golden(torch_cuda, ib, gold, name):
    """iga_rhs(IGA_F_REFERENCE) against the reference's GlobalAssemblyMF::AssemLoad
    (matrix_free/src/GlobalAssemblyMF.cpp:26-80, f of LocalAssemblyMF.hpp:52-55)."""
    torch = torch_cuda
    M = golden_mesh(gold, name)
    plan = ib.Plan(M)
    F = torch.full((plan.nfunc,), float("nan"), dtype=torch.float64, device="cuda")
    plan.rhs(F, fkind=ib.F_REFERENCE)
    torch.cuda.synchronize()
    ref = gold[f"{name}_F"]
    got = F.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    plan.close()


def test_bounded_wait_timeout_is_reported_and_the_plan_recovers(torch_cuda, ib, orc):
    """A wait limit of 0 polls makes every G-stage wait of the MatMult kernel
    give up at once; the kernel records IGA_ERR_TIMEOUT, lets its bulk copies
    land and returns; the status query reports it once; with the default
    limit back the next MatMult matches the oracle."""
    torch = torch_cuda
    M = ib.unit_square(3, 96, 80)
    plan = ib.Plan(M, geometry=ib.GEOM_PRECOMPUTED)
    x_h = splitmix_uniform(41, -1.0, 1.0, plan.nfunc)
    x = torch.from_numpy(x_h).cuda()
    y = torch.zeros_like(x)
    assert plan.device_status() == 0
    plan.set_wait_limit(0)
    plan.apply(x, y)
    assert plan.device_status() == ERR_TIMEOUT
    assert plan.device_status() == 0   # cleared by the query
    plan.set_wait_limit(-1)
    plan.apply(x, y)
    assert plan.device_status() == 0
    ref = orc.apply_mf(M, x_h)
    assert rel(y.cpu().numpy(), ref) < TOL64
    plan.close()
