"""The reference's own GPU MatMult kernel (matrix_free_gpu/src/mult.cu, one
quadrature point per thread, atomicAdd scatter), compiled for sm_100a into
oracle/_ref and run on the same device, against this library's MatMult: the
same y = A_ref x on the reference's own mesh tables to 1e-12 relative (the
reference kernel's atomic summation order varies from run to run)."""
import numpy as np
import pytest

from iga_testlib import RefGpuKernel, load_binding, splitmix_uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("nex,ney", [(64, 48), (130, 97)])
def test_matmult_matches_reference_gpu_kernel(torch_cuda, nex, ney):
    torch = torch_cuda
    if not RefGpuKernel.available():
        pytest.skip("oracle/_ref/libigaref_gpu.so not built (needs the reference tree)")
    ib = load_binding()
    ref = RefGpuKernel(nex, ney)
    plan = ib.Plan(ib.unit_square(3, nex, ney))
    x = torch.from_numpy(splitmix_uniform(11, -1.0, 1.0, plan.nfunc)).cuda()
    y_ref, y = torch.empty_like(x), torch.empty_like(x)
    ref.apply(x.data_ptr(), y_ref.data_ptr())
    plan.apply(x, y)
    torch.cuda.synchronize()
    a, b = y.cpu().numpy(), y_ref.cpu().numpy()
    assert np.abs(a - b).max() / np.abs(b).max() < 1e-12
    ref.close()
    plan.close()
