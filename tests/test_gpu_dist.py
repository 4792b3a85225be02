"""The device-resident multi-rank MatMult and PCG (include/iga_dist.h) on one
GPU: every rank's kernels, ghost exchanges (grouped NCCL send/receive) and
all-reductions run stream-ordered, the host reading the convergence test every
eight iterations. With one GPU only a single rank can run: the one-part
partition of a patch (written in the reference's file format) must give the
single-patch operator and solve, with and without an NCCL communicator of one
rank. The exchange maps of several ranks are checked on CPU against the
torch.distributed path (tests/test_partition_host.py)."""
import os

import numpy as np
import pytest

from iga_testlib import load_binding, splitmix_uniform, write_partition_files

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def one_part(ib, tmp_path, p, ne):
    mesh = ib.unit_square(p, ne)
    write_partition_files(mesh, 1, str(tmp_path))
    part = ib.Part(os.path.join(tmp_path, "info.txt"), ib.partition_filename(os.path.join(tmp_path, "part"), 0), 0)
    return mesh, part


@pytest.mark.parametrize("p,ne,with_comm", [(3, 40, False), (2, 64, True), (4, 33, False)])
def test_single_rank_dist_solver_matches_single_patch(torch_cuda, tmp_path, p, ne, with_comm):
    torch = torch_cuda
    ib = load_binding()
    mesh, part = one_part(ib, tmp_path, p, ne)
    comm = ib.NcclComm(1, 0, ib.NcclComm.unique_id()) if with_comm else None
    ds = ib.DistSolver(part, comm)
    n = part.nowned
    plan = ib.Plan(mesh, sign=ib.SIGN_SPD, bc=ib.BC_IDENTITY)
    assert plan.nfunc == n   # one part: the partition numbering is the patch's
    x = torch.from_numpy(splitmix_uniform(51, -1.0, 1.0, n)).cuda()
    m = ne + p
    mask = torch.zeros(m, m, dtype=torch.bool, device="cuda")
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = True
    x[mask.ravel()] = 0.0
    y_d, y_p = torch.empty_like(x), torch.empty_like(x)
    ds.apply(x, y_d)
    plan.apply(x, y_p)
    torch.cuda.synchronize()
    assert float((y_d - y_p).abs().max() / y_p.abs().max()) < 1e-12
    b = torch.empty_like(x)
    plan.rhs(b, ib.F_SINSIN)
    for pc in (ib.PC_NONE, ib.PC_FEM_EXACT):
        xd, xp = torch.zeros_like(b), torch.zeros_like(b)
        sd = ds.solve(b, xd, pc=pc, rtol=1e-10)
        sp = plan.solve(b, xp, pc=pc, rtol=1e-10)
        assert sd.relres <= 1e-9
        assert abs(sd.iterations - sp.iterations) <= max(2, 0.05 * sp.iterations)
        assert float((xd - xp).norm() / xp.norm()) < 1e-8
    ds.close()
    if comm is not None:
        comm.close()
    plan.close()
    part.close()
