"""The partitioned MatMult on the GPU (include/iga_part.h): every part's
ghosted element loop (iga_part_apply) plus the ghost exchange of
parallel-computing_b200/iga_dist.py, all parts emulated in one process on the
one GPU, against the reference's partitioned MatMulMF (committed fixtures
written by the reference's own preprocessor) and against the single-patch
operator. Tolerance 1e-12 relative, as for the other FP64 MatMult tests.
"""
import os

import numpy as np
import pytest

from iga_testlib import (PARTITIONS, load_binding, partition_numbering, read_info, splitmix_uniform,
                         unit_square_mesh, write_partition_files)

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


def parts_of(ib, d, P, **kw):
    info = os.path.join(d, "info.txt")
    return [ib.Part(info, ib.partition_filename(os.path.join(d, "part"), r), r).build(**kw) for r in range(P * P)]


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", ["p3_9x7_2", "p2_10x12_3", "p4_8x11_2"])
def test_partitioned_matmult_matches_reference(torch_cuda, ib, name):
    torch = torch_cuda
    from iga_dist import emulate_partitioned_matmult
    d = os.path.join(PARTITIONS, name)
    P = int(read_info(os.path.join(d, "info.txt"))["part_num_1d"])
    v = np.load(os.path.join(d, "vectors.npz"))
    parts = parts_of(ib, d, P)
    y = emulate_partitioned_matmult(parts, torch.from_numpy(v["x"]).cuda())
    assert rel(y.cpu().numpy(), v["y"]) < 1e-12


@pytest.mark.parametrize("p,nex,ney,P", [(3, 240, 170, 3), (4, 90, 130, 2), (2, 64, 64, 4)])
def test_partitioned_matmult_matches_single_patch(torch_cuda, ib, orc, tmp_path, p, nex, ney, P):
    """Larger meshes (files from the test writer): the sum over parts equals
    the single-patch plan's MatMult, both sign/boundary modes."""
    torch = torch_cuda
    from iga_dist import emulate_partitioned_matmult
    mesh = unit_square_mesh(orc, p, p, nex, ney)
    write_partition_files(mesh, P, str(tmp_path))
    new = partition_numbering(p, p, nex, ney, P)
    x_nat = splitmix_uniform(21, -1.0, 1.0, (nex + p) * (ney + p))
    x_new = np.empty_like(x_nat)
    x_new[new] = x_nat
    for sign, bc in ((ib.SIGN_REFERENCE, ib.BC_REFERENCE), (ib.SIGN_SPD, ib.BC_IDENTITY)):
        parts = parts_of(ib, str(tmp_path), P, sign=sign, bc=bc)
        y_new = emulate_partitioned_matmult(parts, torch.from_numpy(x_new).cuda()).cpu().numpy()
        plan = ib.Plan(mesh, sign=sign, bc=bc)
        yd = torch.empty(plan.nfunc, dtype=torch.float64, device="cuda")
        plan.apply(torch.from_numpy(x_nat).cuda(), yd)
        torch.cuda.synchronize()
        assert rel(y_new[new], yd.cpu().numpy()) < 1e-12
        for pt in parts:
            pt.close()


def test_partitioned_matmult_is_reproducible(torch_cuda, ib):
    torch = torch_cuda
    from iga_dist import emulate_partitioned_matmult
    d = os.path.join(PARTITIONS, "p2_10x12_3")
    parts = parts_of(ib, d, 3)
    x = torch.from_numpy(np.load(os.path.join(d, "vectors.npz"))["x"]).cuda()
    a = emulate_partitioned_matmult(parts, x)
    b = emulate_partitioned_matmult(parts, x)
    assert torch.equal(a, b)
    with pytest.raises(ib.IgaError):
        parts[0].build()                      # built once


@pytest.mark.parametrize("p,ne,P", [(2, 160, 2), (3, 150, 3)])
def test_partitioned_pcg_matches_single_patch_solve(torch_cuda, ib, orc, tmp_path, p, ne, P):
    """The multi-rank Krylov loop of iga_dist (all parts emulated in one process
    on the one GPU): part MatMults on the device, the block FEM preconditioner
    on each part's sub-patch plan (device exact inverse); the solution equals
    the single-patch FP64 solve; at p = 2 the block preconditioner cuts the
    iteration count of the unpreconditioned loop (at p = 3 on meshes this
    small the FEM preconditioner is no better than none)."""
    torch = torch_cuda
    from iga_dist import BlockFemPC, emulate_partitioned_pcg
    mesh = unit_square_mesh(orc, p, p, ne, ne)
    write_partition_files(mesh, P, str(tmp_path))
    m = ne + p
    new = partition_numbering(p, p, ne, ne, P)
    b = splitmix_uniform(22, -1.0, 1.0, m * m)
    mask = np.zeros((m, m), bool)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = True
    b[mask.ravel()] = 0.0
    plan = ib.Plan(mesh)
    bd = torch.from_numpy(b).cuda()
    xs = torch.zeros_like(bd)
    plan.solve(bd, xs, pc=ib.PC_FEM_EXACT, rtol=1e-12)
    xs_new = torch.empty_like(xs)
    xs_new[torch.from_numpy(new).cuda()] = xs
    b_new = torch.empty_like(bd)
    b_new[torch.from_numpy(new).cuda()] = bd
    parts = parts_of(ib, str(tmp_path), P, sign=ib.SIGN_SPD, bc=ib.BC_IDENTITY)
    x0, it0, r0 = emulate_partitioned_pcg(parts, b_new, rtol=1e-11)
    pcs = [BlockFemPC(pt, "cuda:0") for pt in parts]
    x1, it1, r1 = emulate_partitioned_pcg(parts, b_new, pcs=pcs, rtol=1e-11)
    torch.cuda.synchronize()
    for x in (x0, x1):
        assert float((x - xs_new).norm() / xs_new.norm()) < 1e-9
    assert r0 <= 1e-11 and r1 <= 1e-11
    if p == 2:
        assert it1 < it0


@pytest.mark.parametrize("p,ne,P", [(2, 96, 2), (3, 90, 3)])
def test_partitioned_fem_cg_pc_matches_single_patch_fem_cg(torch_cuda, ib, orc, tmp_path, p, ne, P):
    """The reference's preconditioner across parts (inner Jacobi-CG to 1e-10 on
    the distributed FEM matrix, iga_dist.FemCGPC) with the part MatMults on
    the device, all parts emulated on the one GPU: the single-patch solve with
    IGA_PC_FEM_CG (the same preconditioner on the device), in its iteration
    count within 2."""
    torch = torch_cuda
    from iga_dist import emulate_fem_cg_pc, emulate_partitioned_pcg
    mesh = unit_square_mesh(orc, p, p, ne, ne)
    write_partition_files(mesh, P, str(tmp_path))
    m = ne + p
    new = torch.from_numpy(partition_numbering(p, p, ne, ne, P)).cuda()
    b = splitmix_uniform(23, -1.0, 1.0, m * m)
    mask = np.zeros((m, m), bool)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = True
    b[mask.ravel()] = 0.0
    plan = ib.Plan(mesh)
    bd = torch.from_numpy(b).cuda()
    xs = torch.zeros_like(bd)
    st = plan.solve(bd, xs, pc=ib.PC_FEM_CG, rtol=1e-11)
    b_new = torch.empty_like(bd)
    b_new[new] = bd
    parts = parts_of(ib, str(tmp_path), P, sign=ib.SIGN_SPD, bc=ib.BC_IDENTITY)
    pc = emulate_fem_cg_pc(parts, "cuda:0")
    x, its, r = emulate_partitioned_pcg(parts, b_new, rtol=1e-11, pc_global=pc)
    torch.cuda.synchronize()
    assert r <= 1e-11 and pc.last_iterations > 0
    assert float((x[new] - xs).norm() / xs.norm()) < 1e-9
    assert abs(its - st.iterations) <= 2
