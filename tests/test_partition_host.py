"""Partitioned meshes on the host (no GPU): the reader of the reference's
partition files (include/iga_part.h) against files written by the
reference's own Partition + FileManager (tests/golden/partitions/), and the
multi-rank ghost exchange (parallel-computing_b200/iga_dist.py) over gloo
with one process per part, the local element loop done by the CPU oracle.
"""
import os
import shutil
import socket

import numpy as np
import pytest

from iga_testlib import (PARTITIONS, load_binding, partition_numbering, read_info, splitmix_uniform, unit_square_mesh,
                         write_partition_files)

CASES = ["p3_9x7_2", "p2_10x12_3", "p4_8x11_2"]


@pytest.fixture(scope="module")
def ib():
    return load_binding()


def case_info(name):
    d = os.path.join(PARTITIONS, name)
    info = read_info(os.path.join(d, "info.txt"))
    p, q, nex, ney, P = (int(info[k]) for k in ("p", "q", "nElemX", "nElemY", "part_num_1d"))
    return d, p, q, nex, ney, P


def open_parts(ib, name):
    d, p, q, nex, ney, P = case_info(name)
    return [ib.Part(os.path.join(d, "info.txt"), ib.partition_filename(os.path.join(d, "part"), r), r)
            for r in range(P * P)]


@pytest.mark.parametrize("name", CASES)
def test_reader_accepts_reference_partitions(ib, name):
    d, p, q, nex, ney, P = case_info(name)
    parts = open_parts(ib, name)
    off = 0
    for r, pt in enumerate(parts):
        i = pt.info
        assert (i.p, i.q, i.nElemX, i.nElemY, i.part_num_1d, i.rank) == (p, q, nex, ney, P, r)
        assert pt.owned_offset == off
        off += pt.nowned
        assert np.all(np.diff(pt.ghosts) > 0)                       # the reference sorts them
        assert sorted(pt.block_to_local.tolist()) == list(range(pt.nowned + pt.nghost))
        assert i.block_m * i.block_n == pt.nowned + pt.nghost
    assert off == (nex + p) * (ney + q)
    # every element belongs to exactly one part
    assert sum(pt.info.nlocalelemx * pt.info.nlocalelemy for pt in parts) == nex * ney


@pytest.mark.parametrize("name", CASES)
def test_reference_partitioned_matmult_equals_serial(orc, name):
    """Pins the fixtures: the reference's partitioned element loop (recorded
    y) equals the serial oracle MatMult in the partition numbering."""
    d, p, q, nex, ney, P = case_info(name)
    v = np.load(os.path.join(d, "vectors.npz"))
    new = partition_numbering(p, q, nex, ney, P)
    mesh = unit_square_mesh(orc, p, q, nex, ney)
    y_nat = orc.apply_mf(mesh, v["x"][new], sign=-1.0, bc=0)
    y = np.empty_like(y_nat)
    y[new] = y_nat
    assert np.abs(y - v["y"]).max() <= 1e-12 * np.abs(v["y"]).max()


@pytest.mark.parametrize("name", CASES)
def test_sub_patch_is_the_global_block(ib, orc, name):
    d, p, q, nex, ney, P = case_info(name)
    g = unit_square_mesh(orc, p, q, nex, ney)
    m = nex + p
    cp = g["CP"].reshape(ney + q, m, 2)
    for pt in open_parts(ib, name):
        i = pt.info
        sm = pt.mesh()
        blk = cp[i.elem_y0:i.elem_y0 + i.block_n, i.elem_x0:i.elem_x0 + i.block_m]
        # the files hold 16 significant digits (std::setprecision(16))
        assert np.abs(sm["CP"].reshape(i.block_n, i.block_m, 2) - blk).max() < 1e-15
        e1 = (p + 1) ** 2
        assert np.abs(sm["C1"] - g["C1"][i.elem_x0 * e1:(i.elem_x0 + i.nlocalelemx) * e1]).max() < 1e-15


def local_oracle(orc, part, sub, x_local, sign=-1.0):
    """The part's element loop on the CPU (checker): block gather, oracle
    sub-patch MatMult with no boundary rule, scatter, rows ID < 0 zero."""
    xb = x_local[part.block_to_local]
    yb = orc.apply_mf(sub, xb, sign=sign, bc=2)
    y = np.empty_like(x_local)
    y[part.block_to_local] = yb
    y[part.local_id < 0] = 0.0
    return y


@pytest.mark.parametrize("name", CASES)
def test_emulated_exchange_matches_reference(ib, orc, name):
    import torch
    from iga_dist import emulate_partitioned_matmult
    d, p, q, nex, ney, P = case_info(name)
    v = np.load(os.path.join(d, "vectors.npz"))
    parts = open_parts(ib, name)
    subs = [pt.mesh() for pt in parts]

    def apply(part, xl, yl):
        yl.copy_(torch.from_numpy(local_oracle(orc, part, subs[part.rank], xl.numpy())))
    y = emulate_partitioned_matmult(parts, torch.from_numpy(v["x"]), local_apply=apply).numpy()
    assert np.abs(y - v["y"]).max() <= 1e-12 * np.abs(v["y"]).max()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _gloo_rank(rank, world, port, name, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from iga_testlib import Oracle
        import iga_b200 as ib
        from iga_dist import DistPartOperator
        orc = Oracle()
        d = os.path.join(PARTITIONS, name)
        part = ib.Part(os.path.join(d, "info.txt"), ib.partition_filename(os.path.join(d, "part"), rank), rank)
        sub = part.mesh()

        def apply(xl, yl):
            yl.copy_(torch.from_numpy(local_oracle(orc, part, sub, xl.numpy())))
        op = DistPartOperator(part, dist, "cpu", local_apply=apply)
        v = np.load(os.path.join(d, "vectors.npz"))
        x_owned = torch.from_numpy(v["x"][part.owned_offset:part.owned_offset + part.nowned].copy())
        y_owned = torch.empty_like(x_owned)
        op.matmult(x_owned, y_owned)
        np.save(os.path.join(out_dir, f"y{rank}.npy"), y_owned.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["p3_9x7_2", "p2_10x12_3"])
def test_gloo_ranks_match_reference(ib, name, tmp_path):
    """One process per part over gloo: forward ghost update, local element
    loop, reverse add; the assembled owned rows equal the reference's
    partitioned MatMult."""
    import torch.multiprocessing as mp
    d, p, q, nex, ney, P = case_info(name)
    world = P * P
    mp.start_processes(_gloo_rank, args=(world, _free_port(), name, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    v = np.load(os.path.join(d, "vectors.npz"))
    y = np.concatenate([np.load(os.path.join(tmp_path, f"y{r}.npy")) for r in range(world)])
    assert np.abs(y - v["y"]).max() <= 1e-12 * np.abs(v["y"]).max()


def test_reader_rejects_bad_files(ib, tmp_path):
    src = os.path.join(PARTITIONS, "p3_9x7_2")
    info = os.path.join(src, "info.txt")
    good = os.path.join(src, "part_1.txt")
    with pytest.raises(ib.IgaError):
        ib.Part(info, good, 2)                     # wrong rank for this file
    with pytest.raises(ib.IgaError):
        ib.Part(info, good, 7)                     # rank outside the partition
    lines = open(good).read().split("\n")

    def variant(fn):
        path = str(tmp_path / "bad.txt")
        out = fn(list(lines))
        open(path, "w").write("\n".join(out))
        return path
    bad_count = variant(lambda L: ["nlocalfunc: 31"] + L[1:])
    gi = lines.index("ghostID") + 1
    swapped = lines[gi].split()
    swapped[0], swapped[1] = swapped[1], swapped[0]
    bad_ghost = variant(lambda L: L[:gi] + [" ".join(swapped)] + L[gi + 1:])
    ii = lines.index("IEN") + 1
    short_ien = variant(lambda L: L[:ii] + [" ".join(L[ii].split()[:-1])] + L[ii + 1:])
    no_cp = variant(lambda L: [x for k, x in enumerate(L) if k not in (lines.index("CP"), lines.index("CP") + 1)])
    for path in (bad_count, bad_ghost, short_ien, no_cp):
        with pytest.raises(ib.IgaError):
            ib.Part(info, path, 1)
    with pytest.raises(ib.IgaError):
        ib.Part(str(tmp_path / "missing_info.txt"), good, 1)


@pytest.mark.parametrize("name", CASES)
def test_test_writer_reproduces_reference_files(orc, name, tmp_path):
    """The test-only writer used for large GPU cases writes exactly the
    reference preprocessor's files."""
    import filecmp
    from iga_testlib import write_partition_files
    d, p, q, nex, ney, P = case_info(name)
    write_partition_files(unit_square_mesh(orc, p, q, nex, ney), P, str(tmp_path))
    for f in sorted(os.listdir(d)):
        if f.endswith(".txt"):
            assert filecmp.cmp(os.path.join(d, f), os.path.join(tmp_path, f), shallow=False), f


def local_oracle_spd(orc, part, sub, x_local):
    """The part's SPD MatMult with identity Dirichlet rows on the CPU: the
    local form of K (sign +1) with Dirichlet columns dropped, owned Dirichlet
    rows y = x, ghost Dirichlet rows 0 (the owner supplies the identity)."""
    xb = x_local[part.block_to_local].copy()
    xb[part.local_id[part.block_to_local] < 0] = 0.0
    yb = orc.apply_mf(sub, xb, sign=1.0, bc=2)
    y = np.empty_like(x_local)
    y[part.block_to_local] = yb
    dirl = part.local_id < 0
    y[dirl] = 0.0
    own = np.nonzero(dirl[:part.nowned])[0]
    y[own] = x_local[own]
    return y


def net_lengths(sub):
    """Mean polyline lengths of the control net's rows (x) and columns (y)."""
    m, n = sub["nex"] + sub["p"], sub["ney"] + sub["q"]
    cp = sub["CP"].reshape(n, m, 2)
    lx = np.linalg.norm(np.diff(cp, axis=1), axis=2).sum(axis=1).mean()
    ly = np.linalg.norm(np.diff(cp, axis=0), axis=2).sum(axis=0).mean()
    return lx, ly


def block_fem_solver(orc, sub):
    """CPU stand-in of the device's exact FEM inverse on a sub-patch: the
    dense FEM matrix of the sub-patch's FEM grid (identity boundary rows)."""
    lx, ly = net_lengths(sub)
    gx = orc.fem_nodes(sub["p"], sub["nex"], lx)
    gy = orc.fem_nodes(sub["q"], sub["ney"], ly)
    import scipy.linalg
    import torch
    nb = len(gx) * len(gy)
    lu = scipy.linalg.lu_factor(np.stack([orc.fem_matvec(gx, gy, e) for e in np.eye(nb)], axis=1))
    return lambda rb, zb: zb.copy_(torch.from_numpy(scipy.linalg.lu_solve(lu, rb.numpy())))


def serial_solution(orc, name, seed=21):
    """b (natural numbering, zero on the boundary) and the oracle's FP64 PCG
    solution of the SPD system, both in the partition numbering."""
    d, p, q, nex, ney, P = case_info(name)
    mesh = unit_square_mesh(orc, p, q, nex, ney)
    m, n = nex + p, ney + q
    b = splitmix_uniform(seed, -1.0, 1.0, m * n)
    mask = np.zeros((n, m), bool)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = True
    b[mask.ravel()] = 0.0
    x, it, rr = orc.pcg(mesh, b, rtol=1e-13, maxit=2000)
    new = partition_numbering(p, q, nex, ney, P)
    bp, xp = np.empty_like(b), np.empty_like(x)
    bp[new], xp[new] = b, x
    return bp, xp


def _gloo_pcg_rank(rank, world, port, name, pc, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from iga_testlib import Oracle
        import iga_b200 as ib
        from iga_dist import BlockFemPC, DistPartOperator, DistPCG, dist_fem_cg_pc
        orc = Oracle()
        d = os.path.join(PARTITIONS, name)
        part = ib.Part(os.path.join(d, "info.txt"), ib.partition_filename(os.path.join(d, "part"), rank), rank)
        sub = part.mesh()
        op = DistPartOperator(part, dist, "cpu",
                              local_apply=lambda xl, yl: yl.copy_(torch.from_numpy(
                                  local_oracle_spd(orc, part, sub, xl.numpy()))))
        if pc == "femcg":   # the reference's inner CG-Jacobi on the distributed FEM matrix
            prec = dist_fem_cg_pc(op)
        else:
            prec = BlockFemPC(part, "cpu", local_solve=block_fem_solver(orc, sub)) if pc else None
        bp = np.load(os.path.join(out_dir, "b.npy"))
        b_owned = torch.from_numpy(bp[part.owned_offset:part.owned_offset + part.nowned].copy())
        x_owned = torch.empty_like(b_owned)
        its, rel = DistPCG(op, prec).solve(b_owned, x_owned, rtol=1e-11)
        np.save(os.path.join(out_dir, f"x{rank}.npy"), x_owned.numpy())
        np.save(os.path.join(out_dir, f"its{rank}.npy"), np.array([its, rel]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,pc", [("p3_9x7_2", False), ("p3_9x7_2", True), ("p4_8x11_2", True),
                                     ("p3_9x7_2", "femcg")])
def test_gloo_distributed_pcg_matches_serial_solve(ib, orc, name, pc, tmp_path):
    """The multi-rank Krylov loop (one process per part, gloo): ghost updates,
    local element loops, two all-reductions per iteration, optional block FEM
    preconditioner or the reference's distributed inner FEM-CG; the assembled
    solution equals the serial FP64 solve and every rank agrees on the
    iteration count."""
    import torch.multiprocessing as mp
    d, p, q, nex, ney, P = case_info(name)
    world = P * P
    bp, xp = serial_solution(orc, name)
    np.save(os.path.join(tmp_path, "b.npy"), bp)
    mp.start_processes(_gloo_pcg_rank, args=(world, _free_port(), name, pc, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    x = np.concatenate([np.load(os.path.join(tmp_path, f"x{r}.npy")) for r in range(world)])
    its = [np.load(os.path.join(tmp_path, f"its{r}.npy")) for r in range(world)]
    assert len({int(i[0]) for i in its}) == 1 and its[0][1] <= 1e-11
    assert np.linalg.norm(x - xp) / np.linalg.norm(xp) < 1e-9


def owned_inside_blocks(parts, nfx, nfy):
    """Every owned entry lies off its block's outer ring unless it is on the
    global boundary (so each block preconditioner is an SPD principal block)."""
    for pt in parts:
        i = pt.info
        pos = np.empty(pt.nowned + pt.nghost, dtype=np.int64)
        pos[pt.block_to_local] = np.arange(len(pos))
        bi, bj = pos[:pt.nowned] % i.block_m, pos[:pt.nowned] // i.block_m
        ring = (bi == 0) | (bj == 0) | (bi == i.block_m - 1) | (bj == i.block_n - 1)
        gi, gj = i.elem_x0 + bi, i.elem_y0 + bj
        glob = (gi == 0) | (gj == 0) | (gi == nfx - 1) | (gj == nfy - 1)
        if np.any(ring & ~glob):
            return False
    return True


def emulated_solves(orc, parts, bp):
    import torch
    from iga_dist import BlockFemPC, emulate_partitioned_pcg
    subs = [pt.mesh() for pt in parts]

    def apply(part, xl, yl):
        yl.copy_(torch.from_numpy(local_oracle_spd(orc, part, subs[part.rank], xl.numpy())))
    x0, it0, _ = emulate_partitioned_pcg(parts, torch.from_numpy(bp), local_apply=apply, rtol=1e-11)
    pcs = [BlockFemPC(pt, "cpu", local_solve=block_fem_solver(orc, sub)) for pt, sub in zip(parts, subs)]
    x1, it1, _ = emulate_partitioned_pcg(parts, torch.from_numpy(bp), pcs=pcs, local_apply=apply, rtol=1e-11)
    return x0.numpy(), it0, x1.numpy(), it1


@pytest.mark.parametrize("name", CASES)
def test_emulated_pcg_matches_serial_solve(ib, orc, name):
    """All parts in one process, the same loop, with and without the block
    FEM preconditioner: the serial FP64 solution."""
    d, p, q, nex, ney, P = case_info(name)
    parts = open_parts(ib, name)
    assert owned_inside_blocks(parts, nex + p, ney + q)
    bp, xp = serial_solution(orc, name)
    x0, it0, x1, it1 = emulated_solves(orc, parts, bp)
    for x in (x0, x1):
        assert np.linalg.norm(x - xp) / np.linalg.norm(xp) < 1e-9


def test_emulated_pcg_block_pc_reduces_iterations(ib, orc, tmp_path):
    """p = 2, 64 x 64 elements on 2 x 2 parts (files written by the test
    restatement of the reference preprocessor): the block FEM preconditioner
    roughly halves the iteration count of the unpreconditioned loop."""
    p, ne, P = 2, 64, 2
    mesh = unit_square_mesh(orc, p, p, ne, ne)
    write_partition_files(mesh, P, str(tmp_path))
    parts = [ib.Part(os.path.join(tmp_path, "info.txt"), ib.partition_filename(os.path.join(tmp_path, "part"), r), r)
             for r in range(P * P)]
    m = ne + p
    assert owned_inside_blocks(parts, m, m)
    b = splitmix_uniform(21, -1.0, 1.0, m * m)
    mask = np.zeros((m, m), bool)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = True
    b[mask.ravel()] = 0.0
    new = partition_numbering(p, p, ne, ne, P)
    bp = np.empty_like(b)
    bp[new] = b
    x0, it0, x1, it1 = emulated_solves(orc, parts, bp)
    assert np.linalg.norm(x1 - x0) / np.linalg.norm(x0) < 1e-9
    assert it1 < 0.6 * it0


@pytest.mark.parametrize("name", CASES)
def test_fem_rows_equal_oracle_fem_matrix(ib, orc, name):
    """The rows each part owns of the FEM preconditioner matrix (nodes from
    iga_fem_nodes_1d and the part's info), applied to local forms gathered
    from a global vector: the oracle's assembled FEM matrix-vector product."""
    import torch
    from iga_dist import emulate_fem_cg_pc
    d, p, q, nex, ney, P = case_info(name)
    parts = open_parts(ib, name)
    m, n = nex + p, ney + q
    x = splitmix_uniform(5, -1.0, 1.0, m * n)
    y_ref = orc.fem_matvec(orc.fem_nodes(p, nex), orc.fem_nodes(q, ney), x)
    new = partition_numbering(p, q, nex, ney, P)
    xp = np.empty_like(x)
    xp[new] = x
    pc = emulate_fem_cg_pc(parts, "cpu")
    yp = torch.empty(m * n, dtype=torch.float64)
    pc.spmv(torch.from_numpy(xp), yp)
    y = yp.numpy()[new]
    assert np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref) < 1e-14


@pytest.mark.parametrize("name", CASES)
def test_emulated_pcg_fem_cg_pc_matches_oracle_pcg(ib, orc, name):
    """All parts in one process with the reference's preconditioner (inner
    Jacobi-CG to 1e-10 on the distributed FEM matrix): the serial FP64
    solution, in the iteration count of the oracle's single-patch PCG with
    the same preconditioner (within 2: its outer loop stops on the true
    residual)."""
    import torch
    from iga_dist import emulate_fem_cg_pc, emulate_partitioned_pcg
    d, p, q, nex, ney, P = case_info(name)
    parts = open_parts(ib, name)
    subs = [pt.mesh() for pt in parts]
    bp, xp = serial_solution(orc, name)

    def apply(part, xl, yl):
        yl.copy_(torch.from_numpy(local_oracle_spd(orc, part, subs[part.rank], xl.numpy())))
    pc = emulate_fem_cg_pc(parts, "cpu")
    x, its, rel = emulate_partitioned_pcg(parts, torch.from_numpy(bp), local_apply=apply, rtol=1e-11,
                                          pc_global=pc)
    assert rel <= 1e-11 and pc.last_iterations > 0
    assert np.linalg.norm(x.numpy() - xp) / np.linalg.norm(xp) < 1e-9
    new = partition_numbering(p, q, nex, ney, P)
    b = bp[new]
    _, it_ref, _ = orc.pcg(unit_square_mesh(orc, p, q, nex, ney), b, rtol=1e-11, maxit=500)
    assert it_ref > 0 and abs(its - it_ref) <= 2


@pytest.mark.parametrize("name", CASES)
def test_native_exchange_maps_match_python_maps(ib, name):
    """The device solver's exchange maps (iga_dist_exchange_maps, C++) equal
    build_exchange's (the maps the gloo / NCCL torch.distributed path uses) on
    the reference's own partition files: same peers, same ghost positions,
    same owned-local indices in the peers' ghost-list order."""
    from iga_dist import build_exchange
    parts = open_parts(ib, name)
    offsets = [pt.owned_offset for pt in parts] + [parts[-1].owned_offset + parts[-1].nowned]
    ghosts = [pt.ghosts for pt in parts]
    py = build_exchange(offsets, ghosts)
    for r in range(len(parts)):
        recv_count, recv_pos, send_count, send_idx = ib.dist_exchange_maps(r, offsets, ghosts)
        py_recv, py_send = py[r]
        want_pos = np.concatenate([py_recv[q] for q in sorted(py_recv)]) if py_recv else np.zeros(0, int)
        want_idx = np.concatenate([py_send[q] for q in sorted(py_send)]) if py_send else np.zeros(0, int)
        assert [int(recv_count[q]) for q in range(len(parts))] == [len(py_recv.get(q, [])) for q in range(len(parts))]
        assert [int(send_count[q]) for q in range(len(parts))] == [len(py_send.get(q, [])) for q in range(len(parts))]
        assert np.array_equal(recv_pos, want_pos)
        assert np.array_equal(send_idx, want_idx)


def test_native_exchange_maps_reject_unowned_ghosts(ib):
    with pytest.raises(Exception):
        ib.dist_exchange_maps(0, [0, 4, 8], [[9], []])   # entry 9 is nobody's
