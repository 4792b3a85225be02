"""Multi-rank MatMult over a partitioned mesh: one part per rank (one rank per
GPU), the ghost traffic of the reference's PETSc ghosted vectors done with
torch.distributed (NCCL between GPUs, gloo on CPU).

The reference's MatMult (matrix_free/src/GlobalAssemblyMF.cpp:141-210 on the
vectors of matrix_free/iteration_number_fempc_mf.cpp:62-72) is
    VecGhostUpdate(x, INSERT, FORWARD)     owners' values into every ghost copy
    element loop into y's local form       iga_part_apply (include/iga_part.h)
    VecAssembly(y)                         ghost contributions added to owners
    y[Dir] = 0                             done by iga_part_apply's local ID rule
The exchange here does the first and last steps: every rank learns once which
of its owned entries are ghosts of which peer (from all ranks' ghost lists);
a forward update sends owned values to the peers that hold them as ghosts, a
reverse update sends ghost contributions back, and each owner adds them peer
by peer in ascending rank order (a fixed summation order: bitwise
reproducible across runs).

The Krylov loop over those ranks (DistPCG) is the reference's KSPSolve across
MPI ranks (matrix_free/iteration_number_fempc_mf.cpp:193-233 and the
no-preconditioner driver beside it): flexible PCG on the owned entries, one
MatMult and two all-reductions per iteration ([p.q], then [r.r, r.z, r.z_old]
in one call). The preconditioner is none, BlockFemPC (each rank's exact FEM
inverse on its own block: a block-Jacobi preconditioner that needs no
communication) or FemCGPC, the reference's own: an inner Jacobi-preconditioned
CG to 1e-10 on the FEM matrix distributed over the ranks
(matrix_free/iteration_number_fempc_mf.cpp:11-17,210-224), one ghost update
and two all-reductions per inner iteration, its rows those of iga_fem_apply's
matrix (FemRows).
"""
import numpy as np


def build_exchange(offsets, ghost_lists):
    """Exchange maps of every rank from the owned ranges (offsets[r] ..
    offsets[r+1]-1 in the partition numbering) and every rank's ghost list.
    Returns, per rank r, (recv_pos, send_idx): recv_pos[q] = positions in r's
    ghost list of the ghosts q owns (ascending); send_idx[q] = owned-local
    indices of r's entries that q holds as ghosts, in q's ghost-list order."""
    offsets = np.asarray(offsets, dtype=np.int64)
    world = len(ghost_lists)
    owners = [np.searchsorted(offsets, np.asarray(g, dtype=np.int64), side="right") - 1 for g in ghost_lists]
    for r, (g, o) in enumerate(zip(ghost_lists, owners)):
        if len(g) and (o.min() < 0 or o.max() >= world or np.any(o == r)):
            raise ValueError(f"rank {r}: ghost outside the other ranks' owned ranges")
    plans = []
    for r in range(world):
        recv_pos, send_idx = {}, {}
        for q in range(world):
            if q == r:
                continue
            pos = np.nonzero(owners[r] == q)[0]
            if len(pos):
                recv_pos[q] = pos
            mine = np.asarray(ghost_lists[q], dtype=np.int64)[owners[q] == r]
            if len(mine):
                send_idx[q] = mine - offsets[r]
        plans.append((recv_pos, send_idx))
    return plans


class DistPartOperator:
    """y_owned = A x_owned for this rank's part (torch tensors on `device`).

    part: an iga_b200.Part (built); dist: torch.distributed with an initialised
    process group, one part per rank (rank r reads <base_name>_<r>.txt).
    local_apply(x_local, y_local) defaults to part.apply (the GPU kernels)."""

    def __init__(self, part, dist, device, local_apply=None):
        import torch
        self.torch, self.dist, self.device = torch, dist, device
        self.part = part
        self.local_apply = local_apply or part.apply
        world, rank = dist.get_world_size(), dist.get_rank()
        if part.rank != rank:
            raise ValueError("the part's rank differs from the process rank")
        mine = (part.owned_offset, part.nowned, part.ghosts.tolist())
        everyone = [None] * world
        dist.all_gather_object(everyone, mine)
        offsets = [e[0] for e in everyone] + [everyone[-1][0] + everyone[-1][1]]
        for r in range(world - 1):
            if offsets[r] + everyone[r][1] != offsets[r + 1]:
                raise ValueError("owned ranges are not contiguous in rank order")
        recv_pos, send_idx = build_exchange(offsets, [e[2] for e in everyone])[rank]
        self.recv_pos = {q: torch.as_tensor(v, device=device) for q, v in recv_pos.items()}
        self.send_idx = {q: torch.as_tensor(v, device=device) for q, v in send_idx.items()}
        self.nowned = part.nowned
        self.x_local = torch.zeros(part.nowned + part.nghost, dtype=torch.float64, device=device)
        self.y_local = torch.empty_like(self.x_local)

    def _exchange(self, sends, recv_sizes):
        """Point-to-point exchange: sends {peer: tensor}, receives {peer: size}."""
        torch, dist = self.torch, self.dist
        recvs = {q: torch.empty(n, dtype=torch.float64, device=self.device) for q, n in recv_sizes.items()}
        ops = [dist.P2POp(dist.isend, t.contiguous(), q) for q, t in sorted(sends.items())]
        ops += [dist.P2POp(dist.irecv, t, q) for q, t in sorted(recvs.items())]
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        return recvs

    def forward_update(self, x_owned):
        """x_local = [x_owned | ghost values from their owners]."""
        self.x_local[:self.nowned] = x_owned
        got = self._exchange({q: x_owned[i] for q, i in self.send_idx.items()},
                             {q: len(p) for q, p in self.recv_pos.items()})
        for q, buf in got.items():
            self.x_local[self.nowned + self.recv_pos[q]] = buf
        return self.x_local

    def reverse_add(self, y_local, y_owned):
        """y_owned = owned rows of y_local + the peers' ghost contributions (ascending peer order)."""
        y_owned.copy_(y_local[:self.nowned])
        got = self._exchange({q: y_local[self.nowned + p] for q, p in self.recv_pos.items()},
                             {q: len(i) for q, i in self.send_idx.items()})
        for q in sorted(got):
            y_owned.index_add_(0, self.send_idx[q], got[q])
        return y_owned

    def matmult(self, x_owned, y_owned):
        x_local = self.forward_update(x_owned)
        self.local_apply(x_local, self.y_local)
        return self.reverse_add(self.y_local, y_owned)


def emulate_partitioned_matmult(parts, x_global, local_apply=None):
    """All parts of a partitioned mesh in one process (for a single GPU, or on
    CPU): the same maps and summation order as DistPartOperator, with the
    transfers done in memory. x_global in the partition numbering (torch
    tensor); returns y_global."""
    import torch
    offsets = [p.owned_offset for p in parts] + [parts[-1].owned_offset + parts[-1].nowned]
    plans = build_exchange(offsets, [p.ghosts for p in parts])
    dev = x_global.device
    y_locals = []
    for p, (recv_pos, _) in zip(parts, plans):
        x_local = torch.empty(p.nowned + p.nghost, dtype=torch.float64, device=dev)
        x_local[:p.nowned] = x_global[p.owned_offset:p.owned_offset + p.nowned]
        if p.nghost:
            x_local[p.nowned:] = x_global[torch.as_tensor(p.ghosts, device=dev)]
        y_local = torch.empty_like(x_local)
        (local_apply or (lambda part, a, b: part.apply(a, b)))(p, x_local, y_local)
        y_locals.append(y_local)
    y_global = torch.empty_like(x_global)
    for r, (p, (_, send_idx)) in enumerate(zip(parts, plans)):
        y_owned = y_locals[r][:p.nowned].clone()
        for q in sorted(send_idx):
            recv_pos_q = plans[q][0][r]
            contrib = y_locals[q][parts[q].nowned + torch.as_tensor(recv_pos_q, device=dev)]
            y_owned.index_add_(0, torch.as_tensor(send_idx[q], device=dev), contrib)
        y_global[p.owned_offset:p.owned_offset + p.nowned] = y_owned
    return y_global


def pcg_solve(matmult, pc, allreduce, b, x, rtol=1e-10, max_it=10000):
    """Flexible (Polak-Ribiere) PCG on K x = b from x = 0 over vectors that may
    be one rank's owned entries. matmult(v, out) computes out = K v (all ranks
    together); pc(r, out) applies the preconditioner (None: identity);
    allreduce(t) sums a small FP64 tensor over the ranks in place. Stops when
    ||r|| <= rtol ||b|| (recurrence residual). Returns (iterations, ||r|| / ||b||)."""
    import torch
    x.zero_()
    r = b.clone()
    z = torch.empty_like(b)
    q = torch.empty_like(b)

    def precond(v, out):
        if pc is None:
            out.copy_(v)
        else:
            pc(v, out)
    precond(r, z)
    d = torch.stack([torch.dot(b, b), torch.dot(r, r), torch.dot(r, z)])
    allreduce(d)
    bb, rr, rz = (float(v) for v in d)
    bnorm = bb ** 0.5
    if bnorm == 0.0:
        return 0, 0.0
    p = z.clone()
    it = 0
    while rr ** 0.5 > rtol * bnorm and it < max_it:
        matmult(p, q)
        d = torch.dot(p, q).reshape(1)
        allreduce(d)
        pq = float(d[0])
        if not pq > 0.0:
            raise FloatingPointError("PCG breakdown: p.Kp <= 0")
        alpha = rz / pq
        x.add_(p, alpha=alpha)
        r.add_(q, alpha=-alpha)
        rzo = torch.dot(r, z)
        precond(r, z)
        d = torch.stack([torch.dot(r, r), torch.dot(r, z), rzo])
        allreduce(d)
        rr, rz_new, rzo = (float(v) for v in d)
        it += 1
        beta = (rz_new - rzo) / rz
        rz = rz_new
        p.mul_(beta).add_(z)
    return it, rr ** 0.5 / bnorm


class BlockFemPC:
    """z_owned = [Kf^-1 (r_owned placed in the part's block, zero elsewhere)]_owned:
    Kf is the FEM matrix of the part's sub-patch (identity rows on the block's
    outer ring), inverted exactly by the device's fast-diagonalisation
    preconditioner (iga_pc_apply with IGA_PC_FEM_EXACT on a plan of the
    sub-patch). The owned entries of an interior part lie inside its block, so
    every rank applies a principal submatrix of an SPD inverse: the global
    preconditioner is block diagonal and SPD. local_solve(r_block, z_block)
    replaces the device solve (the host tests use a CPU stand-in)."""

    def __init__(self, part, device, local_solve=None):
        import torch
        nl = part.nowned + part.nghost
        pos = np.empty(nl, dtype=np.int64)
        pos[part.block_to_local] = np.arange(nl)
        self.pos = torch.as_tensor(pos[:part.nowned], device=device)
        self.rb = torch.zeros(nl, dtype=torch.float64, device=device)
        self.zb = torch.empty_like(self.rb)
        self.plan = None
        if local_solve is None:
            import iga_b200 as ib
            dev = torch.device(device)
            self.plan = ib.Plan(part.mesh(), device=dev.index or 0)
            plan = self.plan
            local_solve = lambda rb, zb: plan.pc_apply(rb, zb, pc=ib.PC_FEM_EXACT)  # noqa: E731
        self.local_solve = local_solve

    def __call__(self, r_owned, z_owned):
        self.rb.zero_()
        self.rb[self.pos] = r_owned
        self.local_solve(self.rb, self.zb)
        z_owned.copy_(self.zb[self.pos])


def _fem_1d(g):
    """Diagonals of the 1-D linear-element stiffness (kd, ko) and mass (md, mo)
    matrices on nodes g (2-point Gauss, exact), as the device preconditioner
    builds them."""
    h = np.diff(g)
    kd, md = np.zeros(len(g)), np.zeros(len(g))
    kd[:-1] += 1.0 / h
    kd[1:] += 1.0 / h
    md[:-1] += h / 3.0
    md[1:] += h / 3.0
    ko, mo = np.zeros(len(g)), np.zeros(len(g))
    ko[:-1], mo[:-1] = -1.0 / h, h / 6.0
    return kd, ko, md, mo


class FemRows:
    """The rows a part owns of the patch's FEM preconditioner matrix: bilinear
    elements on the tensor grid of FEM nodes, K = Kx (x) My + Mx (x) Ky on free
    rows with the boundary columns dropped, identity rows on the patch
    boundary (the matrix of iga_fem_apply / iga_fem_assemble_csr, reference
    matrix_free/src/ElementFEM.cpp:3-117 with the SPD sign). Nine (column,
    value) pairs per owned entry, columns in the part's local form (owned |
    ghosts): apply(x_local) needs x_local's ghosts current. gx, gy: the
    patch's 1-D nodes (default: iga_fem_nodes_1d from the part's info)."""

    def __init__(self, part, device, gx=None, gy=None):
        import torch
        i = part.info
        m, n = i.nElemX + i.p, i.nElemY + i.q
        if gx is None or gy is None:
            import iga_b200 as ib
            gx, gy = ib.fem_nodes_1d(i.p, i.nElemX, i.Lx), ib.fem_nodes_1d(i.q, i.nElemY, i.Ly)
        gx, gy = np.asarray(gx, dtype=np.float64), np.asarray(gy, dtype=np.float64)
        if len(gx) != m or len(gy) != n:
            raise ValueError("FEM node arrays do not match the patch")
        kd, ko, md, mo = _fem_1d(gx)
        ld, lo, nd, no = _fem_1d(gy)
        nl = part.nowned + part.nghost
        pos = np.empty(nl, dtype=np.int64)
        pos[part.block_to_local] = np.arange(nl)
        own = np.arange(part.nowned)
        bi, bj = pos[own] % i.block_m, pos[own] // i.block_m
        gi, gj = i.elem_x0 + bi, i.elem_y0 + bj
        free = (gi > 0) & (gj > 0) & (gi < m - 1) & (gj < n - 1)
        cols = np.repeat(own[:, None], 9, axis=1)
        vals = np.zeros((part.nowned, 9))
        vals[~free, 4] = 1.0
        gif, gjf = gi[free], gj[free]
        kx = [ko[gif - 1], kd[gif], ko[gif]]
        mx = [mo[gif - 1], md[gif], mo[gif]]
        ky = [lo[gjf - 1], ld[gjf], lo[gjf]]
        my = [no[gjf - 1], nd[gjf], no[gjf]]
        for b in range(3):
            for a in range(3):
                k = 3 * b + a
                ii, jj = gif + a - 1, gjf + b - 1
                use = (ii >= 1) & (ii <= m - 2) & (jj >= 1) & (jj <= n - 2)
                ci, cj = bi[free] + a - 1, bj[free] + b - 1
                inside = (ci >= 0) & (ci < i.block_m) & (cj >= 0) & (cj < i.block_n)
                if np.any(use & ~inside):
                    raise ValueError("a FEM neighbour of an owned entry lies outside the part's block")
                c = np.where(use, part.block_to_local[np.clip(cj, 0, i.block_n - 1) * i.block_m
                                                      + np.clip(ci, 0, i.block_m - 1)], own[free])
                cols[free, k] = c
                vals[free, k] = np.where(use, kx[a] * my[b] + mx[a] * ky[b], 0.0)
        self.cols = torch.as_tensor(cols, device=device)
        self.vals = torch.as_tensor(vals, device=device)
        self.diag = self.vals[:, 4].clone()

    def apply(self, x_local, y_owned):
        """y_owned = the owned rows of K times the local form x_local."""
        y_owned.copy_((self.vals * x_local[self.cols]).sum(dim=1))
        return y_owned


class FemCGPC:
    """z = K_fem^-1 r by Jacobi-preconditioned CG to ||res|| <= rtol ||r|| from
    z = 0 (the reference's PCSHELL: KSPCG + PCJACOBI on the FEM matrix,
    rtol 1e-10, matrix_free/iteration_number_fempc_mf.cpp:11-17,210-224),
    over vectors that may be one rank's owned entries. spmv(v, out): out = K v
    (all ranks together); diag: K's diagonal (owned entries); allreduce(t)
    sums a small FP64 tensor over the ranks in place. last_iterations: the
    inner iterations of the last apply."""

    def __init__(self, spmv, diag, allreduce, rtol=1e-10, max_it=10000):
        self.spmv, self.diag, self.allreduce = spmv, diag, allreduce
        self.rtol, self.max_it = rtol, max_it
        self.last_iterations = 0

    def __call__(self, r, z):
        import torch
        z.zero_()
        res = r.clone()
        w = res / self.diag
        p = w.clone()
        q = torch.empty_like(r)
        d = torch.stack([torch.dot(res, res), torch.dot(res, w)])
        self.allreduce(d)
        rr, rz = (float(v) for v in d)
        tol2 = self.rtol * self.rtol * rr
        it = 0
        while rr > tol2 and it < self.max_it:
            self.spmv(p, q)
            d = torch.dot(p, q).reshape(1)
            self.allreduce(d)
            if not float(d[0]) > 0.0:
                raise FloatingPointError("inner FEM-CG breakdown: p.Kp <= 0")
            alpha = rz / float(d[0])
            z.add_(p, alpha=alpha)
            res.add_(q, alpha=-alpha)
            torch.div(res, self.diag, out=w)
            d = torch.stack([torch.dot(res, res), torch.dot(res, w)])
            self.allreduce(d)
            rr, rz_new = (float(v) for v in d)
            p.mul_(rz_new / rz).add_(w)
            rz = rz_new
            it += 1
        self.last_iterations = it
        return z


def dist_fem_cg_pc(op, rtol=1e-10, max_it=10000, gx=None, gy=None):
    """FemCGPC over the ranks of op (a DistPartOperator): the FEM rows of op's
    part, ghost updates through op's exchange, all-reductions on op's group."""
    fem = FemRows(op.part, op.device, gx, gy)
    dist = op.dist

    def spmv(v, out):
        fem.apply(op.forward_update(v), out)

    def allreduce(t):
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return FemCGPC(spmv, fem.diag, allreduce, rtol, max_it)


def emulate_fem_cg_pc(parts, device, rtol=1e-10, max_it=10000, gx=None, gy=None):
    """FemCGPC with every part in one process, on the concatenated owned
    vectors (partition numbering): each part's rows applied to its local form
    gathered from the global vector."""
    import torch
    fems = [FemRows(pt, device, gx, gy) for pt in parts]
    ghosts = [torch.as_tensor(pt.ghosts, device=device) for pt in parts]
    diag = torch.cat([f.diag for f in fems])

    def spmv(v, out):
        for pt, f, g in zip(parts, fems, ghosts):
            o = pt.owned_offset
            x_local = torch.cat([v[o:o + pt.nowned], v[g]])
            f.apply(x_local, out[o:o + pt.nowned])
    return FemCGPC(spmv, diag, lambda t: None, rtol, max_it)


class DistPCG:
    """Flexible PCG on K x = b over the ranks of a partitioned mesh: op is a
    DistPartOperator whose part was built with sign SPD and bc IDENTITY (so K
    is SPD with identity Dirichlet rows; b must be zero on them); pc is None
    or a callable on owned vectors (BlockFemPC)."""

    def __init__(self, op, pc=None):
        self.op, self.pc = op, pc

    def solve(self, b_owned, x_owned, rtol=1e-10, max_it=10000):
        dist = self.op.dist

        def allreduce(t):
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return pcg_solve(self.op.matmult, self.pc, allreduce, b_owned, x_owned, rtol, max_it)


def emulate_partitioned_pcg(parts, b_global, pcs=None, local_apply=None, rtol=1e-10, max_it=10000, pc_global=None):
    """DistPCG with every part in one process (one GPU, or the CPU): the same
    operator, preconditioner and loop on the concatenated owned vectors
    (partition numbering). pcs: None or one preconditioner per part;
    pc_global: a preconditioner of the whole vector (emulate_fem_cg_pc)
    instead. Returns (x_global, iterations, relres)."""
    import torch
    off = [p.owned_offset for p in parts] + [parts[-1].owned_offset + parts[-1].nowned]

    def matmult(v, out):
        out.copy_(emulate_partitioned_matmult(parts, v, local_apply=local_apply))

    pc = pc_global
    if pcs is not None:
        def pc(v, out):
            for k, f in enumerate(pcs):
                f(v[off[k]:off[k + 1]], out[off[k]:off[k + 1]])
    x = torch.zeros_like(b_global)
    its, rel = pcg_solve(matmult, pc, lambda t: None, b_global, x, rtol, max_it)
    return x, its, rel
