"""Python binding (ctypes) of the C ABI in include/iga_mf.h, include/iga_solve.h,
include/iga_batch.h and include/iga_part.h.

A thin layer for tests, the benchmark and Python users: it loads the in-tree
libiga_b200.so (built by `make -C parallel-computing_b200`) and fails loudly if
it is missing. There is no fallback path: every operator call runs the CUDA
kernels of that library.

Device arrays are passed as torch CUDA tensors (or raw integer pointers);
torch is used only for device memory and streams.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libiga_b200.so")
# Tile shapes of the batched operator tuned on B200 for the 256-problem
# p in {2, 3}, 32..256-element batch (written by iga_batch_autotune).
TUNE_FILE = os.path.join(HERE, "tune_b200.json")
VP = ctypes.c_void_p

IGA_OK = 0
FP64, FP32, MIXED = 0, 1, 2
MIXED_PC = 3   # solve precision: FP64 PCG with the preconditioner in FP32
GEOM_PRECOMPUTED, GEOM_ON_THE_FLY = 0, 1
SIGN_REFERENCE, SIGN_SPD = -1, 1
BC_REFERENCE, BC_IDENTITY, BC_NONE = 0, 1, 2
F_REFERENCE, F_SINSIN, F_ANNULUS = 0, 1, 2


class IgaError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        super().__init__(f"{what}: {_lib().iga_status_str(status).decode()} ({status}): "
                         f"{_lib().iga_last_error().decode()}")


class MeshDesc(ctypes.Structure):
    _fields_ = [("p", ctypes.c_int), ("q", ctypes.c_int), ("nElemX", ctypes.c_int), ("nElemY", ctypes.c_int),
                ("CP", VP), ("weights", VP), ("C1", VP), ("C2", VP), ("h1", VP), ("h2", VP),
                ("IEN", VP), ("ID", VP), ("Dir", VP), ("nDir", ctypes.c_int), ("kappa", VP)]


class Opts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("geometry", ctypes.c_int), ("sign", ctypes.c_int),
                ("bc", ctypes.c_int), ("device", ctypes.c_int), ("rows_per_strip", ctypes.c_int)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("nfunc", ctypes.c_int64), ("nelem", ctypes.c_int64), ("geom_bytes", ctypes.c_int64),
                ("algo_bytes_f64", ctypes.c_int64), ("algo_bytes_f32", ctypes.c_int64),
                ("rows_per_strip", ctypes.c_int), ("warps_per_cta", ctypes.c_int)]


class SolveOpts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("pc", ctypes.c_int), ("rtol", ctypes.c_double),
                ("max_it", ctypes.c_int), ("pc_rtol", ctypes.c_double), ("pc_max_it", ctypes.c_int),
                ("sweep_rtol", ctypes.c_double), ("max_sweeps", ctypes.c_int), ("x0_nonzero", ctypes.c_int)]


class SolveStats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iterations", ctypes.c_int), ("pc_iterations", ctypes.c_int64),
                ("sweeps", ctypes.c_int), ("relres", ctypes.c_double), ("seconds", ctypes.c_double)]


class BatchOpts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("device", ctypes.c_int), ("tune_file", ctypes.c_char_p)]


class BatchStats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("converged", ctypes.c_int), ("max_iterations", ctypes.c_int),
                ("total_iterations", ctypes.c_int64), ("max_sweeps", ctypes.c_int),
                ("max_relres", ctypes.c_double), ("seconds", ctypes.c_double)]


class PartInfo(ctypes.Structure):
    _fields_ = [("p", ctypes.c_int), ("q", ctypes.c_int), ("nElemX", ctypes.c_int), ("nElemY", ctypes.c_int),
                ("part_num_1d", ctypes.c_int), ("dim", ctypes.c_int), ("Lx", ctypes.c_double),
                ("Ly", ctypes.c_double), ("rank", ctypes.c_int), ("part_x", ctypes.c_int), ("part_y", ctypes.c_int),
                ("nlocalfunc", ctypes.c_int), ("nghost", ctypes.c_int), ("nlocalelemx", ctypes.c_int),
                ("nlocalelemy", ctypes.c_int), ("elem_x0", ctypes.c_int), ("elem_y0", ctypes.c_int),
                ("block_m", ctypes.c_int), ("block_n", ctypes.c_int), ("owned_offset", ctypes.c_int64),
                ("nfunc_global", ctypes.c_int64)]


PC_NONE, PC_FEM_CG, PC_FEM_EXACT = 0, 1, 2

_LIB = None

# (name, restype, argtypes) of every exported C entry point.
SIGNATURES = [
    ("iga_status_str", ctypes.c_char_p, [ctypes.c_int]),
    ("iga_last_error", ctypes.c_char_p, []),
    ("iga_opts_default", None, [ctypes.POINTER(Opts)]),
    ("iga_mesh_unit_square", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, VP, VP, VP]),
    ("iga_mesh_quarter_annulus", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                ctypes.c_double, VP, VP, VP, VP]),
    ("iga_plan_create", ctypes.c_int, [ctypes.POINTER(MeshDesc), ctypes.POINTER(Opts), ctypes.POINTER(VP)]),
    ("iga_plan_destroy", ctypes.c_int, [VP]),
    ("iga_plan_get_info", ctypes.c_int, [VP, ctypes.POINTER(PlanInfo)]),
    ("iga_apply", ctypes.c_int, [VP, VP, VP, VP]),
    ("iga_apply_prec", ctypes.c_int, [VP, ctypes.c_int, VP, VP, VP]),
    ("iga_apply_host", ctypes.c_int, [VP, VP, VP]),
    ("iga_rhs", ctypes.c_int, [VP, ctypes.c_int, VP, VP]),
    ("iga_plan_device_status", ctypes.c_int, [VP, VP]),
    ("iga_plan_set_wait_limit", ctypes.c_int, [VP, ctypes.c_longlong]),
    ("iga_plan_set_pc_split", ctypes.c_int, [VP, ctypes.c_int]),
    ("iga_plan_set_solver_graph", ctypes.c_int, [VP, ctypes.c_int]),
    ("iga_MatrixFreeMatMultCUDA", ctypes.c_int, [ctypes.c_int] * 4 + [VP] * 15),
    ("iga_MatrixFreeMatMultCUDA_release", ctypes.c_int, []),
    ("iga_MatrixFreeMatMultCUDA_noalloc", ctypes.c_int, [ctypes.c_int] * 4 + [VP] * 16),
    ("iga_solve_opts_default", None, [ctypes.POINTER(SolveOpts)]),
    ("iga_solve", ctypes.c_int, [VP, VP, VP, ctypes.POINTER(SolveOpts), ctypes.POINTER(SolveStats), VP]),
    ("iga_fem_apply", ctypes.c_int, [VP, ctypes.c_int, VP, VP, VP]),
    ("iga_fem_assemble_csr", ctypes.c_int, [VP, ctypes.c_int, VP, VP, VP, ctypes.POINTER(ctypes.c_int64), VP]),
    ("iga_fem_nodes", ctypes.c_int, [VP, VP, VP]),
    ("iga_fem_nodes_1d", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, VP]),
    ("iga_pc_apply", ctypes.c_int, [VP, ctypes.c_int, ctypes.c_int, VP, VP, ctypes.c_double, ctypes.c_int, VP]),
    ("iga_plan_set_kappa", ctypes.c_int, [VP, VP, VP]),
    ("iga_adjoint_grad", ctypes.c_int, [VP, VP, VP, VP, VP]),
    ("iga_batch_opts_default", None, [ctypes.POINTER(BatchOpts)]),
    ("iga_batch_create", ctypes.c_int, [VP, ctypes.c_int, ctypes.POINTER(BatchOpts), ctypes.POINTER(VP)]),
    ("iga_batch_destroy", ctypes.c_int, [VP]),
    ("iga_batch_offsets", ctypes.c_int, [VP, VP]),
    ("iga_batch_plan", VP, [VP, ctypes.c_int]),
    ("iga_batch_shape", ctypes.c_int, [VP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    ("iga_batch_apply", ctypes.c_int, [VP, ctypes.c_int, VP, VP, VP]),
    ("iga_batch_pc_apply", ctypes.c_int, [VP, ctypes.c_int, ctypes.c_int, VP, VP, VP]),
    ("iga_batch_solve", ctypes.c_int, [VP, VP, VP, ctypes.POINTER(SolveOpts), ctypes.POINTER(BatchStats), VP, VP,
                                       VP]),
    ("iga_batch_autotune", ctypes.c_int, [VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p]),
    ("iga_tune_lookup", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("iga_spectrum_estimate", ctypes.c_int, [VP, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                             ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_int)]),
    ("iga_part_open", ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(VP)]),
    ("iga_part_close", ctypes.c_int, [VP]),
    ("iga_part_get_info", ctypes.c_int, [VP, ctypes.POINTER(PartInfo)]),
    ("iga_part_ghosts", ctypes.c_int, [VP, VP]),
    ("iga_part_block_map", ctypes.c_int, [VP, VP]),
    ("iga_part_local_id", ctypes.c_int, [VP, VP]),
    ("iga_part_mesh", ctypes.c_int, [VP, ctypes.POINTER(MeshDesc)]),
    ("iga_part_build", ctypes.c_int, [VP, ctypes.POINTER(Opts)]),
    ("iga_part_apply", ctypes.c_int, [VP, VP, VP, VP]),
    ("iga_dist_unique_id", ctypes.c_int, [VP]),
    ("iga_dist_comm_create", ctypes.c_int, [ctypes.c_int, ctypes.c_int, VP, ctypes.c_int, ctypes.POINTER(VP)]),
    ("iga_dist_comm_destroy", ctypes.c_int, [VP]),
    ("iga_dist_exchange_maps", ctypes.c_int, [ctypes.c_int, ctypes.c_int, VP, VP, VP, VP, VP, VP, VP,
                                              ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    ("iga_dist_create", ctypes.c_int, [VP, VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(VP)]),
    ("iga_dist_destroy", ctypes.c_int, [VP]),
    ("iga_dist_apply", ctypes.c_int, [VP, VP, VP, VP]),
    ("iga_dist_solve", ctypes.c_int, [VP, VP, VP, ctypes.POINTER(SolveOpts), ctypes.POINTER(SolveStats), VP]),
]


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(f"{LIBPATH} is missing: build it with `make -C {HERE}` "
                               "(there is no CPU fallback for the operator)")
        L = ctypes.CDLL(LIBPATH)
        for name, res, args in SIGNATURES:
            if hasattr(L, name):
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
        _LIB = L
    return _LIB


def lib():
    return _lib()


def _check(status, what):
    if status != IGA_OK:
        raise IgaError(status, what)


def _ptr(a):
    """Device/host pointer of a torch tensor, numpy array or int."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def fem_nodes_1d(p, ne, L):
    """ne + p node coordinates of one direction of the FEM preconditioner grid
    (iga_fem_nodes_1d; host only)."""
    g = np.empty(ne + p, dtype=np.float64)
    _check(_lib().iga_fem_nodes_1d(p, ne, float(L), g.ctypes.data_as(VP)), "iga_fem_nodes_1d")
    return g


def unit_square(p, nex, ney=None, Lx=1.0, Ly=1.0):
    """Patch arrays of the reference preprocessor (host numpy): dict(p, q, nex, ney, CP, C1, C2)."""
    ney = nex if ney is None else ney
    m, n = nex + p, ney + p
    CP = np.empty(2 * m * n)
    C1 = np.empty(nex * (p + 1) ** 2)
    C2 = np.empty(ney * (p + 1) ** 2)
    _check(_lib().iga_mesh_unit_square(p, nex, ney, Lx, Ly, _ptr(CP), _ptr(C1), _ptr(C2)),
           "iga_mesh_unit_square")
    return dict(p=p, q=p, nex=nex, ney=ney, CP=CP, C1=C1, C2=C2, W=None, kappa=None,
                h1=np.full(nex, Lx / nex), h2=np.full(ney, Ly / ney))


def quarter_annulus(p, nex, ney=None, r_in=1.0, r_out=2.0):
    """Exact NURBS quarter annulus (radial direction first): dict(p, q, nex, ney, CP, W, C1, C2)."""
    ney = nex if ney is None else ney
    m, n = nex + p, ney + p
    CP = np.empty(2 * m * n)
    W = np.empty(m * n)
    C1 = np.empty(nex * (p + 1) ** 2)
    C2 = np.empty(ney * (p + 1) ** 2)
    _check(_lib().iga_mesh_quarter_annulus(p, nex, ney, r_in, r_out, _ptr(CP), _ptr(W), _ptr(C1), _ptr(C2)),
           "iga_mesh_quarter_annulus")
    return dict(p=p, q=p, nex=nex, ney=ney, CP=CP, W=W, C1=C1, C2=C2, kappa=None,
                h1=np.full(nex, 1.0 / nex), h2=np.full(ney, 1.0 / ney))


def splitmix_uniform(seed, n, offset=0):
    """u53 in [0, 1) from the SplitMix64 counter stream (entries offset .. offset+n-1)."""
    i = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def splitmix_normal(seed, n, offset=0):
    """N(0,1) from the SplitMix64 counter stream (Box-Muller on consecutive
    pairs; offset counts pairs)."""
    m = (n + 1) // 2
    u = splitmix_uniform(seed, 2 * m, 2 * offset)
    r = np.sqrt(-2.0 * np.log(1.0 - u[0::2]))
    out = np.empty(2 * m)
    out[0::2] = r * np.cos(2 * np.pi * u[1::2])
    out[1::2] = r * np.sin(2 * np.pi * u[1::2])
    return out[:n]


def grf_qp(mesh, sigma=1.0, ell=0.1, seed=3):
    """Gaussian random field with squared-exponential covariance sigma^2
    exp(-|x-x'|^2 / (2 ell^2)) sampled at the quadrature points of a unit-square
    patch (element-major, qx fastest). The covariance is separable on the tensor
    grid of quadrature points, so g = sigma Lx Z Ly^T with Lx Lx^T = Kx from
    1-D eigendecompositions and Z ~ N(0,1) from the SplitMix64 stream."""
    p, nex, ney = mesh["p"], mesh["nex"], mesh["ney"]
    nq = p + 1
    t = np.polynomial.legendre.leggauss(nq)[0] * 0.5 + 0.5
    xs = ((np.arange(nex)[:, None] + t[None, :]) / nex).ravel()
    ys = ((np.arange(ney)[:, None] + t[None, :]) / ney).ravel()

    def factor(z):
        K = np.exp(-(z[:, None] - z[None, :]) ** 2 / (2 * ell * ell))
        w, V = np.linalg.eigh(K)
        return V * np.sqrt(np.clip(w, 0.0, None))

    Lx, Ly = factor(xs), factor(ys)
    Z = splitmix_normal(seed, len(ys) * len(xs)).reshape(len(ys), len(xs))
    G = sigma * (Ly @ Z @ Lx.T)          # G[b, a]: y point b, x point a
    G = G.reshape(ney, nq, nex, nq).transpose(0, 2, 1, 3)   # [ey][ex][qy][qx]
    return np.ascontiguousarray(G).ravel()


def _mesh_desc(mesh, keep, IEN=None, ID=None, Dir=None):
    """iga_mesh_desc of a mesh dict; the arrays it points to are appended to keep."""
    def arr(v, dt=np.float64):
        if v is None:
            return None
        a = np.ascontiguousarray(v, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    d = MeshDesc()
    d.p, d.q, d.nElemX, d.nElemY = mesh["p"], mesh.get("q", mesh["p"]), mesh["nex"], mesh["ney"]
    d.CP = arr(mesh["CP"])
    d.weights = arr(mesh.get("W"))
    d.C1 = arr(mesh.get("C1"))
    d.C2 = arr(mesh.get("C2"))
    d.h1 = arr(mesh.get("h1"))
    d.h2 = arr(mesh.get("h2"))
    d.IEN = arr(IEN, np.int32)
    d.ID = arr(ID, np.int32)
    d.Dir = arr(Dir, np.int32)
    d.nDir = 0 if Dir is None else len(Dir)
    d.kappa = arr(mesh.get("kappa"))
    return d


def batch_problems(count=256, seed=2, sizes=tuple(range(32, 257, 16)), degrees=(2, 3)):
    """Shapes of a batch of unit-square problems: per problem the degree and the
    element counts per direction, each drawn uniformly (SplitMix64 stream of
    `seed`: three draws per problem, degree, nElemX, nElemY). Returns a list of
    (p, nex, ney)."""
    u = splitmix_uniform(seed, 3 * count).reshape(count, 3)
    out = []
    for a, b, c in u:
        out.append((int(degrees[min(int(a * len(degrees)), len(degrees) - 1)]),
                    int(sizes[min(int(b * len(sizes)), len(sizes) - 1)]),
                    int(sizes[min(int(c * len(sizes)), len(sizes) - 1)])))
    return out


def batch_rhs(shapes, seed=2):
    """Concatenated right-hand sides: N(0,1) entries (SplitMix64 normal stream
    of `seed`, one contiguous slice per problem in batch order) with zeros on
    the boundary ring (homogeneous Dirichlet data)."""
    parts, off = [], 0
    for p, nex, ney in shapes:
        m, n = nex + p, ney + p
        b = splitmix_normal(seed, m * n, offset=off).reshape(n, m)
        off += (m * n + 1) // 2
        b[0, :] = b[-1, :] = 0.0
        b[:, 0] = b[:, -1] = 0.0
        parts.append(b.ravel())
    return np.concatenate(parts)


class Batch:
    """Owns an iga_batch: many independent unit-square-type problems solved together."""

    def __init__(self, meshes, precision=FP64, device=0, tune_file=None):
        L = _lib()
        keep = []
        descs = (MeshDesc * len(meshes))()
        for i, m in enumerate(meshes):
            descs[i] = _mesh_desc(m, keep)
        o = BatchOpts()
        L.iga_batch_opts_default(ctypes.byref(o))
        o.precision, o.device = precision, device
        o.tune_file = tune_file.encode() if tune_file else None
        h = VP()
        _check(L.iga_batch_create(descs, len(meshes), ctypes.byref(o), ctypes.byref(h)), "iga_batch_create")
        self.h = h
        self.count = len(meshes)
        self.precision = precision
        offs = np.empty(self.count + 1, dtype=np.int64)
        _check(L.iga_batch_offsets(h, _ptr(offs)), "iga_batch_offsets")
        self.offsets = offs
        self.ntot = int(offs[-1])

    def close(self):
        if getattr(self, "h", None):
            _lib().iga_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def plan_handle(self, i):
        return _lib().iga_batch_plan(self.h, i)

    def shape(self, i, precision=FP64):
        r, w = ctypes.c_int(), ctypes.c_int()
        _check(_lib().iga_batch_shape(self.h, i, precision, ctypes.byref(r), ctypes.byref(w)), "iga_batch_shape")
        return r.value, w.value

    def apply(self, x, y, precision=FP64, stream=None):
        _check(_lib().iga_batch_apply(self.h, precision, _ptr(x), _ptr(y), _stream(stream)), "iga_batch_apply")

    def pc_apply(self, r, z, pc=PC_FEM_EXACT, precision=FP64, stream=None):
        _check(_lib().iga_batch_pc_apply(self.h, pc, precision, _ptr(r), _ptr(z), _stream(stream)),
               "iga_batch_pc_apply")

    def solve(self, b, x, stream=None, check=True, **kw):
        """Solve every problem; returns (BatchStats, iterations[count], relres[count])."""
        o = SolveOpts()
        _lib().iga_solve_opts_default(ctypes.byref(o))
        o.pc = PC_FEM_EXACT
        for k, v in kw.items():
            setattr(o, k, v)
        st = BatchStats()
        its = np.zeros(self.count, dtype=np.int32)
        rel = np.zeros(self.count)
        status = _lib().iga_batch_solve(self.h, _ptr(b), _ptr(x), ctypes.byref(o), ctypes.byref(st), _ptr(its),
                                        _ptr(rel), _stream(stream))
        if check:
            _check(status, "iga_batch_solve")
        return st, its, rel


def partition_filename(base_name, rank):
    """<base_name>_<rank>.txt, the reference's partition file name."""
    return f"{base_name}_{rank}.txt"


class Part:
    """One part of a partitioned mesh read from the reference's files (info.txt
    and <base_name>_<rank>.txt). Host arrays: ghosts (partition numbering),
    block_to_local, local_id; mesh() gives the sub-patch. build() creates the
    device state; apply(x_local, y_local) is the part's ghosted MatMult."""

    def __init__(self, info_file, part_file, rank):
        h = VP()
        _check(_lib().iga_part_open(info_file.encode(), part_file.encode(), rank, ctypes.byref(h)), "iga_part_open")
        self.h = h
        info = PartInfo()
        _check(_lib().iga_part_get_info(h, ctypes.byref(info)), "iga_part_get_info")
        self.info = info
        self.rank = rank
        self.nowned, self.nghost = info.nlocalfunc, info.nghost
        self.owned_offset = int(info.owned_offset)
        self.ghosts = np.empty(info.nghost, dtype=np.int64)
        if info.nghost:
            _check(_lib().iga_part_ghosts(h, _ptr(self.ghosts)), "iga_part_ghosts")
        nl = info.nlocalfunc + info.nghost
        self.block_to_local = np.empty(nl, dtype=np.int32)
        _check(_lib().iga_part_block_map(h, _ptr(self.block_to_local)), "iga_part_block_map")
        self.local_id = np.empty(nl, dtype=np.int32)
        _check(_lib().iga_part_local_id(h, _ptr(self.local_id)), "iga_part_local_id")

    def mesh(self):
        """Sub-patch as a mesh dict (host copies)."""
        d = MeshDesc()
        _check(_lib().iga_part_mesh(self.h, ctypes.byref(d)), "iga_part_mesh")
        i = self.info
        m, n = i.block_m, i.block_n

        def arr(ptr, k):
            return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)), shape=(k,)).copy()
        return dict(p=i.p, q=i.q, nex=i.nlocalelemx, ney=i.nlocalelemy, CP=arr(d.CP, 2 * m * n),
                    C1=arr(d.C1, i.nlocalelemx * (i.p + 1) ** 2), C2=arr(d.C2, i.nlocalelemy * (i.q + 1) ** 2),
                    h1=arr(d.h1, i.nlocalelemx), h2=arr(d.h2, i.nlocalelemy), W=None, kappa=None)

    def build(self, sign=SIGN_REFERENCE, bc=BC_REFERENCE, geometry=GEOM_PRECOMPUTED, device=0):
        o = Opts()
        _lib().iga_opts_default(ctypes.byref(o))
        o.precision, o.geometry, o.sign, o.bc, o.device = FP64, geometry, sign, bc, device
        _check(_lib().iga_part_build(self.h, ctypes.byref(o)), "iga_part_build")
        return self

    def apply(self, x_local, y_local, stream=None):
        _check(_lib().iga_part_apply(self.h, _ptr(x_local), _ptr(y_local), _stream(stream)), "iga_part_apply")

    def close(self):
        if getattr(self, "h", None):
            _lib().iga_part_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dist_exchange_maps(rank, offsets, ghost_lists):
    """Exchange maps of one rank (host, include/iga_dist.h): returns
    (recv_count[nranks], recv_pos, send_count[nranks], send_idx)."""
    nranks = len(ghost_lists)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    counts = np.array([len(g) for g in ghost_lists], dtype=np.int32)
    ghosts = np.ascontiguousarray(np.concatenate([np.asarray(g, dtype=np.int64) for g in ghost_lists])
                                  if counts.sum() else np.zeros(1, np.int64))
    recv_count = np.zeros(nranks, np.int32)
    send_count = np.zeros(nranks, np.int32)
    recv_pos = np.zeros(max(1, counts[rank]), np.int32)
    send_idx = np.zeros(max(1, int(counts.sum())), np.int32)
    nsend = ctypes.c_int64()
    _check(_lib().iga_dist_exchange_maps(nranks, rank, _ptr(offsets), _ptr(counts), _ptr(ghosts), _ptr(recv_count),
                                         _ptr(recv_pos), _ptr(send_count), _ptr(send_idx), send_idx.size,
                                         ctypes.byref(nsend)), "iga_dist_exchange_maps")
    return recv_count, recv_pos[:counts[rank]], send_count, send_idx[:nsend.value]


class NcclComm:
    """An NCCL communicator made through the library (one rank per process and
    GPU): rank 0 calls unique_id() and shares the 128 bytes; every rank then
    constructs NcclComm(nranks, rank, uid, device)."""

    @staticmethod
    def unique_id():
        buf = ctypes.create_string_buffer(128)
        _check(_lib().iga_dist_unique_id(buf), "iga_dist_unique_id")
        return buf.raw

    def __init__(self, nranks, rank, uid, device=0):
        buf = ctypes.create_string_buffer(bytes(uid), 128)
        h = VP()
        _check(_lib().iga_dist_comm_create(nranks, rank, buf, device, ctypes.byref(h)), "iga_dist_comm_create")
        self.h, self.nranks, self.rank = h, nranks, rank

    def close(self):
        if getattr(self, "h", None):
            _lib().iga_dist_comm_destroy(self.h)
            self.h = None


class DistSolver:
    """The device-resident multi-rank MatMult and PCG of include/iga_dist.h
    over one opened (not yet built) Part per rank. comm: an NcclComm, or None
    for a single rank."""

    def __init__(self, part, comm=None, nranks=1, rank=0, device=0):
        h = VP()
        c = comm.h if comm is not None else None
        if comm is not None:
            nranks, rank = comm.nranks, comm.rank
        _check(_lib().iga_dist_create(part.h, c, nranks, rank, device, ctypes.byref(h)), "iga_dist_create")
        self.h, self.part = h, part
        self.nowned = part.nowned

    def apply(self, x_owned, y_owned, stream=None):
        _check(_lib().iga_dist_apply(self.h, _ptr(x_owned), _ptr(y_owned), _stream(stream)), "iga_dist_apply")

    def solve(self, b_owned, x_owned, stream=None, check=True, **kw):
        o = SolveOpts()
        _lib().iga_solve_opts_default(ctypes.byref(o))
        for k, v in kw.items():
            setattr(o, k, v)
        st = SolveStats()
        status = _lib().iga_dist_solve(self.h, _ptr(b_owned), _ptr(x_owned), ctypes.byref(o), ctypes.byref(st),
                                       _stream(stream))
        if check:
            _check(status, "iga_dist_solve")
        return st

    def close(self):
        if getattr(self, "h", None):
            _lib().iga_dist_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_autotune(meshes, tune_file, precision=FP64, device=0):
    """Times candidate tile shapes for these problems and merges the winners into tune_file."""
    keep = []
    descs = (MeshDesc * len(meshes))()
    for i, m in enumerate(meshes):
        descs[i] = _mesh_desc(m, keep)
    _check(_lib().iga_batch_autotune(descs, len(meshes), precision, device, tune_file.encode()),
           "iga_batch_autotune")


def tune_lookup(tune_file, p, precision, nex, ney):
    """(rows_per_strip, warps_per_cta) the tuning table gives (0 = no entry); host only."""
    r, w = ctypes.c_int(), ctypes.c_int()
    _check(_lib().iga_tune_lookup(tune_file.encode(), p, precision, nex, ney, ctypes.byref(r), ctypes.byref(w)),
           "iga_tune_lookup")
    return r.value, w.value


class Plan:
    """Owns an iga_plan (device tables, precomputed geometry)."""

    def __init__(self, mesh, precision=FP64, geometry=GEOM_PRECOMPUTED, sign=SIGN_REFERENCE,
                 bc=BC_REFERENCE, device=0, rows_per_strip=0, IEN=None, ID=None, Dir=None):
        L = _lib()
        self._keep = []
        d = _mesh_desc(mesh, self._keep, IEN, ID, Dir)
        o = Opts()
        L.iga_opts_default(ctypes.byref(o))
        o.precision, o.geometry, o.sign, o.bc, o.device, o.rows_per_strip = (
            precision, geometry, sign, bc, device, rows_per_strip)
        h = VP()
        _check(L.iga_plan_create(ctypes.byref(d), ctypes.byref(o), ctypes.byref(h)), "iga_plan_create")
        self.h = h
        self._keep = []
        self.mesh = mesh
        self.precision = precision
        info = PlanInfo()
        _check(L.iga_plan_get_info(h, ctypes.byref(info)), "iga_plan_get_info")
        self.info = info
        self.nfunc = info.nfunc

    def close(self):
        if getattr(self, "h", None):
            _lib().iga_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def apply(self, x, y, stream=None, precision=None):
        if precision is None:
            _check(_lib().iga_apply(self.h, _ptr(x), _ptr(y), _stream(stream)), "iga_apply")
        else:
            _check(_lib().iga_apply_prec(self.h, precision, _ptr(x), _ptr(y), _stream(stream)), "iga_apply_prec")

    def apply_host(self, x, y=None):
        x = np.ascontiguousarray(x, dtype=np.float64)
        if y is None:
            y = np.empty_like(x)
        _check(_lib().iga_apply_host(self.h, _ptr(x), _ptr(y)), "iga_apply_host")
        return y

    def rhs(self, F, fkind=F_REFERENCE, stream=None):
        _check(_lib().iga_rhs(self.h, fkind, _ptr(F), _stream(stream)), "iga_rhs")
        return F

    def device_status(self, stream=None):
        """Synchronises the stream and returns (and clears) the status the
        plan's kernels recorded (IGA_OK or e.g. IGA_ERR_TIMEOUT)."""
        return _lib().iga_plan_device_status(self.h, _stream(stream))

    def set_solver_graph(self, enable):
        """Profiling hook: 0 runs the solver's iterations from the host (kernel
        by kernel) instead of inside the conditional-loop graph."""
        _check(_lib().iga_plan_set_solver_graph(self.h, int(enable)), "iga_plan_set_solver_graph")

    def set_wait_limit(self, polls):
        """Test hook: polls per bounded wait of the MatMult kernel (< 0: default)."""
        _check(_lib().iga_plan_set_wait_limit(self.h, int(polls)), "iga_plan_set_wait_limit")

    def set_pc_split(self, enable):
        """Test hook: 0 makes the exact FEM preconditioner use full x
        transforms instead of the parity-split ones (drops the solver state)."""
        _check(_lib().iga_plan_set_pc_split(self.h, int(enable)), "iga_plan_set_pc_split")

    def solve(self, b, x, stream=None, check=True, **kw):
        """Solve K x = b (SPD form) on the device; keyword arguments set iga_solve_opts fields."""
        o = SolveOpts()
        _lib().iga_solve_opts_default(ctypes.byref(o))
        for k, v in kw.items():
            setattr(o, k, v)
        st = SolveStats()
        status = _lib().iga_solve(self.h, _ptr(b), _ptr(x), ctypes.byref(o), ctypes.byref(st), _stream(stream))
        if check:
            _check(status, "iga_solve")
        return st

    def fem_apply(self, x, y, precision=FP64, stream=None):
        _check(_lib().iga_fem_apply(self.h, precision, _ptr(x), _ptr(y), _stream(stream)), "iga_fem_apply")

    def pc_apply(self, r, z, pc=PC_FEM_EXACT, precision=FP64, pc_rtol=1e-10, pc_max_it=10000, stream=None):
        _check(_lib().iga_pc_apply(self.h, pc, precision, _ptr(r), _ptr(z), pc_rtol, pc_max_it, _stream(stream)),
               "iga_pc_apply")

    def set_kappa(self, kappa, stream=None):
        """Coefficient at the quadrature points (device tensor, element-major, qx fastest)."""
        _check(_lib().iga_plan_set_kappa(self.h, _ptr(kappa), _stream(stream)), "iga_plan_set_kappa")

    def adjoint_grad(self, u, lam, g, stream=None):
        _check(_lib().iga_adjoint_grad(self.h, _ptr(u), _ptr(lam), _ptr(g), _stream(stream)), "iga_adjoint_grad")
        return g

    def spectrum(self, pc=PC_FEM_EXACT, steps=200, seed=7):
        """(lam_min, lam_max, steps) of K (pc=PC_NONE) or M^-1 K on the free control points (Lanczos)."""
        lo, hi, k = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _check(_lib().iga_spectrum_estimate(self.h, pc, steps, seed, ctypes.byref(lo), ctypes.byref(hi),
                                            ctypes.byref(k)), "iga_spectrum_estimate")
        return lo.value, hi.value, k.value

    def fem_nodes(self):
        gx = np.empty(self.mesh["nex"] + self.mesh["p"])
        gy = np.empty(self.mesh["ney"] + self.mesh.get("q", self.mesh["p"]))
        _check(_lib().iga_fem_nodes(self.h, _ptr(gx), _ptr(gy)), "iga_fem_nodes")
        return gx, gy

    def fem_csr(self, sign=-1):
        """Device CSR of the FEM preconditioner matrix, returned as host numpy (rowptr, col, val)."""
        import torch
        nnz = ctypes.c_int64()
        _check(_lib().iga_fem_assemble_csr(self.h, sign, None, None, None, ctypes.byref(nnz), None), "csr nnz")
        rp = torch.empty(self.nfunc + 1, dtype=torch.int32, device="cuda")
        col = torch.empty(nnz.value, dtype=torch.int32, device="cuda")
        val = torch.empty(nnz.value, dtype=torch.float64, device="cuda")
        _check(_lib().iga_fem_assemble_csr(self.h, sign, _ptr(rp), _ptr(col), _ptr(val), ctypes.byref(nnz), None),
               "iga_fem_assemble_csr")
        torch.cuda.synchronize()
        return rp.cpu().numpy(), col.cpu().numpy(), val.cpu().numpy()


def kappa_solve_function():
    """torch.autograd.Function u = K(kappa)^-1 F (a thin test binding over
    iga_plan_set_kappa, iga_solve and iga_adjoint_grad): backward runs the
    adjoint solve K lambda = dL/du (lambda = 0 on the boundary) and returns
    dL/dkappa_q = -(grad lambda . grad u) JxW_q."""
    import torch

    class KappaSolve(torch.autograd.Function):
        @staticmethod
        def forward(ctx, kappa, plan, F, bmask, solve_kw):
            plan.set_kappa(kappa.detach().contiguous())
            u = torch.zeros_like(F)
            plan.solve(F, u, **solve_kw)
            ctx.plan, ctx.bmask, ctx.solve_kw = plan, bmask, solve_kw
            ctx.save_for_backward(kappa, u)
            return u

        @staticmethod
        def backward(ctx, grad_u):
            kappa, u = ctx.saved_tensors
            plan = ctx.plan
            plan.set_kappa(kappa.detach().contiguous())
            rhs = grad_u.contiguous().clone()
            rhs[ctx.bmask] = 0.0
            lam = torch.zeros_like(rhs)
            plan.solve(rhs, lam, **ctx.solve_kw)
            g = torch.empty_like(kappa)
            plan.adjoint_grad(u, lam, g)
            return g, None, None, None, None

    return KappaSolve
