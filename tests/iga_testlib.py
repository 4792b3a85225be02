"""Shared helpers for the tests: seeded inputs, and ctypes access to the CPU oracle.

The oracle (oracle/liboracle.so) is the checker only; the product path is the
CUDA library reached through include/iga_mf.h.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "ref_vectors.npz")
VP = ctypes.c_void_p
_GOLD = 0x9E3779B97F4A7C15
_M64 = (1 << 64) - 1


def _mix64(z):
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def splitmix_u53(seed, n, offset=0):
    """u53 of the SplitMix64 counter stream (identical to the oracle's orc_uniform)."""
    i = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed & _M64) + i * np.uint64(_GOLD)
        z = _mix64(z)
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def splitmix_uniform(seed, lo, hi, n):
    return lo + (hi - lo) * splitmix_u53(seed, n)


def splitmix_normal(seed, n):
    m = (n + 1) // 2
    u = splitmix_u53(seed, 2 * m)
    a, b = u[0::2], u[1::2]
    r = np.sqrt(-2.0 * np.log(1.0 - a))
    out = np.empty(2 * m)
    out[0::2] = r * np.cos(2 * np.pi * b)
    out[1::2] = r * np.sin(2 * np.pi * b)
    return out[:n]


def _p(a):
    return a.ctypes.data_as(VP)


class OrcPatch(ctypes.Structure):
    _fields_ = [("p", ctypes.c_int), ("q", ctypes.c_int), ("nex", ctypes.c_int), ("ney", ctypes.c_int),
                ("CP", VP), ("W", VP), ("C1", VP), ("C2", VP), ("h1", VP), ("h2", VP), ("kappa", VP)]


class Oracle:
    """ctypes view of oracle/liboracle.so (built by `make -C oracle`)."""

    def __init__(self):
        path = os.path.join(ROOT, "oracle", "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
        self.L = ctypes.CDLL(path)
        self.L.orc_uniform.argtypes = [ctypes.c_uint64, ctypes.c_double, ctypes.c_double, VP, ctypes.c_long]
        self.L.orc_normal.argtypes = [ctypes.c_uint64, VP, ctypes.c_long]
        self.L.orc_gauss01.argtypes = [ctypes.c_int, VP, VP]
        self.L.orc_bernstein.argtypes = [ctypes.c_int, ctypes.c_double, VP, VP]
        self.L.orc_open_knots.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, VP]
        self.L.orc_extraction.argtypes = [ctypes.c_int, VP, ctypes.c_int, VP]
        self.L.orc_greville.argtypes = [ctypes.c_int, VP, ctypes.c_int, VP]
        self.L.orc_apply_mf.argtypes = [ctypes.POINTER(OrcPatch), VP, VP, ctypes.c_double, ctypes.c_int]
        self.L.orc_apply_sf.argtypes = [ctypes.POINTER(OrcPatch), VP, VP, ctypes.c_double]
        self.L.orc_rhs.argtypes = [ctypes.POINTER(OrcPatch), ctypes.c_int, VP]
        self.L.orc_adjoint_grad.argtypes = [ctypes.POINTER(OrcPatch), VP, VP, VP]
        self.L.orc_qp_points.argtypes = [ctypes.POINTER(OrcPatch), VP, VP]
        self.L.orc_eval_qp.argtypes = [ctypes.POINTER(OrcPatch), VP, VP]
        self.L.orc_fem_nodes.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, VP]
        self.L.orc_fem_matvec.argtypes = [ctypes.c_int, ctypes.c_int, VP, VP, VP, VP, ctypes.c_double]
        self.L.orc_pcg.argtypes = [ctypes.POINTER(OrcPatch), VP, VP, VP, VP, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]

    def uniform(self, seed, lo, hi, n):
        out = np.empty(n)
        self.L.orc_uniform(seed, lo, hi, _p(out), n)
        return out

    def normal(self, seed, n):
        out = np.empty(n)
        self.L.orc_normal(seed, _p(out), n)
        return out

    def gauss01(self, n):
        x, w = np.empty(n), np.empty(n)
        self.L.orc_gauss01(n, _p(x), _p(w))
        return x, w

    def bernstein(self, p, xi):
        B, dB = np.empty(p + 1), np.empty(p + 1)
        self.L.orc_bernstein(p, xi, _p(B), _p(dB))
        return B, dB

    def open_knots(self, p, ne, L=1.0):
        S = np.empty(ne + 2 * p + 1)
        self.L.orc_open_knots(p, ne, L, _p(S))
        return S

    def extraction(self, p, S):
        S = np.ascontiguousarray(S, dtype=np.float64)
        C = np.zeros(max(1, len(S) - 2 * p - 1) * (p + 1) ** 2)
        ne = self.L.orc_extraction(p, _p(S), len(S), _p(C))
        return C[: ne * (p + 1) ** 2].copy()

    def greville(self, p, S):
        S = np.ascontiguousarray(S, dtype=np.float64)
        g = np.empty(len(S) - p - 1)
        self.L.orc_greville(p, _p(S), len(S), _p(g))
        return g

    def patch(self, mesh):
        """mesh: dict with p, q, nex, ney, CP, C1, C2, h1, h2 and optional W, kappa."""
        keep = {k: np.ascontiguousarray(mesh[k], dtype=np.float64) for k in ("CP", "C1", "C2", "h1", "h2")}
        for k in ("W", "kappa"):
            keep[k] = None if mesh.get(k) is None else np.ascontiguousarray(mesh[k], dtype=np.float64)
        P = OrcPatch(mesh["p"], mesh["q"], mesh["nex"], mesh["ney"], _p(keep["CP"]),
                     None if keep["W"] is None else _p(keep["W"]), _p(keep["C1"]), _p(keep["C2"]),
                     _p(keep["h1"]), _p(keep["h2"]), None if keep["kappa"] is None else _p(keep["kappa"]))
        P._keep = keep
        return P

    def apply_mf(self, mesh, x, sign=-1.0, bc=0):
        P = self.patch(mesh)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self.L.orc_apply_mf(ctypes.byref(P), _p(x), _p(y), sign, bc)
        return y

    def apply_sf(self, mesh, x, sign=-1.0):
        P = self.patch(mesh)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self.L.orc_apply_sf(ctypes.byref(P), _p(x), _p(y), sign)
        return y

    def rhs(self, mesh, fkind):
        P = self.patch(mesh)
        F = np.empty((mesh["nex"] + mesh["p"]) * (mesh["ney"] + mesh["q"]))
        self.L.orc_rhs(ctypes.byref(P), fkind, _p(F))
        return F

    def qp_points(self, mesh):
        P = self.patch(mesh)
        nq = mesh["nex"] * mesh["ney"] * (mesh["p"] + 1) * (mesh["q"] + 1)
        xy, jw = np.empty(2 * nq), np.empty(nq)
        self.L.orc_qp_points(ctypes.byref(P), _p(xy), _p(jw))
        return xy.reshape(-1, 2), jw

    def eval_qp(self, mesh, u):
        P = self.patch(mesh)
        vals = np.empty(mesh["nex"] * mesh["ney"] * (mesh["p"] + 1) * (mesh["q"] + 1))
        u = np.ascontiguousarray(u, dtype=np.float64)
        self.L.orc_eval_qp(ctypes.byref(P), _p(u), _p(vals))
        return vals

    def adjoint_grad(self, mesh, u, lam):
        P = self.patch(mesh)
        g = np.empty(mesh["nex"] * mesh["ney"] * (mesh["p"] + 1) * (mesh["q"] + 1))
        u = np.ascontiguousarray(u, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        self.L.orc_adjoint_grad(ctypes.byref(P), _p(u), _p(lam), _p(g))
        return g

    def fem_nodes(self, p, ne, L=1.0):
        g = np.empty(ne + p)
        self.L.orc_fem_nodes(p, ne, L, _p(g))
        return g

    def fem_matvec(self, gx, gy, x, sign=1.0):
        gx = np.ascontiguousarray(gx, dtype=np.float64)
        gy = np.ascontiguousarray(gy, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self.L.orc_fem_matvec(len(gx), len(gy), _p(gx), _p(gy), _p(x), _p(y), sign)
        return y

    def pcg(self, mesh, b, rtol=1e-10, maxit=500, inner_rtol=1e-10, inner_maxit=10000):
        P = self.patch(mesh)
        gx = self.fem_nodes(mesh["p"], mesh["nex"])
        gy = self.fem_nodes(mesh["q"], mesh["ney"])
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        rr = ctypes.c_double()
        it = self.L.orc_pcg(ctypes.byref(P), _p(gx), _p(gy), _p(b), _p(x), rtol, maxit, inner_rtol,
                            inner_maxit, ctypes.byref(rr))
        return x, it, rr.value


def unit_square_mesh(orc, p, q, nex, ney, Lx=1.0, Ly=1.0):
    """Unit-square patch of the reference preprocessor, built with the oracle."""
    S = orc.open_knots(p, nex, Lx)
    T = orc.open_knots(q, ney, Ly)
    gx, gy = orc.greville(p, S), orc.greville(q, T)
    X, Y = np.meshgrid(gx, gy)
    CP = np.stack([X.ravel(), Y.ravel()], axis=1).ravel()
    return dict(p=p, q=q, nex=nex, ney=ney, CP=CP, C1=orc.extraction(p, S), C2=orc.extraction(q, T),
                h1=np.full(nex, Lx / nex), h2=np.full(ney, Ly / ney), W=None, kappa=None)


def boundary_mask(m, n):
    mask = np.zeros((n, m), bool)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = True
    return mask.ravel()


def golden():
    return np.load(GOLDEN)


def golden_mesh(g, name):
    p, q, nex, ney = (int(v) for v in g[f"{name}_dims"])
    return dict(p=p, q=q, nex=nex, ney=ney, CP=g[f"{name}_CP"], C1=g[f"{name}_C1"], C2=g[f"{name}_C2"],
                h1=g[f"{name}_h1"], h2=g[f"{name}_h2"], W=None, kappa=None)


def load_binding():
    import sys
    pkg = os.path.join(ROOT, "parallel-computing_b200")
    if pkg not in sys.path:
        sys.path.insert(0, pkg)
    import iga_b200
    return iga_b200


def distorted(mesh, ax=0.01, ay=0.02):
    """Smoothly distorted copy of a unit-square patch (non-affine geometry)."""
    p, nex, ney = mesh["p"], mesh["nex"], mesh["ney"]
    m, n = nex + p, ney + mesh.get("q", p)
    cp = np.asarray(mesh["CP"]).reshape(n, m, 2).copy()
    x0, y0 = cp[..., 0].copy(), cp[..., 1].copy()
    cp[..., 0] = x0 + ax * np.sin(3 * y0) * x0 * (1 - x0)
    cp[..., 1] = y0 + ay * np.sin(2 * x0) * y0 * (1 - y0)
    out = dict(mesh)
    out["CP"] = cp.ravel()
    return out


def window(mesh, ex_a, ex_b, ey_a, ey_b):
    """Sub-patch of elements [ex_a, ex_b) x [ey_a, ey_b) with its control points and tables."""
    p, q = mesh["p"], mesh.get("q", mesh["p"])
    m = mesh["nex"] + p
    n = mesh["ney"] + q
    cp = np.asarray(mesh["CP"]).reshape(n, m, 2)[ey_a:ey_b + q, ex_a:ex_b + p]
    nb1, nb2 = (p + 1) ** 2, (q + 1) ** 2
    w = dict(p=p, q=q, nex=ex_b - ex_a, ney=ey_b - ey_a, CP=np.ascontiguousarray(cp).ravel(),
             C1=np.asarray(mesh["C1"])[ex_a * nb1:ex_b * nb1], C2=np.asarray(mesh["C2"])[ey_a * nb2:ey_b * nb2],
             h1=np.full(ex_b - ex_a, 1.0 / mesh["nex"]), h2=np.full(ey_b - ey_a, 1.0 / mesh["ney"]),
             W=None, kappa=None)
    return w


def window_rows(mesh, ex_a, ex_b, ey_a, ey_b):
    """Global (R, C) index arrays of the window's rows whose support lies inside it."""
    p, q = mesh["p"], mesh.get("q", mesh["p"])
    m = mesh["nex"] + p
    n = mesh["ney"] + q
    c0 = 0 if ex_a == 0 else ex_a + p
    c1 = m if ex_b == mesh["nex"] else ex_b
    r0 = 0 if ey_a == 0 else ey_a + q
    r1 = n if ey_b == mesh["ney"] else ey_b
    return (r0, r1, c0, c1)


PARTITIONS = os.path.join(os.path.dirname(GOLDEN), "partitions")


def read_info(path):
    """info.txt of the reference preprocessor as a dict."""
    out = {}
    for line in open(path):
        if ": " in line:
            k, v = line.rstrip("\n").split(": ", 1)
            out[k] = v
    return out


def partition_numbering(p, q, nex, ney, P):
    """new[natural index j*m + i] = the partition numbering of
    matrix_free/src/Partition.cpp:23-92 (parts y outer, x inner; each part's
    functions x fastest; runs of ceil(m / P) functions, the last shorter)."""
    m, n = nex + p, ney + q
    sx, sy = -(-m // P), -(-n // P)
    cx = [sx] * (P - 1) + [m - (P - 1) * sx]
    cy = [sy] * (P - 1) + [n - (P - 1) * sy]
    new = np.empty(m * n, dtype=np.int64)
    k = 0
    for jj in range(P):
        for ii in range(P):
            for lj in range(cy[jj]):
                for li in range(cx[ii]):
                    new[(jj * sy + lj) * m + ii * sx + li] = k
                    k += 1
    return new


def write_partition_files(mesh, P, out_dir, base="part"):
    """Test-only restatement of the reference preprocessor's partition output
    (matrix_free/src/Partition.cpp:3-235 with FileManager::WritePartition /
    WritePreprocessInfo, matrix_free/src/FileManager.cpp:3-69,375-396) for a
    unit-square mesh dict, so GPU tests can use meshes larger than the
    committed fixtures. test_partition_host.py checks that it reproduces the
    reference-written fixtures byte for byte."""
    p, q, nex, ney = mesh["p"], mesh.get("q", mesh["p"]), mesh["nex"], mesh["ney"]
    m, n = nex + p, ney + q
    nloc = (p + 1) * (q + 1)
    new = partition_numbering(p, q, nex, ney, P)
    sx, sy = -(-m // P), -(-n // P)
    cx = [sx] * (P - 1) + [m - (P - 1) * sx]
    cy = [sy] * (P - 1) + [n - (P - 1) * sy]
    fx = [i * sx for i in range(P)]
    fy = [j * sy for j in range(P)]
    ex0 = [0] + [fx[i] - p // 2 for i in range(1, P)]
    ey0 = [0] + [fy[j] - q // 2 for j in range(1, P)]
    ex1 = [ex0[i + 1] - 1 for i in range(P - 1)] + [nex - 1]
    ey1 = [ey0[j + 1] - 1 for j in range(P - 1)] + [ney - 1]
    on_bnd = np.zeros((n, m), bool)
    on_bnd[0, :] = on_bnd[-1, :] = on_bnd[:, 0] = on_bnd[:, -1] = True
    new_id = np.where(on_bnd.ravel(), -1, new)          # ID by natural index
    cp = np.asarray(mesh["CP"]).reshape(n, m, 2)
    C1 = np.asarray(mesh["C1"])
    C2 = np.asarray(mesh["C2"])

    def ints(v):
        return "".join(f"{int(t)} " for t in v)

    def dbls(v):
        return "".join(f"{float(t):.16g} " for t in v)
    os.makedirs(out_dir, exist_ok=True)
    with open(os.path.join(out_dir, "info.txt"), "w") as f:
        f.write(f"p: {p}\nq: {q}\nLx: {1:g}\nLy: {1:g}\nnElemX: {nex}\nnElemY: {ney}\n"
                f"part_num_1d: {P}\ndim: 2\nbase_name: {base}\n")
    for j in range(P):
        for i in range(P):
            elems = [(ey, ex) for ey in range(ey0[j], ey1[j] + 1) for ex in range(ex0[i], ex1[i] + 1)]
            owned_nat = [(fy[j] + lj) * m + fx[i] + li for lj in range(cy[j]) for li in range(cx[i])]
            owned_new = [int(new[a]) for a in owned_nat]
            touched = sorted({int(new[(ey + jl) * m + ex + il]) for ey, ex in elems
                              for jl in range(q + 1) for il in range(p + 1)})
            ownset = set(owned_new)
            ghosts = [g for g in touched if g not in ownset]
            local_new = owned_new + ghosts
            pos = {g: k for k, g in enumerate(local_new)}
            nat_of_new = np.empty(m * n, dtype=np.int64)
            nat_of_new[new] = np.arange(m * n)
            loc_nat = nat_of_new[np.asarray(local_new)]
            ien = [pos[int(new[(ey + jl) * m + ex + il])] for ey, ex in elems
                   for jl in range(q + 1) for il in range(p + 1)]
            lid = new_id[loc_nat]
            ldir = [g for g, t in zip(owned_new, lid[:len(owned_new)]) if t == -1]
            lcp = np.stack([cp.reshape(-1, 2)[a] for a in loc_nat]).ravel()
            e1, e2 = (p + 1) ** 2, (q + 1) ** 2
            with open(os.path.join(out_dir, f"{base}_{j * P + i}.txt"), "w") as f:
                f.write(f"nlocalfunc: {len(owned_new)}\nnlocalelemx: {ex1[i] - ex0[i] + 1}\n"
                        f"nlocalelemy: {ey1[j] - ey0[j] + 1}\n")
                f.write("ID\n" + ints(lid) + "\nghostID\n" + ints(ghosts) + "\nDir\n" + ints(ldir) + "\n")
                f.write("IEN\n" + ints(ien) + "\n")
                f.write("ElemSize1\n" + dbls([1.0 / nex] * (ex1[i] - ex0[i] + 1)) + "\n")
                f.write("ElemSize2\n" + dbls([1.0 / ney] * (ey1[j] - ey0[j] + 1)) + "\n")
                f.write("CP\n" + dbls(lcp) + "\n")
                f.write("NURBSExtraction1\n" + dbls(C1[ex0[i] * e1:(ex1[i] + 1) * e1]) + "\n")
                f.write("NURBSExtraction2\n" + dbls(C2[ey0[j] * e2:(ey1[j] + 1) * e2]) + "\n")


REF_CPU_LIB = os.path.join(ROOT, "oracle", "_ref", "libigaref.so")
REF_GPU_LIB = os.path.join(ROOT, "oracle", "_ref", "libigaref_gpu.so")


class RefGpuKernel:
    """The reference's own GPU MatMult kernel (matrix_free_gpu/src/mult.cu,
    compiled for sm_100a with P_ORDER = 3 into oracle/_ref/libigaref_gpu.so)
    on a unit-square p = 3 mesh made by the reference's own preprocessing
    (ref_mesh / ref_tables of oracle/_ref/libigaref.so), tables uploaded once.
    apply(x, y) takes device pointers (ints) of N doubles: y = A_ref x with
    y[Dir] = 0. Test and benchmark infrastructure, a checker and a baseline
    only."""

    P = 3

    @staticmethod
    def available():
        return os.path.exists(REF_GPU_LIB) and os.path.exists(REF_CPU_LIB)

    def __init__(self, nex, ney, Lx=1.0, Ly=1.0, ID=None):
        """ID: equation numbers to use instead of the reference's serial ones
        (the kernel adds control point A's row into y[ID[A]] for ID[A] >= 0)."""
        p = self.P
        ID_in = ID
        cpu = ctypes.CDLL(REF_CPU_LIB)
        self.L = ctypes.CDLL(REF_GPU_LIB)
        m, n = nex + p, ney + p
        nb = (p + 1) ** 2
        self.N = m * n
        CP = np.zeros(2 * m * n)
        IEN = np.zeros(nex * ney * nb, np.int32)
        ID = np.zeros(m * n, np.int32)
        Dir = np.zeros(m * n, np.int32)
        nd = ctypes.c_int()
        C1, C2 = np.zeros(nex * nb), np.zeros(ney * nb)
        h1, h2 = np.zeros(nex), np.zeros(ney)
        cpu.ref_mesh(p, p, nex, ney, ctypes.c_double(Lx), ctypes.c_double(Ly), _p(CP), _p(IEN), _p(ID), _p(Dir),
                     ctypes.byref(nd), _p(C1), _p(C2), _p(h1), _p(h2))
        qp, qw = np.zeros(p + 1), np.zeros(p + 1)
        B, dB = np.zeros(nb), np.zeros(nb)
        cpu.ref_tables(p, _p(qp), _p(qw), _p(B), _p(dB))
        if ID_in is not None:
            ID = np.ascontiguousarray(ID_in, dtype=np.int32)
            assert ID.shape == (m * n,)
        # the reference's arrays of this mesh, for passing the same ones to other entry points
        self.arrays = dict(CP=CP, IEN=IEN, ID=ID, C1=C1, C2=C2, h1=h1, h2=h2, B=B, dB=dB, qw=qw)
        h = VP()
        st = self.L.refgpu_create(p, nex, ney, _p(B), _p(dB), _p(qw), _p(C1), _p(C2), _p(h1), _p(h2), _p(IEN),
                                  _p(ID), _p(CP), ctypes.byref(h))
        if st != 0:
            raise RuntimeError("refgpu_create failed")
        self.h = h

    def apply(self, x_ptr, y_ptr):
        if self.L.refgpu_apply(self.h, VP(x_ptr), VP(y_ptr)) != 0:
            raise RuntimeError("refgpu_apply failed")

    def close(self):
        if getattr(self, "h", None):
            self.L.refgpu_destroy(self.h)
            self.h = None
