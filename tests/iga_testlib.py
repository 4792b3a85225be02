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
