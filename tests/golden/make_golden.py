"""Generate tests/golden/ref_vectors.npz and tests/golden/partitions/ from the
REFERENCE's own code.

Runs only where the reference tree is available: it builds oracle/_ref/libigaref.so
(oracle/Makefile target "ref": the reference's PETSc-free sources compiled in
place plus oracle/ref_harness.cpp) and records its outputs on seeded inputs.
The reference ships no golden vectors, so these recorded outputs are the pins for
the oracle restatement (tests/test_oracle_pin.py) and, through it, for the CUDA
kernels.

The partition fixtures are the reference preprocessor's files (info.txt and
<base>_<rank>.txt written by its Partition + FileManager) for small meshes,
with a seeded x in the partition numbering and y = the reference's partitioned
MatMulMF (every part's element loop on its ghosted local form).

    python tests/golden/make_golden.py                   # everything
    python tests/golden/make_golden.py --partitions-only
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
from iga_testlib import splitmix_uniform  # noqa: E402

VP = ctypes.c_void_p


def _p(a):
    return a.ctypes.data_as(VP)


def load_ref():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    return ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libigaref.so"))


def ref_mesh(L, p, q, nex, ney, Lx=1.0, Ly=1.0):
    m, n = nex + p, ney + q
    nf = m * n
    CP = np.zeros(2 * nf)
    IEN = np.zeros(nex * ney * (p + 1) * (q + 1), np.int32)
    ID = np.zeros(nf, np.int32)
    Dir = np.zeros(nf, np.int32)
    nd = ctypes.c_int()
    C1 = np.zeros(nex * (p + 1) ** 2)
    C2 = np.zeros(ney * (q + 1) ** 2)
    h1 = np.zeros(nex)
    h2 = np.zeros(ney)
    L.ref_mesh(p, q, nex, ney, ctypes.c_double(Lx), ctypes.c_double(Ly), _p(CP), _p(IEN), _p(ID),
               _p(Dir), ctypes.byref(nd), _p(C1), _p(C2), _p(h1), _p(h2))
    return dict(p=p, q=q, nex=nex, ney=ney, CP=CP, IEN=IEN, ID=ID, Dir=Dir[: nd.value].copy(),
                C1=C1, C2=C2, h1=h1, h2=h2)


def _margs(M):
    return [M["p"], M["q"], M["nex"], M["ney"], _p(M["CP"]), _p(M["IEN"]), _p(M["ID"]),
            _p(M["Dir"]), len(M["Dir"]), _p(M["C1"]), _p(M["C2"]), _p(M["h1"]), _p(M["h2"])]


def main():
    L = load_ref()
    out = {}
    # 1-D tables: Gauss points/weights on [0,1], Bernstein B and dB at them.
    for p in range(1, 7):
        qp, qw = np.zeros(p + 1), np.zeros(p + 1)
        B, dB = np.zeros((p + 1) ** 2), np.zeros((p + 1) ** 2)
        L.ref_tables(p, _p(qp), _p(qw), _p(B), _p(dB))
        out[f"tab_p{p}_qp"], out[f"tab_p{p}_qw"] = qp, qw
        out[f"tab_p{p}_B"], out[f"tab_p{p}_dB"] = B, dB
    # Extraction operators and Greville abscissae, incl. a knot vector with a
    # repeated interior knot.
    knots = {
        "open_p2": (2, np.r_[np.zeros(3), np.arange(1, 8) / 8, np.ones(3)]),
        "open_p3": (3, np.r_[np.zeros(4), np.arange(1, 8) / 8, np.ones(4)]),
        "open_p4": (4, np.r_[np.zeros(5), np.arange(1, 8) / 8, np.ones(5)]),
        "rep_p3": (3, np.array([0, 0, 0, 0, 0.2, 0.5, 0.5, 0.7, 1, 1, 1, 1.0])),
        "nonuni_p4": (4, np.array([0, 0, 0, 0, 0, 0.1, 0.25, 0.3, 0.6, 0.65, 0.9, 1, 1, 1, 1, 1.0])),
    }
    for name, (p, S) in knots.items():
        S = np.ascontiguousarray(S, dtype=np.float64)
        C = np.zeros(len(S) * (p + 1) ** 2)
        n = L.ref_extraction(p, _p(S), len(S), _p(C))
        out[f"ext_{name}_knots"] = S
        out[f"ext_{name}_C"] = C[:n].copy()
        g = np.zeros(len(S))
        ng = L.ref_greville(p, _p(S), len(S), _p(g))
        out[f"ext_{name}_greville"] = g[:ng].copy()
    # Operators on seeded inputs. "c1" is the p=2 64x64 configuration with
    # x ~ U[-1,1] (seed 0); the others cover p=3/4, non-square and p != q.
    cases = {
        "c1": (2, 2, 64, 64, 0),
        "p3_16": (3, 3, 16, 16, 5),
        "p4_12": (4, 4, 12, 12, 6),
        "p3_12x7": (3, 3, 12, 7, 7),
        "p2q3_9x6": (2, 3, 9, 6, 8),
    }
    for name, (p, q, nex, ney, seed) in cases.items():
        M = ref_mesh(L, p, q, nex, ney)
        nf = (nex + p) * (ney + q)
        x = splitmix_uniform(seed, -1.0, 1.0, nf)
        y_mf = np.zeros(nf)
        L.ref_apply_mf(*_margs(M), _p(x), _p(y_mf), 1)
        xz = x.copy()
        xz[M["Dir"]] = 0.0
        y_mf0 = np.zeros(nf)
        L.ref_apply_mf(*_margs(M), _p(xz), _p(y_mf0), 1)
        y_K0 = np.zeros(nf)
        L.ref_assembled_matvec(*_margs(M), _p(xz), _p(y_K0))
        F = np.zeros(nf)
        L.ref_rhs(*_margs(M), _p(F))
        for k in ("CP", "IEN", "ID", "Dir", "C1", "C2", "h1", "h2"):
            out[f"{name}_{k}"] = M[k]
        out[f"{name}_dims"] = np.array([p, q, nex, ney], np.int32)
        out[f"{name}_x"] = x
        out[f"{name}_y_mf"] = y_mf
        out[f"{name}_y_mf_x0"] = y_mf0
        out[f"{name}_y_assembled_x0"] = y_K0
        out[f"{name}_F"] = F
        if p == q:
            y_sf = np.zeros(nf)
            L.ref_apply_sf(*_margs(M), _p(x), _p(y_sf), 1)
            out[f"{name}_y_sf"] = y_sf
    # FEM preconditioner grid and matrix (p = 3, 4; the reference gives NaN
    # nodes for p = 2, also recorded).
    for p, ne in ((3, 16), (4, 10), (2, 6)):
        nfx = ne + p
        nf = nfx * nfx
        CP = np.zeros(2 * nf)
        IEN = np.zeros((nfx - 1) ** 2 * 4, np.int32)
        ID = np.zeros(nf, np.int32)
        Dir = np.zeros(nf, np.int32)
        nd = ctypes.c_int()
        L.ref_fem_mesh(p, p, ne, ne, ctypes.c_double(1.0), ctypes.c_double(1.0), _p(CP), _p(IEN),
                       _p(ID), _p(Dir), ctypes.byref(nd))
        out[f"fem_p{p}_nodes"] = CP[0:2 * nfx:2].copy()
        if p >= 3:
            x = splitmix_uniform(11 + p, -1.0, 1.0, nf)
            y = np.zeros(nf)
            Dir = Dir[: nd.value].copy()
            L.ref_fem_matvec(nfx, nfx, _p(CP), _p(IEN), _p(ID), _p(Dir), len(Dir), _p(x), _p(y))
            out[f"fem_p{p}_x"] = x
            out[f"fem_p{p}_y"] = y
    path = os.path.join(HERE, "ref_vectors.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


# (name, p, nElemX, nElemY, part_num_1d)
PARTITION_CASES = [("p3_9x7_2", 3, 9, 7, 2), ("p2_10x12_3", 2, 10, 12, 3), ("p4_8x11_2", 4, 8, 11, 2)]


def write_partitions(L):
    L.ref_write_partition.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 2 + [ctypes.c_int, ctypes.c_char_p,
                                                                                    ctypes.c_char_p]
    L.ref_apply_partitioned.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        VP, VP, ctypes.c_int]
    for k, (name, p, nex, ney, P) in enumerate(PARTITION_CASES):
        d = os.path.join(HERE, "partitions", name)
        os.makedirs(d, exist_ok=True)
        L.ref_write_partition(p, p, nex, ney, 1.0, 1.0, P, d.encode(), b"part")
        nf = (nex + p) * (ney + p)
        x = splitmix_uniform(40 + k, -1.0, 1.0, nf)
        y = np.zeros(nf)
        got = L.ref_apply_partitioned(d.encode(), b"part", p, p, P * P, _p(x), _p(y), nf)
        assert got == nf, (got, nf)
        np.savez_compressed(os.path.join(d, "vectors.npz"), x=x, y=y)
        print(f"wrote {d}: {P * P} parts")


if __name__ == "__main__":
    if "--partitions-only" not in sys.argv:
        main()
    write_partitions(load_ref())
