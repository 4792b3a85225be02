"""CPU-side checks of the C ABI library: it loads, exports every declared
entry point, generates meshes identical to the oracle's, and reports (not
crashes on) the absence of a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from iga_testlib import ROOT, load_binding, unit_square_mesh

HEADERS = [os.path.join(ROOT, "include", h) for h in sorted(os.listdir(os.path.join(ROOT, "include")))
           if h.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z_0-9]*\s*\**\s*(iga_[A-Za-z_0-9]+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    ib = load_binding()
    L = ib.lib()
    names = declared_functions()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    ib = load_binding()
    bound = {s[0] for s in ib.SIGNATURES}
    assert set(declared_functions()) <= bound


@pytest.mark.parametrize("p,nex,ney", [(1, 5, 4), (2, 64, 64), (3, 16, 9), (4, 12, 12), (5, 11, 7)])
def test_mesh_generator_matches_oracle(orc, p, nex, ney):
    ib = load_binding()
    M = ib.unit_square(p, nex, ney)
    R = unit_square_mesh(orc, p, p, nex, ney)
    for k in ("CP", "C1", "C2"):
        assert np.array_equal(M[k], R[k]), k


def test_status_strings():
    ib = load_binding()
    L = ib.lib()
    for s in range(0, 9):
        assert L.iga_status_str(s)
    assert L.iga_status_str(99) == b"unknown status"


def test_invalid_meshes_are_rejected_before_any_device_work():
    ib = load_binding()
    M = ib.unit_square(3, 8, 8)
    bad = dict(M)
    bad["q"] = 2
    with pytest.raises(ib.IgaError) as e:
        ib.Plan(bad)
    assert e.value.status == 2   # IGA_ERR_UNSUPPORTED: p != q
    with pytest.raises(ib.IgaError) as e:
        ib.Plan(dict(M, p=7, q=7))
    assert e.value.status == 2
    ID = np.arange(11 * 11, dtype=np.int32)   # not -1 on the boundary
    with pytest.raises(ib.IgaError) as e:
        ib.Plan(M, ID=ID)
    assert e.value.status == 1


def test_no_gpu_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    ib = load_binding()
    with pytest.raises(ib.IgaError) as e:
        ib.Plan(ib.unit_square(2, 8, 8))
    assert e.value.status == 3   # IGA_ERR_CUDA
