"""Pin the C oracle restatement to the reference's own element code.

The golden vectors were recorded from the reference sources compiled into
oracle/_ref/libigaref.so (tests/golden/make_golden.py). Tolerances are
relative to the largest entry; both sides are FP64 and differ only in the
order of rounding.
"""
import numpy as np
import pytest

from iga_testlib import boundary_mask, golden_mesh, splitmix_normal, splitmix_uniform, unit_square_mesh

CASES = ["c1", "p3_16", "p4_12", "p3_12x7", "p2q3_9x6"]
TOL = 1e-13


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_rng_matches_python(orc):
    assert np.array_equal(orc.uniform(1, -1.0, 1.0, 1001), splitmix_uniform(1, -1.0, 1.0, 1001))
    assert np.allclose(orc.normal(2, 1001), splitmix_normal(2, 1001), rtol=0, atol=1e-15)


@pytest.mark.parametrize("p", range(1, 7))
def test_gauss_and_bernstein(orc, gold, p):
    x, w = orc.gauss01(p + 1)
    assert np.abs(x - gold[f"tab_p{p}_qp"]).max() < 1e-15
    assert np.abs(w - gold[f"tab_p{p}_qw"]).max() < 1e-15
    B = np.concatenate([orc.bernstein(p, xi)[0] for xi in gold[f"tab_p{p}_qp"]])
    dB = np.concatenate([orc.bernstein(p, xi)[1] for xi in gold[f"tab_p{p}_qp"]])
    assert np.abs(B - gold[f"tab_p{p}_B"]).max() < 1e-15
    assert np.abs(dB - gold[f"tab_p{p}_dB"]).max() < 1e-13


@pytest.mark.parametrize("name,p", [("open_p2", 2), ("open_p3", 3), ("open_p4", 4), ("rep_p3", 3),
                                    ("nonuni_p4", 4)])
def test_extraction_and_greville(orc, gold, name, p):
    S = gold[f"ext_{name}_knots"]
    C = orc.extraction(p, S)
    ref = gold[f"ext_{name}_C"]
    assert np.abs(C - ref[: C.size]).max() < 1e-14
    assert np.abs(orc.greville(p, S) - gold[f"ext_{name}_greville"]).max() < 1e-15


@pytest.mark.parametrize("name", CASES)
def test_mesh_generation(orc, gold, name):
    M = golden_mesh(gold, name)
    M2 = unit_square_mesh(orc, M["p"], M["q"], M["nex"], M["ney"])
    for k in ("CP", "C1", "C2", "h1", "h2"):
        assert np.abs(M2[k] - M[k]).max() < 1e-15, k
    m, n = M["nex"] + M["p"], M["ney"] + M["q"]
    assert np.array_equal(np.flatnonzero(boundary_mask(m, n)), gold[f"{name}_Dir"])


@pytest.mark.parametrize("name", CASES)
def test_apply_mf_matches_reference(orc, gold, name):
    M = golden_mesh(gold, name)
    assert rel(orc.apply_mf(M, gold[f"{name}_x"]), gold[f"{name}_y_mf"]) < TOL


@pytest.mark.parametrize("name", [c for c in CASES if c != "p2q3_9x6"])
def test_apply_sf_matches_reference(orc, gold, name):
    M = golden_mesh(gold, name)
    assert rel(orc.apply_sf(M, gold[f"{name}_x"]), gold[f"{name}_y_sf"]) < TOL


@pytest.mark.parametrize("name", CASES)
def test_mf_equals_assembled_on_free_rows(orc, gold, name):
    """Reference semantics: MF == assembled K_ref only with x[Dir] = 0."""
    M = golden_mesh(gold, name)
    x = gold[f"{name}_x"].copy()
    x[gold[f"{name}_Dir"]] = 0.0
    assert rel(orc.apply_mf(M, x), gold[f"{name}_y_assembled_x0"]) < TOL
    assert rel(gold[f"{name}_y_mf_x0"], gold[f"{name}_y_assembled_x0"]) < TOL


@pytest.mark.parametrize("name", CASES)
def test_rhs_matches_reference(orc, gold, name):
    M = golden_mesh(gold, name)
    assert rel(orc.rhs(M, 0), gold[f"{name}_F"]) < TOL


@pytest.mark.parametrize("p,ne", [(3, 16), (4, 10)])
def test_fem_preconditioner_matches_reference(orc, gold, p, ne):
    g = orc.fem_nodes(p, ne)
    assert np.abs(g - gold[f"fem_p{p}_nodes"]).max() < 1e-15
    y = orc.fem_matvec(g, g, gold[f"fem_p{p}_x"], sign=-1.0)
    assert rel(y, gold[f"fem_p{p}_y"]) < TOL


def test_fem_nodes_p2_replacement(orc, gold):
    """The reference's p=2 FEM nodes are NaN (Greville of degree 0 divides by 0);
    the replacement is the degree-2 Greville abscissae of the IGA knots."""
    assert np.isnan(gold["fem_p2_nodes"]).all()
    g = orc.fem_nodes(2, 6)
    assert np.isfinite(g).all() and g[0] == 0.0 and g[-1] == 1.0
    assert np.all(np.diff(g) > 0)


def test_spd_operator_and_sign(orc):
    M = unit_square_mesh(orc, 3, 3, 6, 6)
    m = 9
    x = splitmix_uniform(3, -1, 1, m * m)
    bmask = boundary_mask(m, m)
    yneg = orc.apply_mf(M, x, sign=-1.0, bc=0)
    ypos = orc.apply_mf(M, x, sign=+1.0, bc=0)
    assert np.allclose(yneg, -ypos, rtol=0, atol=1e-15)
    # SPD form: boundary rows are identity and x[Dir] is not read.
    xz = x.copy()
    xz[bmask] = 0.0
    yspd = orc.apply_mf(M, x, sign=1.0, bc=1)
    assert np.allclose(yspd[bmask], x[bmask])
    assert rel(yspd[~bmask], orc.apply_mf(M, xz, sign=1.0, bc=0)[~bmask]) < TOL


def test_cpu_pcg_converges(orc):
    M = unit_square_mesh(orc, 3, 3, 12, 12)
    b = orc.rhs(M, 1)
    x, it, rr = orc.pcg(M, b, rtol=1e-10)
    assert it > 0 and rr <= 1e-10
    # B-spline coefficients approximate sin(pi x) sin(pi y) at the Greville points to O(h^2)
    cp = M["CP"].reshape(-1, 2)
    u = np.sin(np.pi * cp[:, 0]) * np.sin(np.pi * cp[:, 1])
    assert np.abs(x - u).max() < 0.05
