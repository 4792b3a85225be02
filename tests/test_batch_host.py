"""Host logic of the batched solver: the tuning-table reader, the problem
generator and the right-hand sides (no GPU)."""
import json

import numpy as np
import pytest

from iga_testlib import load_binding, splitmix_normal


@pytest.fixture(scope="module")
def ib():
    return load_binding()


def test_tune_lookup_reads_table(ib, tmp_path):
    path = tmp_path / "t.json"
    path.write_text(json.dumps({
        "format": "iga-batch-tune-1", "device": "x", "sm_count": 148,
        "rows": [{"p": 3, "precision": "fp64", "ney_max": 64, "rows_per_strip": 16, "us": 1.5},
                 {"p": 3, "precision": "fp64", "ney_max": 256, "rows_per_strip": 32, "us": 2.0},
                 {"p": 2, "precision": "mixed", "ney_max": 128, "rows_per_strip": 24}],
        "warps": [{"p": 3, "precision": "fp64", "warps": 7, "us": 3.0}]}))
    assert ib.tune_lookup(str(path), 3, ib.FP64, 10, 64) == (16, 7)
    assert ib.tune_lookup(str(path), 3, ib.FP64, 10, 65) == (0, 7)      # bucket 96: no entry
    assert ib.tune_lookup(str(path), 3, ib.FP64, 10, 250) == (32, 7)
    assert ib.tune_lookup(str(path), 2, ib.MIXED, 10, 100) == (24, 0)
    assert ib.tune_lookup(str(path), 2, ib.FP64, 10, 100) == (0, 0)
    assert ib.tune_lookup(str(tmp_path / "absent.json"), 3, ib.FP64, 8, 8) == (0, 0)


@pytest.mark.parametrize("text", ["{", "[]", '{"format": "other"}', '{"format": "iga-batch-tune-1", "rows": [{"p": 3}]}',
                                  '{"format": "iga-batch-tune-1"} x'])
def test_tune_lookup_rejects_bad_tables(ib, tmp_path, text):
    path = tmp_path / "bad.json"
    path.write_text(text)
    with pytest.raises(ib.IgaError):
        ib.tune_lookup(str(path), 3, ib.FP64, 8, 8)


def test_batch_problem_generator(ib):
    a = ib.batch_problems(256, seed=2)
    assert a == ib.batch_problems(256, seed=2) and a != ib.batch_problems(256, seed=3)
    ps = [p for p, _, _ in a]
    ns = [n for _, n, _ in a] + [n for _, _, n in a]
    assert set(ps) == {2, 3} and set(ns) == set(range(32, 257, 16))
    assert 100 < ps.count(2) < 156
    b = ib.batch_rhs(a[:4], seed=2)
    off = 0
    for p, nex, ney in a[:4]:
        m, n = nex + p, ney + p
        v = b[off:off + m * n].reshape(n, m)
        assert np.all(v[0] == 0) and np.all(v[-1] == 0) and np.all(v[:, 0] == 0) and np.all(v[:, -1] == 0)
        off += m * n
    assert off == len(b)
    # problem 0 is the start of the seed's normal stream
    m, n = a[0][1] + a[0][0], a[0][2] + a[0][0]
    ref = splitmix_normal(2, m * n).reshape(n, m)
    assert np.array_equal(b[:m * n].reshape(n, m)[1:-1, 1:-1], ref[1:-1, 1:-1])
