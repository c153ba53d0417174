"""The oracle's line tables and table scorers (precompute.py:18-89) pinned to
the reference's own outputs (tests/golden/make_golden_lines.py): the whole
tables for small grids, SHA-256 digests of the n = 20, 40 and 75 tables, and
the scores of seeded states and edge-case point lists.  Also the host-side
argument handling of the package's drop-in, which runs before any device
call."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from no_three_in_line_b200 import precompute


@pytest.fixture(scope="module")
def lines_golden(golden):
    return golden("lines_golden.npz")


def _digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _lists(g):
    pts, starts = g["points"], g["starts"]
    for i, n in enumerate(g["n"]):
        yield int(n), [tuple(map(int, p)) for p in pts[starts[i]:starts[i + 1]]], i


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 10, 13])
def test_small_tables_match_reference(oracle, lines_golden, n):
    t = oracle.geometry_tables(n)
    assert t["line_count"] == int(lines_golden[f"t{n}_line_count"])
    assert np.array_equal(t["offsets"], lines_golden[f"t{n}_offsets"])
    assert np.array_equal(t["indices"], lines_golden[f"t{n}_indices"])
    assert np.array_equal(t["pair_to_line"], lines_golden[f"t{n}_pair_to_line"])


@pytest.mark.parametrize("n", [20, 40, 75])
def test_large_tables_match_reference_digests(oracle, lines_golden, n):
    t = oracle.geometry_tables(n)
    sizes = lines_golden[f"h{n}_sizes"]
    assert (t["line_count"], len(t["indices"]), len(t["pair_to_line"])) == tuple(int(x) for x in sizes)
    want = [str(x) for x in lines_golden[f"h{n}"]]
    assert [_digest(t["pair_to_line"]), _digest(t["offsets"]), _digest(t["indices"])] == want


def test_scores_match_reference(oracle, lines_golden):
    tables = {}
    for n, pts, i in _lists(lines_golden):
        if n not in tables:
            tables[n] = oracle.geometry_tables(n)
        try:
            ps = oracle.score_pair_table(pts, tables[n])
        except ValueError:
            ps = -1
        try:
            cs = oracle.score_csr(pts, tables[n])
        except IndexError:
            cs = -1
        assert (ps, cs) == (int(lines_golden["pair_scores"][i]), int(lines_golden["csr_scores"][i])), (n, i)


def test_triangular_pair_index_matches_oracle(oracle):
    for args in [(0, 1, 25), (24, 3, 25), (7, 7, 25), (-1, 3, 25), (3, 25, 25), (5624, 0, 5625)]:
        try:
            want = oracle.triangular_pair_index(*args)
        except ValueError:
            with pytest.raises(ValueError):
                precompute.triangular_pair_index(*args)
            continue
        assert precompute.triangular_pair_index(*args) == want


def test_host_checks_raise_before_any_device_call():
    t = precompute.GeometryTables(10, np.zeros(0, np.int32), np.zeros(1, np.int64), np.zeros(0, np.int32), 0, 0.0)
    with pytest.raises(ValueError):
        precompute.score_pair_table([(1, 1), (2, 2), (1, 1)], t)      # a repeated point
    with pytest.raises(ValueError):
        precompute.score_pair_table([(0, -1), (1, 1)], t)             # id -1
    with pytest.raises(ValueError):
        precompute.score_pair_table([(9, 9), (10, 0)], t)             # id 100 >= 100
    assert precompute.score_pair_table([(9, 9)], t) == 0              # no pair: no check, score 0
    with pytest.raises(IndexError):
        precompute.score_csr([(1, 1), (10, 0)], t)
    with pytest.raises(IndexError):
        precompute.score_csr([(-10, -1)], t)                          # id -101 < -100
    with pytest.raises(ValueError):
        precompute.build_geometry_tables(0)
    with pytest.raises(ValueError):
        precompute.build_geometry_tables(76)
