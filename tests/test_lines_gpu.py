"""Line tables and table scorers on the GPU (precompute.py:18-127) through the
C ABI: tables bit-exact against the oracle (itself pinned to the reference by
tests/test_lines_oracle.py) and the reference's digests at n = 75; scores of
the golden point lists and of seeded n = 75 populations, exceptions included."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from no_three_in_line_b200 import gpu, precompute, state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lines_golden(golden):
    return golden("lines_golden.npz")


@pytest.fixture(scope="module")
def tables75(cuda):
    return precompute.build_geometry_tables(75)


def _digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 13, 40])
def test_tables_match_oracle(cuda, oracle, n):
    got = precompute.build_geometry_tables(n)
    ref = oracle.geometry_tables(n)
    assert got.n == n and got.line_count == ref["line_count"]
    assert got.offsets.dtype == np.int64 and got.indices.dtype == np.int32 and got.pair_to_line.dtype == np.int32
    assert np.array_equal(got.offsets, ref["offsets"])
    assert np.array_equal(got.indices, ref["indices"])
    assert np.array_equal(got.pair_to_line, ref["pair_to_line"])


def test_n75_tables_match_reference_digests(tables75, lines_golden):
    sizes = tuple(int(x) for x in lines_golden["h75_sizes"])
    assert (tables75.line_count, len(tables75.indices), len(tables75.pair_to_line)) == sizes
    assert [_digest(tables75.pair_to_line), _digest(tables75.offsets), _digest(tables75.indices)] == \
        [str(x) for x in lines_golden["h75"]]


def test_golden_point_lists(cuda, lines_golden, tables75):
    g = lines_golden
    tables = {75: tables75}
    for i, n in enumerate(g["n"]):
        n = int(n)
        pts = [tuple(map(int, p)) for p in g["points"][g["starts"][i]:g["starts"][i + 1]]]
        if n not in tables:
            tables[n] = precompute.build_geometry_tables(n)
        try:
            ps = precompute.score_pair_table(pts, tables[n])
        except ValueError:
            ps = -1
        try:
            cs = precompute.score_csr(pts, tables[n])
        except IndexError:
            cs = -1
        assert (ps, cs) == (int(g["pair_scores"][i]), int(g["csr_scores"][i])), (n, i)


def test_n75_populations_equal_determinant_scores(cuda, tables75):
    p, q = state.seeded_population(75, 70)  # three occupancy words, the last one partial
    want = np.asarray(gpu.score_population_gpu(p, q), np.int64)
    assert np.array_equal(precompute.score_pair_table_population(p, q, tables75), want)
    assert np.array_equal(precompute.score_csr_population(p, q, tables75), want)


def test_tables_built_elsewhere_are_uploaded(cuda, oracle):
    ref = oracle.geometry_tables(13)
    t = precompute.GeometryTables(13, ref["pair_to_line"], ref["offsets"], ref["indices"], ref["line_count"], 0.0)
    pts = [(r, (3 * r + 1) % 13) for r in range(13)] + [(r, (3 * r + 5) % 13) for r in range(13)]  # distinct
    assert precompute.score_pair_table(pts, t) == oracle.score_pair_table(pts, ref)
    assert precompute.score_csr(pts, t) == oracle.score_csr(pts, ref)


def test_device_rejects_what_the_reference_rejects(cuda, tables75):
    p, q = state.seeded_population(75, 2)
    q[1, 5] = p[1, 5]  # a repeated point
    with pytest.raises(ValueError):
        precompute.score_pair_table_population(p, q, tables75)
    with pytest.raises(ValueError):
        precompute.score_pair_table([(r, c) for r in range(23) for c in range(23)], tables75)  # 529 > 512 points


def test_benchmark_precomputation_agrees(cuda):
    st = state.random_state(20, __import__("random").Random(5))
    pts = [(r, int(st.P[r])) for r in range(20)] + [(r, int(st.Q[r])) for r in range(20)]
    out = precompute.benchmark_precomputation(20, pts)
    assert out["n"] == 20 and out["line_count"] == 6738 and out["line_incidences"] == 25180
    assert set(out["seconds_per_score"]) == {"A_numba_determinants", "B_pair_to_line", "C_canonical_line_dict",
                                             "D_csr_line_scan"}
