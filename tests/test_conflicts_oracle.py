"""Conflict analysis restated in the oracle (conflicts.py:36-72 over
geometry.py:14-40), pinned to outputs of the reference's analyze_points
(tests/golden/conflicts_golden.json.gz, made by make_golden_conflicts.py)."""
from __future__ import annotations

import gzip
import json
from pathlib import Path

import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "conflicts_golden.json.gz"


def load_cases():
    with gzip.open(GOLDEN, "rt", encoding="utf-8") as f:
        return json.load(f)


def as_expected(g):
    return {"triples": g["triples"], "violating_lines": g["violating_lines"],
            "max_line_occupancy": g["max_line_occupancy"], "max_point_badness": g["max_point_badness"],
            "weighted_score": g["weighted_score"], "badness": list(g["badness"]),
            "lines": [(tuple(k), tuple(tuple(p) for p in pts), t) for k, pts, t in g["lines"]],
            "slope_histogram": {(dx, dy): c for dx, dy, c in g["slope_histogram"]}}


def weights_of(g):
    return None if g["weights"] is None else {(a, b, c): w for a, b, c, w in g["weights"]}


def test_fixture_covers_the_cases():
    cases = load_cases()
    assert {"e10", "block9", "two_diagonals", "empty", "pair", "weighted_0", "n75_0", "random_5"} <= set(cases)
    assert cases["e10"]["triples"] == 10 and cases["e10"]["violating_lines"] == 10
    assert cases["block9"]["max_line_occupancy"] == 9


@pytest.mark.parametrize("name", sorted(load_cases()))
def test_oracle_analysis_matches_the_reference(oracle, name):
    g = load_cases()[name]
    got = oracle.analyze_points([tuple(p) for p in g["points"]], weights_of(g))
    assert got == as_expected(g)


def test_geometry_helpers_match_the_reference_keys():
    from no_three_in_line_b200 import geometry

    g = load_cases()["block9"]
    for key, pts, _ in g["lines"][:80]:
        assert geometry.canonical_line(tuple(pts[0]), tuple(pts[-1])) == tuple(key)
        assert geometry.canonical_line(tuple(pts[-1]), tuple(pts[1])) == tuple(key)
        assert geometry.determinant(tuple(pts[0]), tuple(pts[1]), tuple(pts[2])) == 0
    hist = {(dx, dy): c for dx, dy, c in g["slope_histogram"]}
    got = {}
    for key, _, t in g["lines"]:
        s = geometry.primitive_slope(tuple(key))
        got[s] = got.get(s, 0) + t
    assert got == hist
    with pytest.raises(ValueError, match="two distinct points"):
        geometry.canonical_line((3, 4), (3, 4))
