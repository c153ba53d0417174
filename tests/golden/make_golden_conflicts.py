"""Generate the conflict-analysis golden fixture (conflicts_golden.json.gz)
from the reference itself.

Run once, in a container that has the reference checked out and numba:

    NUMBA_CACHE_DIR=/tmp/n3_numba python tests/golden/make_golden_conflicts.py /path/to/reference

(or set N3_REFERENCE to the checkout instead of passing it).

Records ``conflicts.analyze_points`` (conflicts.py:36-72, with
``geometry.canonical_line`` and ``primitive_slope``, geometry.py:14-40) on:
seeded n = 20 and n = 75 states (``state.random_state``), the reference's
fixture results/best-near-solution-E10.json, dense point sets with lines of up
to 40 points, random point subsets, and states scored with line weights.  The
GPU box never runs this script; tests read the fixture.
"""
from __future__ import annotations

import gzip
import json
import os
import sys
from pathlib import Path
from random import Random

HERE = Path(__file__).resolve().parent
if len(sys.argv) > 1:
    REFERENCE = Path(sys.argv[1])
elif os.environ.get("N3_REFERENCE"):
    REFERENCE = Path(os.environ["N3_REFERENCE"])
else:
    raise SystemExit("usage: make_golden_conflicts.py /path/to/reference  (or set N3_REFERENCE)")
sys.path.insert(0, str(REFERENCE / "src"))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/n3_numba_cache")

from no_three_75 import conflicts, io, state  # noqa: E402


def record(points, weights=None) -> dict:
    m = conflicts.analyze_points(list(points), weights)
    return {"points": [list(p) for p in points],
            "weights": None if weights is None else [[*k, w] for k, w in weights.items()],
            "triples": m.triples, "violating_lines": m.violating_lines,
            "max_line_occupancy": m.max_line_occupancy, "max_point_badness": m.max_point_badness,
            "weighted_score": m.weighted_score, "badness": list(m.badness),
            "lines": [[list(line.key), [list(p) for p in line.points], line.triples] for line in m.lines],
            "slope_histogram": [[dx, dy, c] for (dx, dy), c in m.slope_histogram.items()]}


def main():
    cases = {}
    for i in range(24):
        cases[f"n20_{i}"] = record(state.random_state(20, Random(91001 + i)).points())
    for i in range(4):
        cases[f"n75_{i}"] = record(state.random_state(75, Random(91001 + i)).points())
    n, pts, _ = io.load_candidate(REFERENCE / "results" / "best-near-solution-E10.json")
    cases["e10"] = record(pts)
    # dense sets: every point of a 9 x 9 block (lines of 9), a 6 x 6 block,
    # two long diagonals (lines of 40 and 39 points)
    cases["block9"] = record([(r, c) for r in range(9) for c in range(9)])
    cases["block6_offset"] = record([(r + 30, c + 60) for r in range(6) for c in range(6)])
    cases["two_diagonals"] = record([(i, i) for i in range(40)] + [(i, 74 - i) for i in range(40) if i != 37])
    rng = Random(5)
    grid = [(r, c) for r in range(75) for c in range(75)]
    for i, size in enumerate([3, 17, 60, 100, 150, 160]):
        cases[f"random_{i}"] = record(rng.sample(grid, size))
    # line weights on states: the reference's weighted score (breakout line weights)
    for i in range(3):
        pts = state.random_state(20, Random(93001 + i)).points()
        lines = conflicts.analyze_points(pts).lines
        weights = {line.key: 2 + k % 5 for k, line in enumerate(lines[::2])}
        weights[(1, -1, 0)] = 7
        cases[f"weighted_{i}"] = record(pts, weights)
    cases["empty"] = record([])
    cases["pair"] = record([(0, 0), (5, 7)])
    with gzip.open(HERE / "conflicts_golden.json.gz", "wt", encoding="utf-8") as f:
        json.dump(cases, f, separators=(",", ":"))
    print({k: (v["triples"], v["violating_lines"], v["max_line_occupancy"]) for k, v in list(cases.items())[-16:]})


if __name__ == "__main__":
    main()
