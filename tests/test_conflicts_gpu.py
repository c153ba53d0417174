"""Device line analysis (n3_analyze_lines behind conflicts.analyze_points)
against the reference's outputs and the oracle: lines, keys, occupancies,
badness, slope histograms and weighted scores, bit for bit."""
from __future__ import annotations

from random import Random

import numpy as np
import pytest

from no_three_in_line_b200 import conflicts, gpu, state

from test_conflicts_oracle import as_expected, load_cases, weights_of

pytestmark = pytest.mark.gpu


def as_dict(m: conflicts.ConflictMetrics) -> dict:
    return {"triples": m.triples, "violating_lines": m.violating_lines,
            "max_line_occupancy": m.max_line_occupancy, "max_point_badness": m.max_point_badness,
            "weighted_score": m.weighted_score, "badness": list(m.badness),
            "lines": [(line.key, line.points, line.triples) for line in m.lines],
            "slope_histogram": dict(m.slope_histogram)}


def test_every_fixture_case(cuda):
    for name, g in sorted(load_cases().items()):
        got = conflicts.analyze_points([tuple(p) for p in g["points"]], weights_of(g))
        assert as_dict(got) == as_expected(g), name


def test_population_of_n75_states_against_the_oracle_and_scorers(cuda, oracle):
    p, q = state.seeded_population(75, 96, base_seed=94001)
    sets = [state.PairPermutations(tuple(p[b]), tuple(q[b])).points() for b in range(96)]
    got = conflicts.analyze_population(sets)
    scores, bad = gpu.score_population_gpu(p, q, badness=True)
    for b in range(96):
        assert as_dict(got[b]) == oracle.analyze_points(sets[b])
        assert got[b].triples == scores[b]
    # slot-ordered point sets: badness equals the determinant scorer's per-slot badness
    cols = state.pq_to_columns(p, q)
    slot_sets = np.stack([np.stack([np.arange(150) // 2, cols[b]], 1) for b in range(96)])
    by_slot = conflicts.analyze_population(slot_sets)
    assert np.array_equal(np.asarray([m.badness for m in by_slot]), bad)


def test_capacity_overflow_is_rerun(cuda):
    g = load_cases()["block9"]
    got = conflicts.analyze_population([[tuple(p) for p in g["points"]]], capacity=7)[0]
    assert as_dict(got) == as_expected(g)


def test_reference_helpers(cuda):
    s = state.random_state(20, Random(91001))
    pts = s.points()
    assert conflicts.full_triple_score(pts) == int(gpu.score_population_gpu(
        np.asarray([s.P], np.int32), np.asarray([s.Q], np.int32))[0])
    done = 0
    for layer, a, b in [(0, 2, 7), (1, 0, 19), (0, 5, 6), (1, 3, 11)]:
        try:
            cand = s.swapped(layer, a, b)
        except ValueError:
            continue
        want = conflicts.full_triple_score(cand.points()) - conflicts.full_triple_score(pts)
        assert conflicts.reference_swap_delta(s, layer, a, b) == want
        done += 1
    assert done >= 2


def test_invalid_point_sets(cuda):
    with pytest.raises(ValueError, match="two distinct points"):
        conflicts.analyze_points([(0, 0), (1, 2), (0, 0)])
    with pytest.raises(ValueError, match="coordinates"):
        conflicts.analyze_points([(0, 0), (1, 2), (75, 3)])
    with pytest.raises(ValueError, match="at most"):
        conflicts.analyze_points([(r, c) for r in range(13) for c in range(13)])
    assert conflicts.analyze_points([]).triples == 0
