"""Device beam search (gpu_device_search.py:17-432): the CPU oracle against the
golden fixture written from the reference's own mutation kernel source,
rank_elites/elite_key and random.Random (tests/golden/make_golden_beam.py)."""
from __future__ import annotations

import numpy as np
import pytest


@pytest.fixture(scope="module")
def beam_golden(golden):
    return golden("beam_golden.npz")


def test_oracle_mutation_matches_reference_kernel(beam_golden, oracle):
    g = beam_golden
    pp, pq = g["mut_parent_p"], g["mut_parent_q"]
    _, pb = oracle.score_population(pp, pq, badness=True)
    cp_, cq_ = oracle.beam_mutate(pp, pq, pb, quality_count=2, population=64, active_strength=3, max_strength=6,
                                  bad_bias=85, seed=5, generation=2)
    assert np.array_equal(cp_, g["mut_child_p"]) and np.array_equal(cq_, g["mut_child_q"])


@pytest.mark.parametrize("name", ["a", "b"])
def test_oracle_beam_search_matches_reference(beam_golden, oracle, name):
    g = beam_golden
    n, seed, gens, pop, elite, max_s, window = map(int, g[f"{name}_config"])
    extra = g.get(f"{name}_extra")
    res = oracle.beam_search(g[f"{name}_initial_p"], g[f"{name}_initial_q"], extra, seed=seed, generations=gens,
                             population=pop, elite_size=elite, max_strength=max_s, energy_window=window)
    assert res["completed"] == int(g[f"{name}_completed"])
    assert res["best_score"] == int(g[f"{name}_best_score"])
    assert res["evaluations"] == int(g[f"{name}_evaluations"])
    assert np.array_equal(res["generation_best"], g[f"{name}_generation_best"])
    assert np.array_equal(np.stack(res["elite_scores"]), g[f"{name}_elite_scores"])
    assert np.array_equal(np.stack(res["elite_p"]), g[f"{name}_elite_p"])
    assert np.array_equal(np.stack(res["elite_q"]), g[f"{name}_elite_q"])
    assert np.array_equal(res["best_p_raw"], g[f"{name}_best_p_raw"])
