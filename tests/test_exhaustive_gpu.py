"""Exhaustive 2-switch beam on the device (n3_exh_*) against trajectories of
the reference's own gpu_exhaustive_beam_search (tests/golden/exhaustive_golden.npz,
made by make_golden_exhaustive.py): every generation's best scores, evaluation
count, elite scores and elites, and the final result."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from no_three_in_line_b200 import gpu_exhaustive_beam as gx
from no_three_in_line_b200.state import PairPermutations

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "exhaustive_golden.npz"


def load(name):
    with np.load(GOLDEN) as z:
        return {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}


@pytest.mark.parametrize("name", ["a", "b", "c"])
def test_trajectory_matches_the_reference(cuda, name):
    g = load(name)
    snaps = []
    extra = g["extra"] if len(g["extra"]) else None
    res = gx.gpu_exhaustive_beam_search(
        PairPermutations(tuple(int(x) for x in g["initial_p"]), tuple(int(x) for x in g["initial_q"])),
        seed=int(g["seed"]), generations=int(g["generations"]), elite_size=int(g["elite_size"]),
        energy_window=int(g["energy_window"]), initial_elites=extra, global_every=int(g["global_every"]),
        report_every=1, callback=snaps.append)
    assert [s.generation for s in snaps] == g["generation"].tolist()
    for k, s in enumerate(snaps):
        assert s.generation_best == g["generation_best"][k], (name, k)
        assert s.best_score == g["best_score"][k], (name, k)
        assert s.evaluations == g["evaluations"][k], (name, k)
        want = g["elite_scores"][k]
        assert list(s.elite_scores) == want[want >= 0].tolist(), (name, k)
        assert np.array_equal(s.elite_values, g["elites"][k][:len(s.elite_values)].astype(np.int32)), (name, k)
    assert res.score == int(g["result_score"]) and res.generations == int(g["result_generations"])
    assert res.evaluations == int(g["result_evaluations"])
    assert list(res.state.P) == g["result_p"].tolist() and list(res.state.Q) == g["result_q"].tolist()


def test_argument_checks(cuda):
    s = PairPermutations(tuple(range(4)), (1, 2, 3, 0))
    with pytest.raises(ValueError):
        gx.gpu_exhaustive_beam_search(s, seed=1, generations=0, elite_size=4, energy_window=2)
    with pytest.raises(ValueError):
        gx.gpu_exhaustive_beam_search(s, seed=1, generations=2, elite_size=4, energy_window=2,
                                      initial_elites=np.zeros((2, 3, 2), np.int32))
