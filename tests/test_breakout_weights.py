"""Line-weighted energies of breakout search (breakout.py:39-86): the oracle
(CPU) and the device kernels (GPU) against the reference's own outputs
(tests/golden/breakout_golden.npz, written by make_golden_breakout.py)."""
from __future__ import annotations

from random import Random

import numpy as np
import pytest


@pytest.fixture(scope="module")
def bw(golden):
    return golden("breakout_golden.npz")


def cases(bw):
    return [f"w{k}" for k in range(int(bw["count"]))]


def test_oracle_matches_reference(bw, oracle):
    for tag in cases(bw):
        p, q, keys, vals = bw[tag + "_p"], bw[tag + "_q"], bw[tag + "_keys"], bw[tag + "_vals"]
        for i, u in enumerate(bw[tag + "_sel"]):
            got = oracle.weighted_switch_scores(p, q, int(u), bw[tag + "_raw"][i], keys, vals)
            assert np.array_equal(got, bw[tag + "_scores"][i]), (tag, u)
        assert oracle.weighted_state_score(p, q, int(bw[tag + "_raw_score"]), keys, vals) == int(bw[tag + "_state"])


@pytest.mark.gpu
def test_device_matches_reference(cuda, bw):
    from no_three_in_line_b200 import breakout

    for tag in cases(bw):
        p, q = bw[tag + "_p"], bw[tag + "_q"]
        weights = {tuple(map(int, k)): int(v) for k, v in zip(bw[tag + "_keys"], bw[tag + "_vals"])}
        for i, u in enumerate(bw[tag + "_sel"]):
            got = breakout.weighted_candidate_scores(p, q, int(u), bw[tag + "_raw"][i], weights)
            assert np.array_equal(got, bw[tag + "_scores"][i]), (tag, u)
        assert breakout.weighted_state_score(p, q, int(bw[tag + "_raw_score"]), weights) == int(bw[tag + "_state"])


@pytest.mark.gpu
def test_device_batch_matches_oracle(cuda, oracle):
    from no_three_in_line_b200 import breakout, state

    rng = Random(3)
    p, q = state.seeded_population(40, 300)
    keys = np.asarray([(rng.randint(-3, 3), rng.randint(-3, 3), rng.randint(-60, 60)) for _ in range(200)], np.int64)
    vals = np.asarray([rng.randint(0, 9) for _ in range(200)], np.int64)
    raw = oracle.score_population(p, q)
    weights = {tuple(map(int, k)): int(v) for k, v in zip(keys, vals)}
    keys = np.asarray(list(weights), np.int64)
    vals = np.asarray(list(weights.values()), np.int64)
    got = breakout.weighted_state_scores(p, q, raw.astype(np.int64), weights)
    ref = [oracle.weighted_state_score(p[b], q[b], int(raw[b]), keys, vals) for b in range(len(p))]
    assert np.array_equal(got, np.asarray(ref, np.int64))
    # no weight above 1: the raw scores come back unchanged
    assert np.array_equal(breakout.weighted_state_scores(p, q, raw.astype(np.int64), {(1, 0, -3): 1}), raw)
