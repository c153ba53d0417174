"""Multi-point moves on the GPU: three-cycle scores (accelerated.py:196-276)
and four-cycle / double-switch scans (gpu_neighborhood.py:70-211) against the
reference's own outputs (tests/golden/neighborhood_golden.npz) and the CPU
oracle.  Integer work: bit-exact."""
from __future__ import annotations

from random import Random

import numpy as np
import pytest

from no_three_in_line_b200 import accelerated, gpu_neighborhood, state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb(golden):
    return golden("neighborhood_golden.npz")


def test_three_cycles_match_reference(cuda, nb):
    tags = sorted({k[:-2] for k in nb if k.startswith("tc_") and k.endswith("_p")})
    for tag in tags:
        p, q = nb[tag + "_p"], nb[tag + "_q"]
        score, bad = accelerated.score_and_badness(p, q)
        cand = accelerated.legal_three_cycle_candidates(p, q, int(nb[tag + "_anchor"]))
        assert np.array_equal(cand, nb[tag + "_cand"]), tag
        got = accelerated.evaluate_three_cycles(p, q, cand, score, bad)
        assert np.array_equal(got, nb[tag + "_scores"]), tag


@pytest.mark.parametrize("n", [5, 9, 33, 60, 75])
def test_three_cycles_match_oracle(cuda, oracle, n):
    s = state.random_state(n, Random(500 + n))
    p, q = np.asarray(s.P, np.int32), np.asarray(s.Q, np.int32)
    score, bad = oracle.score_and_badness(p, q)
    for anchor in (0, 2 * n - 1, n):
        cand = oracle.legal_three_cycle_candidates(p, q, anchor)
        if len(cand) == 0:
            continue
        ref = oracle.three_cycles(p, q, cand, score, bad)
        assert np.array_equal(accelerated.evaluate_three_cycles(p, q, cand, score, bad), ref)
    # a candidate the generator would not make (repeated column) scores the sentinel
    bogus = np.asarray([[0, 2, 2, 0], [0, 1, 4, 0]], np.int32)
    assert (accelerated.evaluate_three_cycles(p, q, bogus, score, bad) == 1 << 60).all()


def test_scans_match_reference(cuda, nb):
    for n, a in nb["nb_cases"]:
        tag = f"nb_n{n}_a{a}"
        s = state.PairPermutations(tuple(nb[tag + "_p"].tolist()), tuple(nb[tag + "_q"].tolist()))
        for kind, fn in (("four", gpu_neighborhood.best_four_cycle), ("double", gpu_neighborhood.best_double_switch)):
            r = fn(s, int(a))
            assert (r.score, r.evaluated, r.legal) == tuple(map(int, nb[f"{tag}_{kind}"])), (tag, kind)
            assert list(r.state.P) == nb[f"{tag}_{kind}_P"].tolist(), (tag, kind)
            assert list(r.state.Q) == nb[f"{tag}_{kind}_Q"].tolist(), (tag, kind)
    picks = gpu_neighborhood.bad_anchor_indices(
        state.PairPermutations(tuple(nb["nb_n14_a8_p"].tolist()), tuple(nb["nb_n14_a8_q"].tolist())), 2)
    assert picks == nb["nb_n14_anchors"].tolist()


@pytest.mark.parametrize("n,seed", [(7, 1), (21, 2), (26, 3)])
def test_scans_match_oracle(cuda, oracle, n, seed):
    s = state.random_state(n, Random(seed))
    p, q = np.asarray(s.P, np.int32), np.asarray(s.Q, np.int32)
    for a in (0, 2 * n - 1):
        for kind, fn in (("four", gpu_neighborhood.best_four_cycle), ("double", gpu_neighborhood.best_double_switch)):
            best, ev, lg, P, Q = oracle.neighborhood_scan(p, q, a, kind=kind)
            r = fn(s, a)
            assert (r.score, r.evaluated, r.legal) == (best, ev, lg), (n, a, kind)
            ref = state.points_to_permutations([(i, int(P[i])) for i in range(n)] + [(i, int(Q[i])) for i in range(n)],
                                               n)
            assert r.state == ref, (n, a, kind)


def test_scan_at_full_size_is_exact(cuda):
    """n = 75: 3.1 M four-cycles and 1.6 M double switches through a bad anchor;
    the winners are re-counted by both device scorers inside the call."""
    s = state.random_state(75, Random(91001))
    a = gpu_neighborhood.bad_anchor_indices(s, 1)[0]
    r4 = gpu_neighborhood.best_four_cycle(s, a)
    r2 = gpu_neighborhood.best_double_switch(s, a)
    assert r4.evaluated == 64824 * 48 and r2.evaluated == 64824 * 24
    base = accelerated.score_and_badness(np.asarray(s.P), np.asarray(s.Q))[0]
    assert r4.score < base and r2.score < base
