"""Multi-point moves (accelerated.py:196-276, search.py:38-65,
gpu_neighborhood.py:70-211): the CPU oracle against the fixture written from
the reference's own functions (tests/golden/make_golden_neighborhood.py)."""
from __future__ import annotations

import numpy as np
import pytest


@pytest.fixture(scope="module")
def nb(golden):
    return golden("neighborhood_golden.npz")


def tc_tags(nb):
    return sorted({k[:-2] for k in nb if k.startswith("tc_") and k.endswith("_p")})


def test_oracle_three_cycles_match_reference(nb, oracle):
    for tag in tc_tags(nb):
        p, q = nb[tag + "_p"], nb[tag + "_q"]
        score, bad = oracle.score_and_badness(p, q)
        cand = oracle.legal_three_cycle_candidates(p, q, int(nb[tag + "_anchor"]))
        assert np.array_equal(cand, nb[tag + "_cand"]), tag
        assert np.array_equal(oracle.three_cycles(p, q, cand, score, bad), nb[tag + "_scores"]), tag


def test_oracle_neighborhood_scans_match_reference(nb, oracle):
    from no_three_in_line_b200 import state

    for n, a in nb["nb_cases"]:
        tag = f"nb_n{n}_a{a}"
        p, q = nb[tag + "_p"], nb[tag + "_q"]
        for kind in ("four", "double"):
            best, ev, lg, P, Q = oracle.neighborhood_scan(p, q, int(a), kind=kind)
            assert (best, ev, lg) == tuple(map(int, nb[f"{tag}_{kind}"])), (tag, kind)
            s = state.points_to_permutations([(r, int(P[r])) for r in range(n)] + [(r, int(Q[r])) for r in range(n)],
                                             int(n))
            assert list(s.P) == nb[f"{tag}_{kind}_P"].tolist() and list(s.Q) == nb[f"{tag}_{kind}_Q"].tolist()
