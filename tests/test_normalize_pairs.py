"""The host C routine n3_normalize_pairs (canonical P/Q of raw rows) against
state.points_to_permutations, the restatement of the reference's
state.py:47-85 (pinned there by the state tests): same P and Q for random
2-factors of every size, both column orders of a row, and the same refusals.
Host code only: no GPU."""
from __future__ import annotations

from random import Random

import numpy as np
import pytest

from no_three_in_line_b200 import state
from no_three_in_line_b200.gpu_device_search import _normalize_raw, normalize_rows


def random_rows(n, rng):
    s = state.random_state(n, rng)
    p, q = np.asarray(s.P, np.int32), np.asarray(s.Q, np.int32)
    swap = np.asarray([rng.random() < 0.5 for _ in range(n)])  # raw rows: either column first
    return np.where(swap, q, p), np.where(swap, p, q)


@pytest.mark.parametrize("n", [2, 3, 4, 5, 8, 20, 41, 75])
def test_same_pairs_as_points_to_permutations(n):
    rng = Random(1000 + n)
    rows = [random_rows(n, rng) for _ in range(40)]
    p = np.stack([r[0] for r in rows])
    q = np.stack([r[1] for r in rows])
    po, qo = normalize_rows(p, q)
    for b in range(len(rows)):
        points = [(r, int(p[b, r])) for r in range(n)] + [(r, int(q[b, r])) for r in range(n)]
        want = state.points_to_permutations(points, n)
        assert tuple(po[b].tolist()) == want.P and tuple(qo[b].tolist()) == want.Q
        got = _normalize_raw(p[b], q[b])
        assert got.P == want.P and got.Q == want.Q


def test_structured_states():
    n = 75
    r = np.arange(n)
    for p, q in [(r, (r + 1) % n), ((r + 1) % n, r), (r, (r + 37) % n), ((2 * r) % n, (2 * r + 1) % n)]:
        po, qo = normalize_rows(p, q)
        points = [(k, int(p[k])) for k in range(n)] + [(k, int(q[k])) for k in range(n)]
        want = state.points_to_permutations(points, n)
        assert tuple(po[0].tolist()) == want.P and tuple(qo[0].tolist()) == want.Q


def test_refuses_what_is_not_a_two_factor():
    n = 6
    p = np.asarray([0, 1, 2, 3, 4, 5], np.int32)
    with pytest.raises(ValueError):
        normalize_rows(p, p)  # a row with one column twice
    with pytest.raises(ValueError):
        normalize_rows(p, np.asarray([1, 2, 3, 4, 5, 5], np.int32))  # column 5 three times, column 0 once
    with pytest.raises(ValueError):
        normalize_rows(p, np.asarray([1, 2, 3, 4, 5, 6], np.int32))  # column outside the grid
    po, qo = normalize_rows(np.zeros((0, n), np.int32), np.zeros((0, n), np.int32))
    assert po.shape == (0, n) and qo.shape == (0, n)
