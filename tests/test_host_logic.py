"""Host-side logic that needs no GPU: status mapping, threshold tables,
ladder inference, state helpers, and that a planted oracle mistake is caught
by the comparisons the GPU tests use."""
from __future__ import annotations

import math

import numpy as np
import pytest

from no_three_in_line_b200 import _lib, state, tempering


def test_status_codes_map_to_reference_exceptions(monkeypatch):
    monkeypatch.setattr(_lib, "last_error", lambda: "planted")
    _lib.check(_lib.N3_OK, "x")
    for code, exc in [(_lib.N3_ERR_ARG, ValueError), (_lib.N3_ERR_RANGE, ValueError), (_lib.N3_ERR_STATE, ValueError),
                      (_lib.N3_ERR_MISMATCH, AssertionError), (_lib.N3_ERR_TIMEOUT, TimeoutError),
                      (_lib.N3_ERR_CUDA, RuntimeError)]:
        with pytest.raises(exc, match="planted"):
            _lib.check(code, "x")


def test_metropolis_and_exchange_tables():
    T = tempering.geometric_ladder(0.05, 5.0, 64)
    acc = tempering.metropolis_table(T)
    assert acc.dtype == np.uint32 and acc.shape[0] == 64
    # floor(2^32 exp(-dE/T)), below 1 at the last column for the hottest ladder rung
    assert acc[-1, 1] == math.floor(2 ** 32 * math.exp(-1 / 5.0))
    assert math.exp(-(acc.shape[1] - 1) / 5.0) * 2 ** 32 < 1.0
    assert np.all(np.diff(acc[:, 1:].astype(np.int64), axis=1) <= 0)
    ex = tempering.exchange_table(T)
    dbeta = 1 / T[0] - 1 / T[1]
    assert ex[0, 3] == math.floor(2 ** 32 * math.exp(-dbeta * 3))
    with pytest.raises(ValueError):
        tempering.exchange_table(T[::-1])


def test_ladder_inference():
    T = np.tile(tempering.geometric_ladder(0.2, 4.0, 16), 8)
    assert tempering.TemperingChains._infer_ladder(T) == 16
    with pytest.raises(ValueError):
        tempering.TemperingChains._infer_ladder(np.array([1.0, 0.5, 2.0]))


def test_state_helpers_round_trip():
    p, q = state.seeded_population(12, 3)
    cols = state.pq_to_columns(p, q)
    p2, q2 = state.columns_to_pq(cols)
    assert np.array_equal(p, p2) and np.array_equal(q, q2)
    for row in cols:
        state.check_two_factor(row)
        st = state.points_to_permutations(state.columns_to_points(row), 12)
        assert sorted(st.points()) == state.columns_to_points(row)
    bad = cols[0].copy()
    bad[1] = bad[0]
    with pytest.raises(ValueError):
        state.check_two_factor(bad)


def test_planted_oracle_mistake_is_caught(golden, oracle):
    """The exact-equality comparison the GPU parity tests use does fail when
    the checker (here: the oracle's output) carries one wrong count."""
    c1 = golden("c1_n20.npz")
    s = oracle.score_population(c1["p"], c1["q"], threads=0)
    assert np.array_equal(s, c1["E"])
    s[17] += 1
    assert not np.array_equal(s, c1["E"])
    ok, dE, dbad = oracle.walk_delta(state.pq_to_columns(c1["p"][0], c1["q"][0]), 0, 2)
    if ok:
        dbad[0] += 1
        assert int(dbad.sum()) != 3 * dE
