"""Badness-biased proposals and the umbrella restraint on the GPU
(tempering.py:49-63, 91-97, 173-174): every chain replayed bit for bit by the
CPU oracle, the distance kept exact, exchanges refused under an umbrella,
the learned candidate draw with the same bias, and checkpoints in the
reference's format."""
from __future__ import annotations

import json

import numpy as np
import pytest

from no_three_in_line_b200 import learned, state, tempering

pytestmark = pytest.mark.gpu


def snapshot(ch) -> dict:
    g = lambda x: x.cpu().numpy()  # noqa: E731
    return {"cols": g(ch.cols).astype(np.int32), "bad": g(ch.badness_dev), "E": g(ch.energy),
            "bestE": g(ch.best_energy), "best_cols": g(ch.best_cols).astype(np.int32), "temp_of": g(ch.temp_of),
            "chain_at": g(ch.chain_at), "counter": g(ch.counter).astype(np.uint64),
            "accepted": g(ch.accepted_dev).astype(np.uint32), "ladder_n": g(ch.ladder_n),
            "ladder_round": g(ch.ladder_round).astype(np.uint32),
            "ladder_exch": g(ch.ladder_exchanges).astype(np.uint32), "removed": g(ch.removed_dev)}


def assert_same(a: dict, b: dict, keys=None):
    for k in keys or a:
        assert np.array_equal(np.asarray(a[k]).astype(np.int64), np.asarray(b[k]).astype(np.int64)), k


def make_chains(n, chains, L, seed=7, tmin=0.05, tmax=5.0, base_seed=91001):
    p, q = state.seeded_population(n, chains, base_seed=base_seed)
    temps = np.tile(tempering.geometric_ladder(tmin, tmax, L), chains // L)
    return tempering.TemperingChains(state.pq_to_columns(p, q), temps, seed, ladder_size=L)


def replay(ch, before, *, umbrella=False, **kw):
    from oracle import oracle

    extra = {}
    if umbrella:
        extra = dict(reference=np.pad(ch.reference_host, (0, 150 - len(ch.reference_host))),
                     umbrella=tempering.umbrella_coefficients(ch.strengths, ch.centers),
                     frac=ch.frac_table.cpu().numpy().view(np.uint32))
    return oracle.temper_run(before, ladder_size=ch.L, acc=ch.acc_table.cpu().numpy().view(np.uint32),
                             exch=ch.exch_table.cpu().numpy().view(np.uint32), seed=ch.seed, **kw, **extra)


@pytest.mark.parametrize("bad_bias", [0, 50, 85, 100])
def test_biased_proposals_replay_exactly(cuda, bad_bias):
    ch = make_chains(20, 8, 4, seed=23)
    before = snapshot(ch)
    ch.run(30, exchange_every=3, chains_per_block=4, graph=False, bad_bias=bad_bias)
    ref = replay(ch, before, rounds=10, round_sweeps=3, bad_bias=bad_bias)
    assert_same(snapshot(ch), ref, [k for k in before if k != "removed"])
    assert int(snapshot(ch)["accepted"].sum()) > 0
    ch.validate()


def test_biased_proposals_n75_cluster_ladder(cuda):
    """n = 75, ladders of 16 split over 2-CTA clusters, bias 85, graph capture."""
    ch = make_chains(75, 32, 16, seed=2025)
    before = snapshot(ch)
    ch.run(4, exchange_every=2, chains_per_block=8, graph=True, bad_bias=85)
    ref = replay(ch, before, rounds=2, round_sweeps=2, bad_bias=85)
    assert_same(snapshot(ch), ref, [k for k in before if k != "removed"])
    ch.validate()


def test_bias_lowers_energy_faster_than_uniform(cuda):
    """Same chains, same proposals budget: badness-weighted u reaches lower E."""
    best = {}
    for bias in (0, 85):
        ch = make_chains(75, 64, 16, seed=5)
        ch.run(200, exchange_every=10, sweeps_per_launch=100, bad_bias=bias)
        ch.validate()
        best[bias] = int(ch.best_energy.min().item())
    assert best[85] < best[0], best


@pytest.mark.parametrize("bad_bias", [0, 85])
def test_umbrella_replays_exactly(cuda, bad_bias):
    ch = make_chains(20, 8, 4, seed=31, base_seed=91301)
    ch.centers = np.repeat(np.linspace(0, 12, 2), 4).astype(np.float32)
    ch.strengths.fill(0.5)
    before = snapshot(ch)
    ch.advance(300, bad_bias)
    ref = replay(ch, before, rounds=1, round_proposals=300, exchange=False, bad_bias=bad_bias, umbrella=True)
    assert_same(snapshot(ch), ref)
    ch.validate()  # energies, badness and the distance to the reference state
    # run(): rounds without exchanges, in a CUDA graph
    before = snapshot(ch)
    ch.run(20, exchange_every=5, graph=True, exchange=False, bad_bias=bad_bias)
    ref = replay(ch, before, rounds=4, round_sweeps=5, exchange=False, bad_bias=bad_bias, umbrella=True)
    assert_same(snapshot(ch), ref)
    ch.validate()
    removed = ch.removed_points.cpu().numpy()
    assert removed[:4].mean() < removed[4:].mean()  # the restraint pulls each ladder toward its centre


def test_umbrella_disables_exchange(cuda):
    ch = make_chains(20, 8, 4, seed=3)
    ch.strengths.fill(0.2)
    with pytest.raises(ValueError, match="disabled with umbrella"):
        ch.exchange(4)
    with pytest.raises(ValueError, match="disabled with umbrella"):
        ch.run(10, exchange_every=5)
    ch.strengths.fill(0.0)
    ch.exchange(4)


def test_distance_recounted_after_unrestrained_moves(cuda):
    """Moves made without an umbrella leave the distance stale; switching the
    umbrella on recounts it from the states before the first restrained move."""
    ch = make_chains(20, 8, 4, seed=41)
    ch.run(20, exchange_every=5, graph=False)
    ch.centers = np.full(8, 6.0, np.float32)
    ch.strengths.fill(1.0)
    ch.advance(100)
    ch.validate()
    want = tempering.reference_distance(ch.reference_host, ch.cols.cpu().numpy())
    assert np.array_equal(ch.removed_dev.cpu().numpy(), want)


def test_learned_candidates_follow_the_bias_rule(cuda, oracle):
    ch = make_chains(75, 32, 16, seed=4)
    lp = learned.LearnedProposal(ch, seed=9, ring_capacity=1 << 12, batch=256, bad_bias=85)
    lp.propose_scores()
    cand = lp.cand.cpu().numpy()
    cols = ch.cols.cpu().numpy()
    bad = ch.badness_dev.cpu().numpy()
    k0, k1 = lp.seed & 0xFFFFFFFF, lp.seed >> 32
    biased = 0
    for c in (0, 5, 17, 31):
        m = 150
        total = int(bad[c, :m].sum())
        for j in range(128):
            r = oracle.philox4x32_10([0, 0, c, 0xC0000000 | j], k0, k1)
            u, v = (r[0] * m) >> 32, (r[1] * m) >> 32
            if total > 0 and (r[2] * 100) >> 32 < 85:
                u = oracle.bias_slot(bad[c], m, (r[3] * total) >> 32)
                biased += 1
            legal = (u >> 1) != (v >> 1) and cols[c, u] != cols[c, v] and cols[c, u ^ 1] != cols[c, v] and \
                cols[c, v ^ 1] != cols[c, u]
            code = int(cand[c, j])
            assert (code & 0xFF, (code >> 8) & 0xFF, code < 0) == (u, v, legal), (c, j)
    assert biased > 300
    for _ in range(3):
        lp.step()
    ch.validate()


def test_restores_a_checkpoint_in_the_reference_format(cuda, tmp_path, oracle):
    """The keys and dtypes the reference's save writes (tempering.py:206-212)."""
    R, L, n = 8, 4, 20
    p, q = state.seeded_population(n, R, base_seed=92001)
    cols = state.pq_to_columns(p, q).astype(np.int32)
    scores = np.empty(R, np.int32)
    bad = np.empty((R, 2 * n), np.int32)
    for i in range(R):
        scores[i], bad[i] = oracle.score_columns(cols[i])
    temps = np.tile(np.geomspace(0.2, 4.0, L), R // L).astype(np.float32)
    reference = cols[0].copy()
    removed = tempering.reference_distance(reference, cols)
    host_rng = np.random.default_rng(11)
    arrays = dict(columns=cols, badness=bad, scores=scores,
                  rngs=host_rng.integers(1, 2 ** 64 - 1, size=R, dtype=np.uint64), best_columns=cols.copy(),
                  best_scores=scores - 1, accepted=np.arange(R, dtype=np.int32), reference=reference,
                  removed_points=removed, centers=np.linspace(0, 5, R).astype(np.float32),
                  strengths=np.zeros(R, np.float32))
    path = tmp_path / "checkpoint.npz"
    np.savez_compressed(path, **arrays, temperatures=temps, round=np.asarray(7),
                        host_rng=np.asarray(json.dumps(host_rng.bit_generator.state)))
    ch = tempering.TemperingChains.restore(path)
    assert ch.L == L and ch.round == 7
    assert np.array_equal(ch.scores.cpu().numpy(), scores)
    assert np.array_equal(ch.badness.cpu().numpy(), bad)
    assert np.array_equal(ch.best_scores.cpu().numpy(), scores - 1)
    assert np.array_equal(ch.accepted.cpu().numpy(), np.arange(R))
    assert np.array_equal(ch.removed_points.cpu().numpy(), removed)
    assert np.allclose(ch.centers, arrays["centers"])
    ch.run(10, exchange_every=5, graph=False, bad_bias=50)
    ch.validate()
    # a checkpoint whose energies disagree with its states is refused
    arrays["scores"] = scores + 1
    np.savez_compressed(path, **arrays, temperatures=temps, round=np.asarray(7),
                        host_rng=np.asarray(json.dumps(host_rng.bit_generator.state)))
    with pytest.raises(AssertionError):
        tempering.TemperingChains.restore(path)
