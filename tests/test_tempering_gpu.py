"""(c) Replica-exchange tempering on the GPU: every chain replayed bit for bit
by the CPU oracle (pair-formulation deltas, same Philox stream, same tables),
invariance to the launch layout, device audit, graphs, checkpoints."""
from __future__ import annotations

import numpy as np
import pytest

from no_three_in_line_b200 import state, tempering

pytestmark = pytest.mark.gpu


def snapshot(ch) -> dict:
    g = lambda x: x.cpu().numpy()  # noqa: E731
    return {"cols": g(ch.cols).astype(np.int32), "bad": g(ch.badness_dev), "E": g(ch.energy),
            "bestE": g(ch.best_energy), "best_cols": g(ch.best_cols).astype(np.int32), "temp_of": g(ch.temp_of),
            "chain_at": g(ch.chain_at), "counter": g(ch.counter).astype(np.uint64),
            "accepted": g(ch.accepted_dev).astype(np.uint32), "ladder_n": g(ch.ladder_n),
            "ladder_round": g(ch.ladder_round).astype(np.uint32),
            "ladder_exch": g(ch.ladder_exchanges).astype(np.uint32)}


def assert_same(a: dict, b: dict):
    for k in a:
        assert np.array_equal(np.asarray(a[k]).astype(np.int64), np.asarray(b[k]).astype(np.int64)), k


def make_chains(n, chains, L, seed=7, tmin=0.05, tmax=5.0):
    p, q = state.seeded_population(n, chains)
    temps = np.tile(tempering.geometric_ladder(tmin, tmax, L), chains // L)
    return tempering.TemperingChains(state.pq_to_columns(p, q), temps, seed, ladder_size=L)


def replay(ch, before, *, rounds=0, round_sweeps=0, round_proposals=0, exchange=True, ladder_rounds=None):
    from oracle import oracle

    return oracle.temper_run(before, ladder_size=ch.L, acc=ch.acc_table.cpu().numpy().view(np.uint32),
                             exch=ch.exch_table.cpu().numpy().view(np.uint32), seed=ch.seed, rounds=rounds,
                             round_sweeps=round_sweeps, round_proposals=round_proposals, exchange=exchange,
                             ladder_rounds=ladder_rounds)


def test_philox_known_answers(oracle):
    assert oracle.philox4x32_10([0, 0, 0, 0], 0, 0) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert oracle.philox4x32_10([0xFFFFFFFF] * 4, 0xFFFFFFFF, 0xFFFFFFFF) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                                            0x6D5451FD]


@pytest.mark.parametrize("cpb", [4, 2, 8])
def test_small_ladders_replay_exactly(cuda, cpb):
    """n=12, two ladders of 4: whole ladders per CTA (cpb 4, 8) and a ladder
    split over a 2-CTA cluster (cpb 2) all match the CPU replay."""
    ch = make_chains(12, 8, 4, seed=11)
    before = snapshot(ch)
    ch.run(30, exchange_every=3, chains_per_block=cpb, graph=False)
    after = snapshot(ch)
    ref = replay(ch, before, rounds=10, round_sweeps=3)
    assert_same(after, ref)
    assert after["accepted"].sum() > 0 and after["ladder_exch"].sum() > 0
    ch.validate()


def test_n75_ladder_of_16_replays_exactly(cuda):
    ch = make_chains(75, 32, 16, seed=2024)
    before = snapshot(ch)
    ch.run(4, exchange_every=2, graph=False)
    ref = replay(ch, before, rounds=2, round_sweeps=2)
    assert_same(snapshot(ch), ref)
    ch.validate()


def test_results_do_not_depend_on_launch_layout(cuda):
    """Same seed: one launch vs split launches vs a CUDA graph vs other cpb."""
    runs = []
    for cpb, per_launch, graph in [(16, 40, False), (8, 10, False), (16, 20, True), (4, 40, True)]:
        ch = make_chains(40, 64, 16, seed=99)
        ch.run(40, exchange_every=10, chains_per_block=cpb, sweeps_per_launch=per_launch, graph=graph)
        runs.append(snapshot(ch))
        ch.validate()
    for r in runs[1:]:
        assert_same(runs[0], r)


def test_mixed_sizes_one_launch_replay(cuda):
    L = 4
    groups = []
    for k, n in enumerate([40, 52, 60, 68, 75]):
        p, q = state.seeded_population(n, L, base_seed=91001 + 100 * k)
        groups.append((n, state.pq_to_columns(p, q)))
    ch = tempering.TemperingChains.mixed(groups, tempering.geometric_ladder(0.05, 5.0, L), seed=5)
    before = snapshot(ch)
    ch.run(4, exchange_every=2, chains_per_block=4, graph=False)
    assert_same(snapshot(ch), replay(ch, before, rounds=2, round_sweeps=2))
    ch.validate()


def test_per_ladder_sweeps(cuda):
    """Per-size sweeps-per-launch (the autotuner's load-balancing knob)."""
    L = 4
    groups = []
    for k, n in enumerate([20, 30]):
        p, q = state.seeded_population(n, 2 * L, base_seed=5000 + k * 10)
        groups.append((n, state.pq_to_columns(p, q)))
    ch = tempering.TemperingChains.mixed(groups, tempering.geometric_ladder(0.1, 4.0, L), seed=3)
    before = snapshot(ch)
    ch.run(20, exchange_every=2, chains_per_block=4, ladder_sweeps=[20, 20, 10, 10], graph=False)
    # ladders of n=20 ran 10 rounds, ladders of n=30 ran 5
    assert_same(snapshot(ch), replay(ch, before, round_sweeps=2, ladder_rounds=[10, 10, 5, 5]))


def test_reference_api_advance_exchange_save_restore(cuda, tmp_path):
    ch = make_chains(20, 8, 4, seed=17)
    before = snapshot(ch)
    ch.advance(50)
    ref = replay(ch, before, rounds=1, round_proposals=50, exchange=False)
    assert_same(snapshot(ch), ref)
    n_ex = ch.exchange(4)
    ref2 = replay(ch, ref, rounds=1, round_proposals=0, exchange=True)
    assert_same(snapshot(ch), ref2)
    assert n_ex == int(ref2["ladder_exch"].sum())
    # replica-order views: row l*L+t holds the chain at temperature t
    scores = ch.scores.cpu().numpy()
    E = ch.energy.cpu().numpy()
    at = ch.chain_at.cpu().numpy()
    for r in range(8):
        assert scores[r] == E[(r // 4) * 4 + at[r]]
    path = tmp_path / "checkpoint.npz"
    ch.save(path)
    with np.load(path) as z:
        for key in ("columns", "badness", "scores", "rngs", "best_columns", "best_scores", "accepted",
                    "temperatures", "round"):
            assert key in z.files
    back = tempering.TemperingChains.restore(path)
    assert_same(snapshot(back), snapshot(ch))
    ch.run(10, exchange_every=5, graph=False)
    back.run(10, exchange_every=5, graph=False)
    assert_same(snapshot(back), snapshot(ch))


def test_target_hit_stops_the_run(cuda):
    ch = make_chains(30, 16, 8, seed=1)
    start = int(ch.energy.min().item())
    res = ch.run(2000, exchange_every=10, target=start - 40, sweeps_per_launch=100)
    assert res.hit is not None and res.best <= start - 40
    assert res.sweeps < 2000
    chain, counter, seconds = res.hit
    assert 0 <= chain < 16 and counter > 0 and 0 <= seconds < 600
    ch.validate()


def test_long_n75_run_audits_clean(cuda):
    """C3 shape in miniature: 64 temperatures (a 4-CTA cluster per ladder),
    200 sweeps; incremental energies and badness equal a full recompute."""
    ch = make_chains(75, 128, 64, seed=3)
    e0 = ch.energy.cpu().numpy().copy()
    res = ch.run(200, exchange_every=10, sweeps_per_launch=100)
    ch.validate()
    assert int(ch.error_word.item()) == 0
    assert res.best < int(e0.min())
    from no_three_in_line_b200 import gpu

    best = ch.best_columns.cpu().numpy()
    s = gpu.score_columns_gpu(best)
    assert np.array_equal(s, ch.best_energy.cpu().numpy())
