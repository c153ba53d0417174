"""Tempering with 2-, 4- and 8-warp teams per chain (threads_per_chain 64,
128, 256): the same trajectories as one warp per chain, replayed bit for bit
by the CPU oracle, for uniform and badness-biased proposals, the umbrella
restraint, mixed sizes and split ladders; and the autotuner's search over
team widths."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from no_three_in_line_b200 import _lib, autotune, state, tempering

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


NO_REMOVED = ["cols", "bad", "E", "bestE", "best_cols", "temp_of", "chain_at", "counter", "accepted", "ladder_n",
              "ladder_round", "ladder_exch"]


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


@pytest.mark.parametrize("tpc", [64, 128, 256])
@pytest.mark.parametrize("bad_bias", [0, 85])
def test_n75_teams_replay_exactly(cuda, tpc, bad_bias):
    """n = 75, ladders of 16 split over clusters (cpb 8 at 64 threads: 2 CTAs;
    cpb 4 at 128 threads: 4 CTAs; cpb 2 at 256 threads: 8 CTAs), exchanges
    every 2 sweeps."""
    ch = make_chains(75, 32, 16, seed=2026)
    before = snapshot(ch)
    ch.run(4, exchange_every=2, graph=False, bad_bias=bad_bias, threads_per_chain=tpc)
    ref = replay(ch, before, rounds=2, round_sweeps=2, bad_bias=bad_bias)
    after = snapshot(ch)
    assert_same(after, ref, NO_REMOVED)
    assert after["accepted"].sum() > 0 and after["ladder_exch"].sum() > 0
    ch.validate()


def test_team_width_and_layout_do_not_change_results(cuda):
    """Same seed: teams of 1, 2 and 4 warps, several chains per CTA, one launch
    or split launches, eager or graph: identical chains."""
    runs = []
    for tpc, cpb, per_launch, graph in [(32, 16, 40, False), (64, 8, 40, False), (64, 4, 10, True),
                                        (128, 4, 20, False), (128, 2, 40, True), (256, 2, 20, False)]:
        ch = make_chains(40, 64, 16, seed=99)
        ch.run(40, exchange_every=10, chains_per_block=cpb, sweeps_per_launch=per_launch, graph=graph,
               threads_per_chain=tpc)
        runs.append(snapshot(ch))
        ch.validate()
    for r in runs[1:]:
        assert_same(runs[0], r)


@pytest.mark.parametrize("tpc", [64, 128, 256])
def test_small_grid_teams_replay(cuda, tpc):
    """n = 12 (24 slots): most threads of a 64- or 128-thread team own no slot."""
    ch = make_chains(12, 8, 4, seed=11)
    before = snapshot(ch)
    ch.run(30, exchange_every=3, chains_per_block=min(4, 512 // tpc), graph=False, threads_per_chain=tpc)
    assert_same(snapshot(ch), replay(ch, before, rounds=10, round_sweeps=3), NO_REMOVED)
    ch.validate()


@pytest.mark.parametrize("tpc", [64, 256])
def test_umbrella_teams_replay(cuda, tpc):
    ch = make_chains(20, 8, 4, seed=31, base_seed=91301)
    ch.centers = np.repeat(np.linspace(0, 12, 2), 4).astype(np.float32)
    ch.strengths.fill(0.5)
    ch.threads_per_chain = tpc
    before = snapshot(ch)
    ch.advance(300, 85)
    ref = replay(ch, before, rounds=1, round_proposals=300, exchange=False, bad_bias=85, umbrella=True)
    assert_same(snapshot(ch), ref)
    ch.validate()


def test_mixed_sizes_teams_replay(cuda):
    L = 4
    groups = []
    for k, n in enumerate([40, 52, 60, 68, 75]):
        p, q = state.seeded_population(n, L, base_seed=91001 + 100 * k)
        groups.append((n, state.pq_to_columns(p, q)))
    ch = tempering.TemperingChains.mixed(groups, tempering.geometric_ladder(0.05, 5.0, L), seed=5)
    before = snapshot(ch)
    ch.run(4, exchange_every=2, chains_per_block=4, graph=False, threads_per_chain=64)
    assert_same(snapshot(ch), replay(ch, before, rounds=2, round_sweeps=2), NO_REMOVED)
    ch.validate()


def test_launch_shape_arguments_are_checked(cuda):
    ch = make_chains(20, 16, 16, seed=1)
    with pytest.raises(ValueError, match="32, 64, 128 or 256"):
        ch.run(2, exchange_every=2, threads_per_chain=96, graph=False)
    # 16 chains x 2 warps = 32 warps per CTA: refused by the library
    cfg = ch._config(rounds=1, round_sweeps=1, chains_per_block=16, threads_per_chain=64)
    d = ch._descriptor()
    rc = _lib.lib().n3_temper_run(ctypes.byref(d), ctypes.byref(cfg), _lib.stream_ptr())
    assert rc == _lib.N3_ERR_ARG
    cfg = ch._config(rounds=1, round_sweeps=1, chains_per_block=4, threads_per_chain=96)
    rc = _lib.lib().n3_temper_run(ctypes.byref(d), ctypes.byref(cfg), _lib.stream_ptr())
    assert rc == _lib.N3_ERR_ARG


def test_autotuner_searches_team_widths(cuda):
    """128 chains in ladders of 16 (the reference CLI's default shape): every
    (threads per chain, cpb) pair is timed, and the result is a valid shape."""
    ch = make_chains(75, 128, 16, seed=3, tmin=0.2, tmax=4.0)
    tune = autotune.autotune(ch, probe_sweeps=4, exchange_every=2)
    widths = {int(k.split("x")[0]) for k in tune.candidates}
    assert widths == {32, 64, 128, 256}
    assert tune.threads_per_chain in (32, 64, 128, 256)
    assert tune.chains_per_block in autotune._valid_cpb(16, 8, tune.threads_per_chain)
    assert f"{tune.threads_per_chain}x{tune.chains_per_block}" in tune.candidates
    # the tuner worked on copies: the chain set has not moved
    assert int(ch.counter.cpu().numpy().astype(np.uint64).sum()) == 0
