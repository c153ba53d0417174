"""Launch shapes the tempering autotuner searches (host logic, no GPU)."""
from __future__ import annotations

from no_three_in_line_b200 import autotune


def test_valid_chains_per_block_respect_warps_and_clusters():
    # ladder of 64 (the n = 75 tempering shape): clusters of at most 8 CTAs
    assert autotune._valid_cpb(64, 32, 32) == [8, 16]
    assert autotune._valid_cpb(64, 32, 64) == [8]
    assert autotune._valid_cpb(64, 32, 128) == []  # 16 CTAs per ladder: no cluster that large
    # ladder of 16, 8 ladders (128 replicas, the reference CLI's default)
    assert autotune._valid_cpb(16, 8, 32) == [2, 4, 8, 16]
    assert autotune._valid_cpb(16, 8, 64) == [2, 4, 8]
    assert autotune._valid_cpb(16, 8, 128) == [2, 4]
    assert autotune._valid_cpb(16, 8, 256) == [2]
    # ladders of 4: whole ladders per CTA when the ladder count allows it
    assert autotune._valid_cpb(4, 3, 32) == [1, 2, 4, 12]
    assert autotune._valid_cpb(4, 3, 128) == [1, 2, 4]


def test_shapes_cover_every_team_width():
    shapes = autotune._shapes(16, 8)
    assert {t for t, _ in shapes} == {32, 64, 128, 256}
    for tpc, cpb in shapes:
        assert cpb * tpc // 32 <= 16
    assert (128, 4) in shapes and (32, 16) in shapes and (64, 16) not in shapes


class _FakeChains:
    """What autotune() reads from a chain set: ladder size, per-ladder n, columns."""

    def __init__(self, L, ladder_n):
        import numpy as np

        self.L = L
        self.ladder_n_host = np.asarray(ladder_n, np.int32)
        self.cols = np.zeros((L * len(ladder_n), 150), np.int16)

    def default_chains_per_block(self, threads_per_chain=32):
        return 16 // (threads_per_chain // 32) if self.L >= 16 else self.L


def _fake_timer(cost):
    """A stand-in for the device timing: seconds = cost(tpc, cpb, chains) x sweeps."""

    def timed(ch, sweeps, *, exchange_every, cpb, ladder_sweeps=None, tpc=32):
        return cost(tpc, cpb, ch.cols.shape[0]) * sweeps

    return timed


def test_autotune_picks_the_fastest_shape(monkeypatch):
    import numpy as np

    monkeypatch.setattr(autotune, "_clone", lambda ch, rows=None: _FakeChains(
        ch.L, ch.ladder_n_host if rows is None else ch.ladder_n_host[np.unique(np.asarray(rows) // ch.L)]))
    # few chains: wider teams and smaller CTAs are faster
    monkeypatch.setattr(autotune, "_timed", _fake_timer(lambda tpc, cpb, c: 1.0 / tpc + 0.001 * cpb))
    tune = autotune.autotune(_FakeChains(16, [75] * 8), probe_sweeps=10, exchange_every=10)
    assert (tune.threads_per_chain, tune.chains_per_block) == (256, 2)
    assert set(tune.candidates) == {f"{t}x{c}" for t, c in autotune._shapes(16, 8)}
    assert tune.deltas_per_s[75] == tune.candidates["256x2"]
    # many chains: one warp per chain, large CTAs
    monkeypatch.setattr(autotune, "_timed", _fake_timer(lambda tpc, cpb, c: tpc / 32 - 0.01 * cpb))
    tune = autotune.autotune(_FakeChains(64, [75] * 32), probe_sweeps=10, exchange_every=10)
    assert (tune.threads_per_chain, tune.chains_per_block) == (32, 16)


def test_autotune_mixed_sizes_balances_sweeps(monkeypatch):
    import numpy as np

    monkeypatch.setattr(autotune, "_clone", lambda ch, rows=None: _FakeChains(
        ch.L, ch.ladder_n_host if rows is None else ch.ladder_n_host[np.unique(np.asarray(rows) // ch.L)]))

    def cost(tpc, cpb, chains):
        return 1e-4 * chains  # per sweep: proportional to the chains probed

    monkeypatch.setattr(autotune, "_timed", _fake_timer(cost))
    ch = _FakeChains(32, [40, 40, 75])
    tune = autotune.autotune(ch, probe_sweeps=20, exchange_every=10)
    # the n = 40 group (2 ladders) probes twice as slow per sweep as n = 75 (1 ladder)
    assert tune.size_sweeps[75] == 2 * tune.size_sweeps[40]
    assert tune.ladder_sweeps == [tune.size_sweeps[40]] * 2 + [tune.size_sweeps[75]]
    assert tune.threads_per_chain in (32, 64, 128)
