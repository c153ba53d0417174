"""Autotuner for the tempering launch (threads per chain, chains per CTA,
sweeps per launch, and per-size sweeps for mixed-size launches).

The reference sizes its launches by a fixed rule (one 128-thread block per
replica, src/no_three_75/tempering.py:161; population `1 << bits(SMs * 2048)`,
src/no_three_75/hardware.py:48-80).  Here the choices are measured:

* threads per chain (32, 64, 128 or 256) and chains per CTA (`cpb`), searched
  together: every pair the ladder admits (at most 16 warps per CTA; cpb a
  divisor of L with at most 8 CTAs per cluster, or a multiple of L) is timed on
  a copy of the chains and the fastest kept.  A team of 2, 4 or 8 warps shares
  one chain's direction histogram (one 8-bit counter per gcd-reduced
  direction, 6.8 KB of shared memory per chain) and splits its 2n slots, so a
  proposal takes fewer dependent steps at the price of barriers and fewer
  chains per SM: wider teams win when there are too few chains to fill the
  GPU's warps (the reference's default of 128 replicas), one warp per chain
  when there are thousands.
* per-size sweeps per launch: in one mixed-size launch every CTA runs its own
  ladders' rounds, and the launch ends with its slowest CTA.  The tuner times
  each size alone, then gives each size a number of sweeps proportional to its
  measured sweep rate, so that all CTAs finish together; sizes therefore advance
  at different sweep rates but the GPU is not left idle behind the largest n.
* sweeps per launch: long enough that the launch cost is below 1 % of the
  launch, short enough that a target hit or a time limit is noticed quickly.

Tuning never changes results: chains draw their randomness by (seed, chain,
proposal index), so any cpb or launch split gives the same trajectories.
"""
from __future__ import annotations

import json
import time
from dataclasses import asdict, dataclass, field
from pathlib import Path

import numpy as np

from . import _lib
from .tempering import TemperingChains


@dataclass
class TuneResult:
    threads_per_chain: int
    chains_per_block: int
    exchange_every: int
    sweeps_per_launch: int                 # sweeps of the slowest size per launch
    ladder_sweeps: list[int] | None        # per ladder, for mixed sizes (else None)
    size_sweeps: dict[int, int] = field(default_factory=dict)
    deltas_per_s: dict[int, float] = field(default_factory=dict)   # measured, per grid size
    total_deltas_per_s: float = 0.0
    candidates: dict[str, float] = field(default_factory=dict)     # "threads x cpb" -> total deltas/s

    def save(self, path) -> None:
        Path(path).write_text(json.dumps(asdict(self), indent=1) + "\n")


def _valid_cpb(L: int, ladders: int, threads_per_chain: int = 32) -> list[int]:
    """Chains per CTA that the launch admits for this ladder and team width."""
    cap = 16 // (threads_per_chain // 32)
    out = []
    for cpb in range(1, cap + 1):
        if cpb < L:
            if L % cpb == 0 and L // cpb <= 8:
                out.append(cpb)
        elif cpb % L == 0 and ladders % (cpb // L) == 0:
            out.append(cpb)
    return out


def _shapes(L: int, ladders: int) -> list[tuple[int, int]]:
    """(threads per chain, chains per CTA) pairs to time."""
    return [(tpc, cpb) for tpc in (32, 64, 128, 256) for cpb in _valid_cpb(L, ladders, tpc)]


def _clone(ch: TemperingChains, rows=None) -> TemperingChains:
    """A fresh chain set with the same states, temperatures and seed."""
    sel = np.arange(ch.cols.shape[0]) if rows is None else np.asarray(rows)
    lad = np.unique(sel // ch.L)
    cols = ch.cols.cpu().numpy()[sel]
    temps = np.tile(ch.ladder_temperatures, len(lad))
    return TemperingChains(cols if len(np.unique(ch.ladder_n_host[lad])) > 1 else cols[:, :2 * int(ch.ladder_n_host[lad[0]])],
                           temps, ch.seed, ladder_size=ch.L, ladder_n=ch.ladder_n_host[lad])


def _timed(ch: TemperingChains, sweeps, *, exchange_every, cpb, ladder_sweeps=None, tpc=32) -> float:
    t = _lib.torch()
    ch.run(exchange_every, exchange_every=exchange_every, chains_per_block=cpb, graph=False,
           ladder_sweeps=None if ladder_sweeps is None else np.minimum(ladder_sweeps, exchange_every),
           threads_per_chain=tpc)
    t.cuda.synchronize()
    res = ch.run(sweeps, exchange_every=exchange_every, chains_per_block=cpb, graph=False,
                 ladder_sweeps=ladder_sweeps, threads_per_chain=tpc)
    return res.seconds


def autotune(ch: TemperingChains, *, exchange_every: int = 10, probe_sweeps: int = 20,
             launch_seconds: float = 0.05) -> TuneResult:
    """Measure and choose the launch parameters for the chain set `ch` (which
    is not modified: all probes run on copies)."""
    L = ch.L
    sizes = sorted(int(n) for n in np.unique(ch.ladder_n_host))
    ladders_of = {n: np.nonzero(ch.ladder_n_host == n)[0] for n in sizes}
    # 1. per-size sweep rate, each size alone, default cpb
    rate = {}
    for n in sizes:
        rows = np.concatenate([np.arange(l * L, (l + 1) * L) for l in ladders_of[n]])
        sub = _clone(ch, rows)
        secs = _timed(sub, probe_sweeps, exchange_every=exchange_every, cpb=sub.default_chains_per_block())
        rate[n] = probe_sweeps / secs  # sweeps per second for this size's ladders
    # 2. per-size sweeps so that every CTA of a mixed launch runs for about as long
    slow = min(rate.values())
    base = probe_sweeps
    size_sweeps = {n: max(exchange_every, int(round(base * rate[n] / slow / exchange_every)) * exchange_every)
                   for n in sizes}
    ladder_sweeps = None
    if len(sizes) > 1:
        ladder_sweeps = [size_sweeps[int(n)] for n in ch.ladder_n_host]
    # 3. threads per chain and chains per CTA
    candidates = {}
    best = None
    for tpc, cpb in _shapes(L, len(ch.ladder_n_host)):
        if ladder_sweeps is not None and cpb > L:
            ls = np.asarray(ladder_sweeps).reshape(-1, cpb // L)
            if np.any(ls != ls[:, :1]):
                continue
        sub = _clone(ch)
        secs = _timed(sub, base, exchange_every=exchange_every, cpb=cpb, ladder_sweeps=ladder_sweeps, tpc=tpc)
        props = sum(size_sweeps[n] * 2 * n * L * len(ladders_of[n]) for n in sizes) if ladder_sweeps else \
            base * 2 * sizes[0] * ch.cols.shape[0]
        key = f"{tpc}x{cpb}"
        candidates[key] = props / secs
        if best is None or candidates[key] > candidates[best[0]]:
            best = (key, tpc, cpb, secs)
    key, tpc, cpb, secs = best
    # 4. per-size deltas/s of the chosen layout and the sweeps per launch
    per_size = {n: size_sweeps[n] * 2 * n * L * len(ladders_of[n]) / secs for n in sizes} if ladder_sweeps else \
        {sizes[0]: candidates[key]}
    scale = max(1, int(launch_seconds / secs))
    spl = base * scale
    if ladder_sweeps is not None:
        ladder_sweeps = [s * scale for s in ladder_sweeps]
        size_sweeps = {n: s * scale for n, s in size_sweeps.items()}
    else:
        size_sweeps = {sizes[0]: spl}
    return TuneResult(tpc, cpb, exchange_every, spl, ladder_sweeps, size_sweeps, per_size,
                      float(sum(per_size.values())), candidates)
