"""Replica-exchange tempering on the B200 (drop-in for ``no_three_75.tempering``).

``TemperingChains`` keeps the reference's constructor, methods and checkpoint
keys (src/no_three_75/tempering.py:119-225): ``advance`` (proposals without
exchange), ``exchange`` (one neighbour-exchange round), ``validate`` (full
recompute), ``save``/``restore`` (npz).  The native entry point is ``run``:
many rounds of proposals + on-device exchanges in one persistent kernel per
launch, optionally captured in a CUDA graph.

Differences from the reference, all deliberate:
* exchanges swap temperature labels between chains instead of copying
  states; ``columns``/``scores``/``badness`` are still returned in replica
  order (entry ``l*L + t`` is the state at temperature ``t`` of ladder ``l``);
* the RNG is Philox4x32-10 keyed by the seed, counter = (proposal, chain);
* Metropolis and exchange probabilities are compared as 32-bit integers
  against tables of ``floor(2^32 exp(-x))`` built here in float64, so runs are
  reproducible bit for bit (the CPU oracle replays them);
* chains of different grid sizes may share one launch (``mixed``).
"""
from __future__ import annotations

import ctypes
import json
import math
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib
from .state import MAX_N, check_two_factor, columns_to_points, points_to_permutations

STRIDE = 2 * MAX_N


class N3Chains(ctypes.Structure):
    _fields_ = [("n_chains", ctypes.c_int), ("ladder_size", ctypes.c_int),
                ("cols", ctypes.c_void_p), ("badness", ctypes.c_void_p), ("energy", ctypes.c_void_p),
                ("best_energy", ctypes.c_void_p), ("best_cols", ctypes.c_void_p), ("temp_of", ctypes.c_void_p),
                ("chain_at", ctypes.c_void_p), ("counter", ctypes.c_void_p), ("accepted", ctypes.c_void_p),
                ("ladder_n", ctypes.c_void_p), ("ladder_round", ctypes.c_void_p),
                ("ladder_exchanges", ctypes.c_void_p), ("acc_thresh", ctypes.c_void_p), ("acc_width", ctypes.c_int),
                ("exch_thresh", ctypes.c_void_p), ("exch_width", ctypes.c_int), ("global_best", ctypes.c_void_p),
                ("hit", ctypes.c_void_p), ("stop", ctypes.c_void_p), ("error_word", ctypes.c_void_p),
                ("reference", ctypes.c_void_p), ("removed", ctypes.c_void_p), ("umbrella", ctypes.c_void_p),
                ("acc_frac", ctypes.c_void_p)]


class N3TemperConfig(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("chains_per_block", ctypes.c_int), ("rounds", ctypes.c_int),
                ("ladder_rounds", ctypes.c_void_p), ("round_sweeps", ctypes.c_int),
                ("round_proposals", ctypes.c_int), ("exchange", ctypes.c_int), ("target_energy", ctypes.c_int),
                ("bad_bias", ctypes.c_int), ("threads_per_chain", ctypes.c_int)]


_lib.register("n3_temper_run", [ctypes.POINTER(N3Chains), ctypes.POINTER(N3TemperConfig), ctypes.c_void_p])
_lib.register("n3_temper_audit", [ctypes.POINTER(N3Chains), ctypes.c_void_p, ctypes.c_void_p])

_TWO32 = float(2 ** 32)


def metropolis_table(temperatures) -> np.ndarray:
    """uint32 [L, W]: entry [t, dE] = floor(2^32 exp(-dE / T_t)) (dE >= 1); a
    proposal with dE >= W is rejected (its probability is below 2^-32)."""
    T = np.asarray(temperatures, dtype=np.float64)
    W = int(math.ceil(T.max() * 32 * math.log(2))) + 2
    dE = np.arange(W, dtype=np.float64)
    p = np.exp(-dE[None, :] / T[:, None])
    tab = np.minimum(np.floor(p * _TWO32), _TWO32 - 1).astype(np.uint64).astype(np.uint32)
    tab[:, 0] = 0xFFFFFFFF
    return tab


def exchange_table(temperatures) -> np.ndarray:
    """uint32 [L-1, XW]: entry [t, d] = floor(2^32 exp(-(1/T_t - 1/T_t+1) d)), the
    reference's exchange probability exp(min(0, log_ratio)) (tempering.py:181-182)
    for an energy gap E(lower T) - E(higher T) = -d < 0."""
    T = np.asarray(temperatures, dtype=np.float64)
    dbeta = 1.0 / T[:-1] - 1.0 / T[1:]
    if np.any(dbeta <= 0):
        raise ValueError("ladder temperatures must increase")
    XW = int(math.ceil(32 * math.log(2) / dbeta.min())) + 2
    d = np.arange(XW, dtype=np.float64)
    p = np.exp(-dbeta[:, None] * d[None, :])
    tab = np.minimum(np.floor(p * _TWO32), _TWO32 - 1).astype(np.uint64).astype(np.uint32)
    tab[:, 0] = 0xFFFFFFFF
    return tab


def fraction_table(temperatures) -> np.ndarray:
    """uint32 [L, 768]: the fraction factors of the umbrella acceptance test,
    floor(2^32 exp(-k / (2^j T))) for j = 8, 16, 24 and k < 256.  An acceptance
    energy e = a + b / 2^24 (a, b integers, 0 <= b < 2^24) is accepted iff a
    32-bit uniform lies below acc[a] x f8[b >> 16] x f16[(b >> 8) & 255] x
    f24[b & 255] in 32-bit fixed point (a factor with index 0 is skipped)."""
    T = np.asarray(temperatures, dtype=np.float64)
    k = np.arange(256, dtype=np.float64)
    parts = [np.exp(-k[None, :] / (float(2 ** j) * T[:, None])) for j in (8, 16, 24)]
    tab = np.minimum(np.floor(np.concatenate(parts, 1) * _TWO32), _TWO32 - 1)
    return tab.astype(np.uint64).astype(np.uint32)


def umbrella_coefficients(strengths, centers) -> np.ndarray:
    """int64 [R, 2]: round(2^24 s) and round(2^24 * 2 s c) of each replica
    position's float32 strength s and centre c.  The acceptance energy of a
    move that changes the distance by dd at distance `removed` is then
    dE + (s_q (2 removed dd + dd^2) - c2s_q dd) / 2^24, the reference's
    dE + s (2 (removed - c) dd + dd^2) (tempering.py:93-94) in 2^-24 units."""
    s = np.asarray(strengths, dtype=np.float32).astype(np.float64)
    c = np.asarray(centers, dtype=np.float32).astype(np.float64)
    q = float(1 << 24)
    return np.stack([np.rint(q * s), np.rint(q * 2.0 * s * c)], 1).astype(np.int64)


def reference_distance(reference, rows) -> np.ndarray:
    """Points of the reference state missing from each slot-column row (the
    reference's removed_points, tempering.py:148-150)."""
    ref = np.asarray(reference).reshape(-1)
    rows = np.atleast_2d(np.asarray(rows))
    m = len(ref)
    r_pts = set((i // 2, int(c)) for i, c in enumerate(ref))
    return np.asarray([len(r_pts - set((i // 2, int(c)) for i, c in enumerate(row[:m]))) for row in rows], np.int32)


def geometric_ladder(tmin: float, tmax: float, size: int) -> np.ndarray:
    """The reference's ladder, np.geomspace(tmin, tmax, ladder) (tempering.py:263)."""
    return np.geomspace(tmin, tmax, size)


@dataclass
class RunResult:
    rounds: int
    sweeps: int
    proposals: int
    seconds: float
    best: int
    hit: tuple | None  # (chain, proposal counter, seconds since run start) of the first E <= target


class TemperingChains:
    """Device-resident replica-exchange chains (tempering.py:119-225)."""

    def __init__(self, columns, temperatures, seed: int, *, ladder_size: int | None = None, device=None,
                 ladder_n=None):
        t = _lib.torch()
        self.device = device if device is not None else _lib.require_device()
        cols = np.asarray(columns)
        temps = np.asarray(temperatures, dtype=np.float64)
        if cols.ndim != 2 or cols.shape[1] % 2 or not 4 <= cols.shape[1] <= STRIDE:
            raise ValueError("columns must have shape (replicas,2n), 2<=n<=75")
        R = cols.shape[0]
        if temps.shape != (R,) or np.any(~np.isfinite(temps)) or np.any(temps <= 0):
            raise ValueError("one positive finite temperature is required per replica")
        L = ladder_size or self._infer_ladder(temps)
        if L < 2 or R % L:
            raise ValueError("ladder_size must divide replica count")
        ladder = temps[:L]
        if not np.allclose(np.tile(ladder, R // L), temps):
            raise ValueError("temperatures must tile one increasing ladder")
        self.L = L
        self.ladder_temperatures = ladder
        self.temperatures_host = temps.astype(np.float32)
        if ladder_n is None:
            ladder_n = np.full(R // L, cols.shape[1] // 2, np.int32)
        self.ladder_n_host = np.asarray(ladder_n, np.int32)
        self.n = int(self.ladder_n_host.max())
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        # launch shape (threads that evaluate one chain's moves: 32, 64, 128
        # or 256; chains per CTA, None for the default), e.g. the autotuner's
        # choice; results do not depend on it
        self.threads_per_chain = 32
        self.chains_per_block = None
        padded = np.zeros((R, STRIDE), np.int16)
        for lad, n in enumerate(self.ladder_n_host):
            block = cols[lad * L:(lad + 1) * L, :2 * n]
            for row in block:
                check_two_factor(row)
            padded[lad * L:(lad + 1) * L, :2 * n] = block
        dev = self.device
        self.cols = t.from_numpy(padded).to(dev)
        self.badness_dev = t.zeros((R, STRIDE), dtype=t.int32, device=dev)
        self.energy = t.zeros(R, dtype=t.int32, device=dev)
        self._score_initial()
        self.best_energy = self.energy.clone()
        self.best_cols = self.cols.clone()
        self.temp_of = t.arange(R, dtype=t.int32, device=dev) % L
        self.chain_at = t.arange(R, dtype=t.int32, device=dev) % L
        self.counter = t.zeros(R, dtype=t.int64, device=dev)
        self.accepted_dev = t.zeros(R, dtype=t.int32, device=dev)
        self.ladder_n = t.from_numpy(self.ladder_n_host).to(dev)
        self.ladder_round = t.zeros(R // L, dtype=t.int32, device=dev)
        self.ladder_exchanges = t.zeros(R // L, dtype=t.int32, device=dev)
        self.acc_table = t.from_numpy(metropolis_table(ladder).view(np.int32)).to(dev)
        self.exch_table = t.from_numpy(exchange_table(ladder).view(np.int32)).to(dev)
        self.global_best = t.full((1,), 2 ** 31 - 1, dtype=t.int32, device=dev)
        self.hit = t.full((4,), -1, dtype=t.int32, device=dev)
        self.stop = t.zeros(1, dtype=t.int32, device=dev)
        self.error_word = t.zeros(1, dtype=t.int32, device=dev)
        self.round = 0
        self._graphs = {}
        # Umbrella restraint (tempering.py:148-152): the reference state is
        # replica 0's initial state; centres and strengths are per replica
        # position (host float32 arrays, like the reference's, which callers
        # assign or fill); `removed` is kept exact on the device while an
        # umbrella is active and recounted from the states before one starts.
        m0 = 2 * int(self.ladder_n_host[0])
        self.reference_host = np.asarray(cols[0, :m0], np.int32)
        ref = np.zeros(STRIDE, np.int16)
        ref[:m0] = self.reference_host
        self.reference_dev = t.from_numpy(ref).to(dev)
        self.removed_dev = t.from_numpy(reference_distance(self.reference_host, padded)).to(dev)
        self._removed_exact = True
        self.centers = np.zeros(R, np.float32)
        self.strengths = np.zeros(R, np.float32)
        self.umbrella_dev = t.zeros((R, 2), dtype=t.int64, device=dev)
        self.frac_table = t.from_numpy(fraction_table(ladder).view(np.int32)).to(dev)

    @classmethod
    def mixed(cls, groups, ladder_temperatures, seed: int, device=None):
        """Chains of several grid sizes in one set: ``groups`` is a list of
        (n, columns[count, 2n]) with count a multiple of the ladder size."""
        L = len(ladder_temperatures)
        cols, temps, lad_n = [], [], []
        for n, c in groups:
            c = np.asarray(c)
            if c.shape[1] != 2 * n or c.shape[0] % L:
                raise ValueError(f"group n={n}: columns must be (k*{L}, {2 * n})")
            pad = np.zeros((c.shape[0], STRIDE), np.int16)
            pad[:, :2 * n] = c
            cols.append(pad)
            temps.append(np.tile(ladder_temperatures, c.shape[0] // L))
            lad_n += [n] * (c.shape[0] // L)
        return cls(np.concatenate(cols), np.concatenate(temps), seed, ladder_size=L, device=device,
                   ladder_n=np.asarray(lad_n, np.int32))

    @staticmethod
    def _infer_ladder(temps: np.ndarray) -> int:
        R = len(temps)
        for L in range(2, R + 1):
            if R % L == 0 and np.all(np.diff(temps[:L]) > 0) and np.allclose(np.tile(temps[:L], R // L), temps):
                return L
        raise ValueError("temperatures do not tile an increasing ladder")

    # -- set-up ------------------------------------------------------------
    def _score_initial(self):
        t = _lib.torch()
        for n in np.unique(self.ladder_n_host):
            rows = np.nonzero(np.repeat(self.ladder_n_host, self.L) == n)[0]
            idx = t.from_numpy(rows).to(self.device)
            block = self.cols[idx, :2 * n].contiguous()
            scores = t.empty(len(rows), dtype=t.int32, device=self.device)
            bad = t.empty((len(rows), 2 * n), dtype=t.int32, device=self.device)
            _lib.call("n3_score_columns", block.data_ptr(), len(rows), int(n), scores.data_ptr(), bad.data_ptr(),
                      _lib.stream_ptr())
            self.energy[idx] = scores
            full = t.zeros((len(rows), STRIDE), dtype=t.int32, device=self.device)
            full[:, :2 * n] = bad
            self.badness_dev[idx] = full

    def _descriptor(self) -> N3Chains:
        d = N3Chains()
        d.n_chains = self.cols.shape[0]
        d.ladder_size = self.L
        d.cols, d.badness, d.energy = self.cols.data_ptr(), self.badness_dev.data_ptr(), self.energy.data_ptr()
        d.best_energy, d.best_cols = self.best_energy.data_ptr(), self.best_cols.data_ptr()
        d.temp_of, d.chain_at = self.temp_of.data_ptr(), self.chain_at.data_ptr()
        d.counter, d.accepted = self.counter.data_ptr(), self.accepted_dev.data_ptr()
        d.ladder_n, d.ladder_round = self.ladder_n.data_ptr(), self.ladder_round.data_ptr()
        d.ladder_exchanges = self.ladder_exchanges.data_ptr()
        d.acc_thresh, d.acc_width = self.acc_table.data_ptr(), self.acc_table.shape[1]
        d.exch_thresh, d.exch_width = self.exch_table.data_ptr(), self.exch_table.shape[1]
        d.global_best, d.hit, d.stop = self.global_best.data_ptr(), self.hit.data_ptr(), self.stop.data_ptr()
        d.error_word = self.error_word.data_ptr()
        d.reference, d.removed = self.reference_dev.data_ptr(), self.removed_dev.data_ptr()
        d.acc_frac = self.frac_table.data_ptr()
        d.umbrella = self.umbrella_dev.data_ptr() if self.umbrella_active() else None
        return d

    # -- umbrella restraint ------------------------------------------------------------
    def umbrella_active(self) -> bool:
        return bool(np.any(np.asarray(self.strengths) != 0))

    def _prepare_umbrella(self) -> None:
        """Uploads the fixed-point coefficients of the current centres and
        strengths and, if the distance counts went stale under launches without
        an umbrella, recounts them (called outside any graph capture)."""
        t = _lib.torch()
        R = self.cols.shape[0]
        s, c = np.asarray(self.strengths, np.float32), np.asarray(self.centers, np.float32)
        if s.shape != (R,) or c.shape != (R,):
            raise ValueError("one umbrella centre and strength is required per replica")
        if not np.all(np.isfinite(s)) or not np.all(np.isfinite(c)):
            raise ValueError("umbrella centres and strengths must be finite")
        if not self.umbrella_active():
            return
        if len(np.unique(self.ladder_n_host)) != 1:
            raise ValueError("an umbrella needs chains of one grid size")
        self.umbrella_dev.copy_(t.from_numpy(umbrella_coefficients(s, c)))
        self._refresh_removed()

    def _refresh_removed(self) -> None:
        if self._removed_exact:
            return
        t = _lib.torch()
        cols = self.cols.cpu().numpy()
        self.removed_dev.copy_(t.from_numpy(reference_distance(self.reference_host, cols)))
        self._removed_exact = True

    def _moved(self, umbrella: bool) -> None:
        """Bookkeeping after a launch that may have moved states."""
        if not umbrella:
            self._removed_exact = False

    def default_chains_per_block(self, threads_per_chain: int = 32) -> int:
        """Chains per CTA for teams of ``threads_per_chain`` threads (at most 16
        warps per CTA, so cap = 16 / warps per chain): whole ladders per CTA
        when L <= cap (as many as fit and divide the ladder count), else the
        largest divisor of L up to cap whose cluster (L / cpb CTAs) has at most
        8 CTAs."""
        if threads_per_chain not in (32, 64, 128, 256):
            raise ValueError("threads_per_chain must be 32, 64, 128 or 256")
        cap = 16 // (threads_per_chain // 32)
        L, ladders = self.L, self.cols.shape[0] // self.L
        if L <= cap:
            k = max(k for k in range(1, cap // L + 1) if ladders % k == 0)
            return k * L
        for d in range(cap, 0, -1):
            if L % d == 0 and L // d <= 8:
                return d
        raise ValueError(f"ladder size {L} cannot be split over at most 8 CTAs of at most {cap} chains "
                         f"({threads_per_chain} threads per chain)")

    def _shape_cpb(self, threads_per_chain: int) -> int:
        """The set's chains_per_block when it was chosen for this team width,
        else the default."""
        if self.chains_per_block and threads_per_chain == self.threads_per_chain:
            return int(self.chains_per_block)
        return self.default_chains_per_block(threads_per_chain)

    def _config(self, *, rounds, round_sweeps=0, round_proposals=0, exchange=True, chains_per_block=None,
                target=-1, ladder_rounds=None, bad_bias=0, threads_per_chain=None) -> N3TemperConfig:
        c = N3TemperConfig()
        c.seed = self.seed
        c.threads_per_chain = int(threads_per_chain or self.threads_per_chain)
        c.chains_per_block = chains_per_block or self._shape_cpb(c.threads_per_chain)
        c.rounds = rounds
        c.ladder_rounds = None if ladder_rounds is None else ladder_rounds.data_ptr()
        c.round_sweeps = round_sweeps
        c.round_proposals = round_proposals
        c.exchange = int(exchange)
        c.target_energy = target
        c.bad_bias = int(bad_bias)
        return c

    def _launch(self, cfg: N3TemperConfig, stream=None):
        d = self._descriptor()
        _lib.check(_lib.lib().n3_temper_run(ctypes.byref(d), ctypes.byref(cfg), _lib.stream_ptr(stream)),
                   "n3_temper_run")

    # -- reference API ---------------------------------------------------------
    def advance(self, steps: int, bad_bias: int = 0) -> None:
        """``steps`` proposals per replica, no exchange (tempering.py:158-167).
        With ``bad_bias`` > 0 that percentage of proposals draws slot u in
        proportion to badness (tempering.py:51-55); active umbrella centres and
        strengths restrain the distance to the reference state (:59-63, 93-94)."""
        if steps < 1 or not 0 <= bad_bias <= 100:
            raise ValueError("steps must be positive and bad_bias in [0,100]")
        self._prepare_umbrella()
        umb = self.umbrella_active()
        self._launch(self._config(rounds=1, round_proposals=int(steps), exchange=False, bad_bias=bad_bias))
        self._moved(umb)
        _lib.torch().cuda.current_stream().synchronize()

    def exchange(self, ladder_size: int | None = None) -> int:
        """One neighbour-exchange round in every ladder (tempering.py:169-191);
        returns the number of accepted exchanges."""
        if ladder_size is not None and ladder_size != self.L:
            raise ValueError("ladder_size must divide replica count and match the chains' ladders")
        if self.umbrella_active():
            raise ValueError("temperature-only exchange is disabled with umbrella potentials")
        before = int(self.ladder_exchanges.sum().item())
        cfg = self._config(rounds=1, round_sweeps=0, round_proposals=0, exchange=True)
        cfg.round_proposals = 0
        cfg.round_sweeps = 0
        self._launch(cfg)
        self.round += 1
        return int(self.ladder_exchanges.sum().item()) - before

    def epoch(self, steps: int, bad_bias: int = 0) -> int:
        """One epoch of the reference's driver loop (tempering.py:276-278):
        ``steps`` proposals per replica, then one neighbour-exchange round
        unless an umbrella is active, in a single launch.  Returns the number
        of accepted exchanges."""
        if steps < 1 or not 0 <= bad_bias <= 100:
            raise ValueError("steps must be positive and bad_bias in [0,100]")
        self._prepare_umbrella()
        umb = self.umbrella_active()
        before = int(self.ladder_exchanges.sum().item())
        self._launch(self._config(rounds=1, round_proposals=int(steps), exchange=not umb, bad_bias=bad_bias))
        self._moved(umb)
        if not umb:
            self.round += 1
        return int(self.ladder_exchanges.sum().item()) - before

    def run(self, sweeps: int, *, exchange_every: int = 10, chains_per_block: int | None = None,
            sweeps_per_launch: int | None = None, target: int | None = None, ladder_sweeps=None,
            max_seconds: float | None = None, graph: bool = True, bad_bias: int = 0,
            exchange: bool = True, threads_per_chain: int | None = None) -> RunResult:
        """Native path: ``sweeps`` sweeps (one sweep = 2n proposals per chain)
        with a neighbour exchange every ``exchange_every`` sweeps, all on the
        device.  With ``target`` the run stops at the first exchange boundary
        after some chain reaches E <= target; ``hit`` then reports when.
        ``bad_bias`` as in ``advance``; ``exchange=False`` runs the rounds
        without exchanges (required while an umbrella is active).
        ``threads_per_chain`` (32, 64, 128 or 256; default the chain set's
        ``threads_per_chain``) and ``chains_per_block`` shape the launch only:
        results are the same for every choice."""
        t = _lib.torch()
        if sweeps % exchange_every:
            raise ValueError("sweeps must be a multiple of exchange_every")
        if not 0 <= bad_bias <= 100:
            raise ValueError("bad_bias must lie in [0,100]")
        self._prepare_umbrella()
        umb = self.umbrella_active()
        if umb and exchange:
            raise ValueError("temperature-only exchange is disabled with umbrella potentials")
        per_launch = sweeps_per_launch or sweeps
        per_launch = max(exchange_every, per_launch - per_launch % exchange_every)
        launches = -(-sweeps // per_launch)
        rounds_per_launch = per_launch // exchange_every
        ladder_rounds = None
        tpc = int(threads_per_chain or self.threads_per_chain)
        cpb = chains_per_block or self._shape_cpb(tpc)
        if ladder_sweeps is not None:
            ls = np.asarray(ladder_sweeps, np.int32)
            if ls.shape != (self.cols.shape[0] // self.L,) or np.any(ls % exchange_every) or np.any(ls < 0):
                raise ValueError("ladder_sweeps: one multiple of exchange_every per ladder")
            if cpb > self.L and np.any(ls.reshape(-1, cpb // self.L) != ls.reshape(-1, cpb // self.L)[:, :1]):
                raise ValueError("ladders sharing a CTA must run the same number of sweeps")
            ladder_rounds = t.from_numpy(ls // exchange_every).to(self.device)
        tgt = -1 if target is None else int(target)
        self.stop.zero_()
        self.hit.fill_(-1)
        cfg = self._config(rounds=rounds_per_launch, round_sweeps=exchange_every, exchange=exchange,
                           chains_per_block=cpb, target=tgt, ladder_rounds=ladder_rounds,
                           bad_bias=bad_bias, threads_per_chain=tpc)
        stream = t.cuda.current_stream()
        if graph:
            key = (rounds_per_launch, exchange_every, cfg.chains_per_block, tpc, tgt,
                   None if ladder_sweeps is None else tuple(int(x) for x in np.asarray(ladder_sweeps)),
                   int(bad_bias), bool(exchange), umb)
            if key not in self._graphs:
                self._graphs[key] = (self._capture(cfg), ladder_rounds)
            exec_handle = self._graphs[key][0]

            def launch():
                _lib.call("n3_graph_launch", exec_handle, _lib.stream_ptr(stream))
        else:
            def launch():
                self._launch(cfg)
        start_ev = t.cuda.Event(enable_timing=True)
        end_ev = t.cuda.Event(enable_timing=True)
        t0_ns = _device_now_ns(self.device)
        wall0 = time.perf_counter()
        start_ev.record(stream)
        done = 0
        for _ in range(launches):
            launch()
            done += rounds_per_launch
            if tgt >= 0 or max_seconds is not None:
                stop = int(self.stop.item())
                if stop or (max_seconds is not None and time.perf_counter() - wall0 > max_seconds):
                    break
        end_ev.record(stream)
        end_ev.synchronize()
        seconds = start_ev.elapsed_time(end_ev) / 1e3
        self.round += done
        self._moved(umb)
        hit = None
        h = self.hit.cpu().numpy().astype(np.int64)
        if h[0] >= 0:
            ns = (int(h[2]) & 0xFFFFFFFF) | ((int(h[3]) & 0xFFFFFFFF) << 32)
            hit = (int(h[0]), int(h[1]) & 0xFFFFFFFF, (ns - t0_ns) / 1e9)
        swept = done * exchange_every
        if ladder_sweeps is None:
            proposals = swept * int(2 * np.repeat(self.ladder_n_host, self.L).sum())
        else:  # each launch ran every ladder for its own number of sweeps
            launched = done // rounds_per_launch
            proposals = launched * int((np.asarray(ladder_sweeps) * 2 * self.ladder_n_host).sum()) * self.L
        return RunResult(done, swept, proposals, seconds, int(self.best_energy.min().item()), hit)

    def _capture(self, cfg: N3TemperConfig):
        """CUDA graph of one launch with `cfg` (arguments frozen at capture)."""
        t = _lib.torch()
        warm = N3TemperConfig.from_buffer_copy(cfg)
        warm.rounds = 0
        warm.ladder_rounds = None
        self._launch(warm)  # sets kernel attributes and device tables outside the capture
        cur = t.cuda.current_stream()
        side = t.cuda.Stream(device=self.device)
        side.wait_stream(cur)
        handle = ctypes.c_void_p()
        with t.cuda.stream(side):
            _lib.call("n3_graph_begin", _lib.stream_ptr(side))
            try:
                self._launch(cfg, stream=side)
            finally:
                _lib.call("n3_graph_end", _lib.stream_ptr(side), ctypes.byref(handle))
        cur.wait_stream(side)
        return handle

    def release_graphs(self) -> None:
        for h, _ in self._graphs.values():
            _lib.lib().n3_graph_destroy(h)
        self._graphs.clear()

    def __del__(self):
        try:
            self.release_graphs()
        except Exception:  # interpreter shutdown
            pass

    def validate(self, indices=None) -> None:
        """Full recompute of every chain's energy and badness on the device
        (determinant + slope kernels) against the maintained values; raises
        AssertionError on any difference (tempering.py:193-204)."""
        t = _lib.torch()
        mism = t.zeros(1, dtype=t.int32, device=self.device)
        d = self._descriptor()
        _lib.check(_lib.lib().n3_temper_audit(ctypes.byref(d), mism.data_ptr(), _lib.stream_ptr()),
                   "n3_temper_audit")
        bad = int(mism.item())
        err = int(self.error_word.item())
        if bad or err:
            raise AssertionError(f"{bad} chain(s): incremental score/badness differs from full determinant check "
                                 f"(device error bits {err:#x})")
        if self._removed_exact and len(np.unique(self.ladder_n_host)) == 1:
            # the distance to the reference state (tempering.py:202-204)
            if not np.array_equal(reference_distance(self.reference_host, self.cols.cpu().numpy()),
                                  self.removed_dev.cpu().numpy()):
                raise AssertionError("incremental distance mismatch")

    @property
    def removed_points(self):
        """Reference points missing from each state, in replica order."""
        self._refresh_removed()
        return self.removed_dev[self._replica_index()]

    @property
    def reference(self):
        return self.reference_host

    # -- replica-order views -------------------------------------------------------
    def _replica_index(self):
        t = _lib.torch()
        R = self.cols.shape[0]
        base = (t.arange(R, device=self.device) // self.L) * self.L
        return base + self.chain_at.long()

    @property
    def columns(self):
        """States in replica order: row l*L+t is the chain at temperature t."""
        n = self.n
        return self.cols[self._replica_index()][:, :2 * n]

    @property
    def scores(self):
        return self.energy[self._replica_index()]

    @property
    def badness(self):
        return self.badness_dev[self._replica_index()][:, :2 * self.n]

    @property
    def best_scores(self):
        return self.best_energy

    @property
    def best_columns(self):
        return self.best_cols[:, :2 * self.n]

    @property
    def temperatures(self):
        return self.ladder_temperatures[self.temp_of.cpu().numpy()]

    @property
    def accepted(self):
        return self.accepted_dev

    def to_state(self, row):
        """P/Q of one slot-column row (tempering.py:155-156)."""
        row = np.asarray(row).reshape(-1)
        n = len(row) // 2
        return points_to_permutations(columns_to_points(row), n)

    # -- checkpoints ---------------------------------------------------------------
    _SAVE = ("cols", "badness_dev", "energy", "best_energy", "best_cols", "temp_of", "chain_at", "counter",
             "accepted_dev", "ladder_n", "ladder_round", "ladder_exchanges")

    def save(self, path) -> None:
        """npz checkpoint with every key the reference writes (tempering.py:206-212:
        columns, badness, scores, rngs, best_*, accepted, reference,
        removed_points, centers, strengths, temperatures, round, host_rng) plus
        this engine's own: the chain-order arrays, the Philox counters (also
        stored as ``rngs``), the temperature labels and the key."""
        self._refresh_removed()
        arrays = {k: getattr(self, k).cpu().numpy() for k in self._SAVE}
        arrays.update(columns=self.columns.cpu().numpy(), badness=self.badness.cpu().numpy(),
                      scores=self.scores.cpu().numpy(), best_columns=self.best_columns.cpu().numpy(),
                      best_scores=self.best_energy.cpu().numpy(), accepted=self.accepted_dev.cpu().numpy(),
                      rngs=self.counter.cpu().numpy().astype(np.uint64), reference=self.reference_host,
                      removed_points=self.removed_points.cpu().numpy(), removed=self.removed_dev.cpu().numpy(),
                      centers=np.asarray(self.centers, np.float32), strengths=np.asarray(self.strengths, np.float32))
        np.savez_compressed(path, **arrays, temperatures=self.temperatures_host, ladder_size=np.asarray(self.L),
                            seed=np.asarray(self.seed, dtype=np.uint64), round=np.asarray(self.round),
                            host_rng=np.asarray(json.dumps({"philox_key": self.seed})))

    @classmethod
    def restore(cls, path):
        """Restores a checkpoint written by ``save`` or by the reference's
        ``TemperingChains.save`` (tempering.py:206-225).  A reference checkpoint
        carries xorshift states rather than Philox counters: its chains restart
        their counters at 0 under the key ``rngs[0]``, at the temperatures and
        round parity it records.  Either way every energy and badness is then
        recomputed and compared (AssertionError on a difference, as the
        reference's restore does through validate)."""
        t = _lib.torch()
        with np.load(path, allow_pickle=False) as z:
            if "ladder_size" not in z:
                return cls._restore_reference(z)
            L = int(z["ladder_size"])
            ladder_n = z["ladder_n"]
            cols = z["cols"]
            R = cols.shape[0]
            n = int(ladder_n.max())
            obj = cls(cols[:, :2 * n] if len(np.unique(ladder_n)) == 1 else cols, z["temperatures"],
                      int(z["seed"]), ladder_size=L, ladder_n=ladder_n)
            for k in cls._SAVE:
                setattr(obj, k, t.from_numpy(np.ascontiguousarray(z[k])).to(obj.device))
            obj.round = int(z["round"])
            assert obj.cols.shape[0] == R
            obj._restore_umbrella(z, chain_order=True)
        obj.validate()
        return obj

    def _restore_umbrella(self, z, *, chain_order: bool) -> None:
        t = _lib.torch()
        if "reference" in z:
            m0 = len(self.reference_host)
            self.reference_host = np.asarray(z["reference"], np.int32).reshape(-1)[:m0]
            ref = np.zeros(STRIDE, np.int16)
            ref[:m0] = self.reference_host
            self.reference_dev.copy_(t.from_numpy(ref))
        for k in ("centers", "strengths"):
            if k in z:
                setattr(self, k, np.asarray(z[k], np.float32).copy())
        key = "removed" if chain_order else "removed_points"
        if key in z:
            self.removed_dev.copy_(t.from_numpy(np.ascontiguousarray(z[key], dtype=np.int32)))
            self._removed_exact = True
        else:
            self._removed_exact = False
            self._refresh_removed()

    @classmethod
    def _restore_reference(cls, z):
        t = _lib.torch()
        cols = np.asarray(z["columns"])
        rngs = np.asarray(z["rngs"], np.uint64) if "rngs" in z else np.zeros(1, np.uint64)
        obj = cls(cols, np.asarray(z["temperatures"]), int(rngs[0]))
        # the reference's chains sit at their replica positions: identity labels
        scores, bad = obj.energy.cpu().numpy(), obj.badness_dev.cpu().numpy()[:, :cols.shape[1]]
        if "scores" in z and not np.array_equal(np.asarray(z["scores"], np.int64), scores.astype(np.int64)):
            raise AssertionError("checkpoint scores differ from the full determinant check")
        if "badness" in z and not np.array_equal(np.asarray(z["badness"], np.int64), bad.astype(np.int64)):
            raise AssertionError("checkpoint badness differs from the full determinant check")
        R, m = cols.shape
        if "best_scores" in z and "best_columns" in z:
            obj.best_energy.copy_(t.from_numpy(np.asarray(z["best_scores"], np.int32)))
            best = np.zeros((R, STRIDE), np.int16)
            best[:, :m] = np.asarray(z["best_columns"])
            obj.best_cols.copy_(t.from_numpy(best))
        if "accepted" in z:
            obj.accepted_dev.copy_(t.from_numpy(np.asarray(z["accepted"], np.int32)))
        obj.round = int(z["round"]) if "round" in z else 0
        obj.ladder_round.fill_(obj.round)
        obj._restore_umbrella(z, chain_order=False)
        obj.validate()
        return obj


def _device_now_ns(device) -> int:
    """The device's %globaltimer (ns), read through a one-thread kernel."""
    t = _lib.torch()
    out = t.zeros(1, dtype=t.int64, device=device)
    _lib.call("n3_device_clock_ns", out.data_ptr(), _lib.stream_ptr())
    return int(out.item())


_lib.register("n3_device_clock_ns", [ctypes.c_void_p, ctypes.c_void_p])


def _state_columns(state) -> np.ndarray:
    """Slot-column row of a P/Q state (the reference's column_stack((P, Q)).flatten())."""
    return np.column_stack((state.P, state.Q)).flatten().astype(np.int32)


def _symmetric_distance(reference: set, row) -> int:
    return len(reference.symmetric_difference((i // 2, int(c)) for i, c in enumerate(row)))


def main(argv=None) -> int:
    """The reference's tempering driver (tempering.py:228-319) on this engine:
    same arguments and the same output directory layout (parameters.json,
    best-E<k>.json records, history.jsonl every 10 epochs with an audit,
    frontier-bin<k>.json under an umbrella, checkpoint.npz every 50 epochs and
    at the end, summary.json).  An epoch is one launch: ``steps`` proposals
    per replica then an exchange round.  A new record is rescored by both
    device counts (determinant and slope) before it is written, as the
    reference rescores it with score_and_badness; a record of E = 0 must pass
    both counts with zero, as it must pass both verifiers there."""
    import argparse

    from . import gpu
    from .io import load_candidate, write_candidate

    parser = argparse.ArgumentParser(description="Persistent replica-exchange tempering with exact integer deltas.")
    parser.add_argument("--initial", nargs="+", required=True)
    parser.add_argument("--output", required=True)
    parser.add_argument("--seed", type=int, required=True)
    parser.add_argument("--replicas", type=int, default=128)
    parser.add_argument("--ladder-size", type=int, default=16)
    parser.add_argument("--tmin", type=float, default=0.2)
    parser.add_argument("--tmax", type=float, default=4)
    parser.add_argument("--rounds", type=int, default=200)
    parser.add_argument("--steps", type=int, default=100)
    parser.add_argument("--bad-bias", type=int, default=0)
    parser.add_argument("--resume")
    parser.add_argument("--umbrella-max", type=float, default=0)
    parser.add_argument("--umbrella-strength", type=float, default=0.2)
    parser.add_argument("--threads-per-chain", default="auto", choices=["auto", "32", "64", "128", "256"],
                        help="launch shape; auto: the autotuner times every shape on copies of the chains")
    args = parser.parse_args(argv)
    output = Path(args.output)
    output.mkdir(parents=True, exist_ok=True)
    rows, n = [], None
    for path in args.initial:
        size, points, _ = load_candidate(path)
        if n is not None and n != size:
            raise ValueError("all initial sizes must agree")
        n = size
        rows.append(_state_columns(points_to_permutations(points, n)))
    if args.replicas % args.ladder_size or args.ladder_size < 2:
        raise ValueError("replicas must be a multiple of ladder-size >=2")
    if args.resume:
        chains = TemperingChains.restore(Path(args.resume))
        if chains.cols.shape[0] != args.replicas or chains.n != n:
            raise ValueError("checkpoint dimensions differ from arguments")
    else:
        columns = np.asarray([rows[(i // args.ladder_size) % len(rows)] for i in range(args.replicas)], np.int32)
        temperatures = np.tile(geometric_ladder(args.tmin, args.tmax, args.ladder_size),
                               args.replicas // args.ladder_size)
        chains = TemperingChains(columns, temperatures, args.seed, ladder_size=args.ladder_size)
    if args.umbrella_max:
        chains.centers = np.repeat(np.linspace(0, args.umbrella_max, args.replicas // args.ladder_size),
                                   args.ladder_size).astype(np.float32)
        chains.strengths.fill(args.umbrella_strength)
    if args.threads_per_chain == "auto":
        from .autotune import autotune

        tune = autotune(chains, probe_sweeps=2, exchange_every=2)
        chains.threads_per_chain, chains.chains_per_block = tune.threads_per_chain, tune.chains_per_block
    else:
        chains.threads_per_chain = int(args.threads_per_chain)
    reference = set((i // 2, int(c)) for i, c in enumerate(rows[0]))
    start = time.perf_counter()
    best, proposals, archive = 10 ** 9, 0, {}
    # the reference's parameters (the launch shape does not change results)
    params = {k: v for k, v in vars(args).items() if k != "threads_per_chain"}
    (output / "parameters.json").write_text(json.dumps(params, indent=2) + "\n", encoding="utf-8")
    for epoch in range(1, args.rounds + 1):
        exchanges = chains.epoch(args.steps, args.bad_bias)
        proposals += args.steps * args.replicas
        best_scores = chains.best_scores.cpu().numpy()
        index = int(np.argmin(best_scores))
        if int(best_scores[index]) < best:
            best = int(best_scores[index])
            row = chains.best_columns[index].cpu().numpy()
            state = chains.to_state(row)
            exact = gpu.score_checked_gpu(_state_columns(state)[None])
            if int(exact.scores[0]) != best:
                raise AssertionError("record differs from independent full score")
            write_candidate(output / f"best-E{best}.json", n, state.points(), conflicts=best, seed=args.seed,
                            epoch=epoch, proposals=proposals, method="persistent CUDA replica exchange")
            print(f"epoch={epoch} best={best} proposals={proposals} seconds={time.perf_counter() - start:.2f}",
                  flush=True)
            if best == 0:
                break
        if epoch % 10 == 0 or epoch == args.rounds:
            chains.validate()
            columns = chains.columns.cpu().numpy()
            scores = chains.scores.cpu().numpy()
            distances = [_symmetric_distance(reference, r) for r in columns]
            if args.umbrella_max:
                for i, (score, distance) in enumerate(zip(scores, distances)):
                    bucket = distance // 8
                    if int(score) < archive.get(bucket, 10 ** 9):
                        archive[bucket] = int(score)
                        candidate = chains.to_state(columns[i])
                        write_candidate(output / f"frontier-bin{bucket:02d}.json", n, candidate.points(),
                                        conflicts=int(score), symmetric_difference=distance, epoch=epoch,
                                        seed=args.seed)
            payload = {"epoch": epoch, "proposals": proposals, "elapsed_seconds": time.perf_counter() - start,
                       "best": best, "scores": scores.tolist(), "distances": distances, "exchanges": exchanges,
                       "accepted": int(chains.accepted.cpu().numpy().astype(np.int64).sum())}
            with (output / "history.jsonl").open("a", encoding="utf-8") as stream:
                stream.write(json.dumps(payload) + "\n")
        if epoch % 50 == 0:
            chains.save(output / "checkpoint.npz")
    chains.validate()
    chains.save(output / "checkpoint.npz")
    result = {"best": best, "proposals": proposals, "elapsed_seconds": time.perf_counter() - start,
              "accepted": int(chains.accepted.cpu().numpy().astype(np.int64).sum()), "distance_frontier": archive}
    (output / "summary.json").write_text(json.dumps(result, indent=2) + "\n", encoding="utf-8")
    print(json.dumps(result), flush=True)
    return 0

