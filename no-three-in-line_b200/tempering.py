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
                ("hit", ctypes.c_void_p), ("stop", ctypes.c_void_p), ("error_word", ctypes.c_void_p)]


class N3TemperConfig(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("chains_per_block", ctypes.c_int), ("rounds", ctypes.c_int),
                ("ladder_rounds", ctypes.c_void_p), ("round_sweeps", ctypes.c_int),
                ("round_proposals", ctypes.c_int), ("exchange", ctypes.c_int), ("target_energy", ctypes.c_int)]


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
        return d

    def default_chains_per_block(self) -> int:
        """Chains (warps) per CTA: whole ladders per CTA when L <= 16 (as many as
        fit in 16 warps and divide the ladder count), else the largest divisor
        of L up to 16 whose cluster (L / cpb CTAs) has at most 8 CTAs."""
        L, ladders = self.L, self.cols.shape[0] // self.L
        if L <= 16:
            k = max(k for k in range(1, 16 // L + 1) if ladders % k == 0)
            return k * L
        for d in range(16, 0, -1):
            if L % d == 0 and L // d <= 8:
                return d
        raise ValueError(f"ladder size {L} cannot be split over at most 8 CTAs of at most 16 chains")

    def _config(self, *, rounds, round_sweeps=0, round_proposals=0, exchange=True, chains_per_block=None,
                target=-1, ladder_rounds=None) -> N3TemperConfig:
        c = N3TemperConfig()
        c.seed = self.seed
        c.chains_per_block = chains_per_block or self.default_chains_per_block()
        c.rounds = rounds
        c.ladder_rounds = None if ladder_rounds is None else ladder_rounds.data_ptr()
        c.round_sweeps = round_sweeps
        c.round_proposals = round_proposals
        c.exchange = int(exchange)
        c.target_energy = target
        return c

    def _launch(self, cfg: N3TemperConfig, stream=None):
        d = self._descriptor()
        _lib.check(_lib.lib().n3_temper_run(ctypes.byref(d), ctypes.byref(cfg), _lib.stream_ptr(stream)),
                   "n3_temper_run")

    # -- reference API ---------------------------------------------------------
    def advance(self, steps: int, bad_bias: int = 0) -> None:
        """``steps`` proposals per replica, no exchange (tempering.py:158-167)."""
        if steps < 1 or not 0 <= bad_bias <= 100:
            raise ValueError("steps must be positive and bad_bias in [0,100]")
        if bad_bias:
            raise ValueError("badness-biased slot selection is not provided by this engine; use bad_bias=0")
        self._launch(self._config(rounds=1, round_proposals=int(steps), exchange=False))
        _lib.torch().cuda.current_stream().synchronize()

    def exchange(self, ladder_size: int | None = None) -> int:
        """One neighbour-exchange round in every ladder (tempering.py:169-191);
        returns the number of accepted exchanges."""
        if ladder_size is not None and ladder_size != self.L:
            raise ValueError("ladder_size must divide replica count and match the chains' ladders")
        before = int(self.ladder_exchanges.sum().item())
        cfg = self._config(rounds=1, round_sweeps=0, round_proposals=0, exchange=True)
        cfg.round_proposals = 0
        cfg.round_sweeps = 0
        self._launch(cfg)
        self.round += 1
        return int(self.ladder_exchanges.sum().item()) - before

    def run(self, sweeps: int, *, exchange_every: int = 10, chains_per_block: int | None = None,
            sweeps_per_launch: int | None = None, target: int | None = None, ladder_sweeps=None,
            max_seconds: float | None = None, graph: bool = True) -> RunResult:
        """Native path: ``sweeps`` sweeps (one sweep = 2n proposals per chain)
        with a neighbour exchange every ``exchange_every`` sweeps, all on the
        device.  With ``target`` the run stops at the first exchange boundary
        after some chain reaches E <= target; ``hit`` then reports when."""
        t = _lib.torch()
        if sweeps % exchange_every:
            raise ValueError("sweeps must be a multiple of exchange_every")
        per_launch = sweeps_per_launch or sweeps
        per_launch = max(exchange_every, per_launch - per_launch % exchange_every)
        launches = -(-sweeps // per_launch)
        rounds_per_launch = per_launch // exchange_every
        ladder_rounds = None
        cpb = chains_per_block or self.default_chains_per_block()
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
        cfg = self._config(rounds=rounds_per_launch, round_sweeps=exchange_every, exchange=True,
                           chains_per_block=chains_per_block, target=tgt, ladder_rounds=ladder_rounds)
        stream = t.cuda.current_stream()
        if graph:
            key = (rounds_per_launch, exchange_every, cfg.chains_per_block, tgt,
                   None if ladder_sweeps is None else tuple(int(x) for x in np.asarray(ladder_sweeps)))
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
        """npz checkpoint; carries the reference's keys (tempering.py:206-212)
        plus the Philox counters and temperature labels."""
        arrays = {k: getattr(self, k).cpu().numpy() for k in self._SAVE}
        arrays.update(columns=self.columns.cpu().numpy(), badness=self.badness.cpu().numpy(),
                      scores=self.scores.cpu().numpy(), best_columns=self.best_columns.cpu().numpy(),
                      best_scores=self.best_energy.cpu().numpy(), accepted=self.accepted_dev.cpu().numpy(),
                      rngs=self.counter.cpu().numpy().astype(np.uint64))
        np.savez_compressed(path, **arrays, temperatures=self.temperatures_host, ladder_size=np.asarray(self.L),
                            seed=np.asarray(self.seed, dtype=np.uint64), round=np.asarray(self.round),
                            host_rng=np.asarray(json.dumps({"philox_key": self.seed})))

    @classmethod
    def restore(cls, path):
        t = _lib.torch()
        with np.load(path, allow_pickle=False) as z:
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
        obj.validate()
        return obj


def _device_now_ns(device) -> int:
    """The device's %globaltimer (ns), read through a one-thread kernel."""
    t = _lib.torch()
    out = t.zeros(1, dtype=t.int64, device=device)
    _lib.call("n3_device_clock_ns", out.data_ptr(), _lib.stream_ptr())
    return int(out.item())


_lib.register("n3_device_clock_ns", [ctypes.c_void_p, ctypes.c_void_p])
