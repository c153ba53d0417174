"""Learned move proposal for the tempering chains (no reference counterpart).

Per chain and step, 128 candidate swaps are scored by a 192 -> 256 -> 256 -> 1
MLP (bf16 tensor-core inference, fp32 accumulation); one candidate is drawn
from softmax(-predicted dE / T) and accepted by the exact integer delta with
the chain's Metropolis threshold row (the same rule as the uniform-proposal
tempering, which stays available as ``TemperingChains.run``).  Every step
pushes the chosen candidate's (features, exact dE) into a ring buffer (2M
tuples by default); ``train`` takes Adam steps (lr 1e-3) on batches drawn
from it with the hand-written kernels of libn3.

Softmax proposals are not symmetric, so without a Hastings correction the
learned chains are an optimiser rather than a sampler of the Boltzmann
distribution; the exact-delta acceptance keeps every energy exact.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from .tempering import N3Chains, RunResult, TemperingChains

N_CAND = 128
N_IN, N_H = 192, 256


class N3Mlp(ctypes.Structure):
    _fields_ = [("params", ctypes.c_void_p), ("w2_img", ctypes.c_void_p), ("w1a_img", ctypes.c_void_p),
                ("a1_img", ctypes.c_void_p), ("badn", ctypes.c_void_p), ("c1", ctypes.c_void_p),
                ("cand", ctypes.c_void_p), ("pred", ctypes.c_void_p), ("rb_feat", ctypes.c_void_p),
                ("rb_bad", ctypes.c_void_p), ("rb_dE", ctypes.c_void_p), ("rb_capacity", ctypes.c_int64),
                ("stats", ctypes.c_void_p), ("counters", ctypes.c_void_p), ("loss_out", ctypes.c_void_p),
                ("error_word", ctypes.c_void_p)]


_P = ctypes.c_void_p
_lib.register("n3_mlp_param_count", [])
_lib.register("n3_mlp_scratch_floats", [ctypes.c_int])
_lib.register("n3_mlp_pack", [ctypes.POINTER(N3Mlp), _P])
_lib.register("n3_mlp_candidates", [ctypes.POINTER(N3Chains), ctypes.POINTER(N3Mlp), ctypes.c_uint64, ctypes.c_int,
                                     _P])
_lib.register("n3_mlp_infer", [ctypes.POINTER(N3Mlp), ctypes.c_int, _P])
_lib.register("n3_mlp_step", [ctypes.POINTER(N3Chains), ctypes.POINTER(N3Mlp), _P, ctypes.c_uint64, ctypes.c_int,
                              _P])
_lib.register("n3_mlp_step_team", [ctypes.POINTER(N3Chains), ctypes.POINTER(N3Mlp), _P, ctypes.c_uint64,
                                   ctypes.c_int, ctypes.c_int, _P])
_lib.register("n3_mlp_train", [ctypes.POINTER(N3Mlp), ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_uint64,
                               _P, _P, _P, _P, _P])

# parameter offsets (fp32 buffer)
O_W1 = 0
O_B1 = O_W1 + N_H * N_IN
O_W2 = O_B1 + N_H
O_B2 = O_W2 + N_H * N_H
O_W3 = O_B2 + N_H
O_B3 = O_W3 + N_H


def init_params(seed: int) -> np.ndarray:
    """He-uniform weights, zero biases (float32 [n3_mlp_param_count()])."""
    count = int(_lib.lib().n3_mlp_param_count())
    rng = np.random.default_rng(seed)
    p = np.zeros(count, np.float32)
    p[O_W1:O_B1] = rng.uniform(-1, 1, N_H * N_IN) * math.sqrt(6.0 / 162)
    p[O_W2:O_B2] = rng.uniform(-1, 1, N_H * N_H) * math.sqrt(6.0 / N_H)
    p[O_W3:O_B3] = rng.uniform(-1, 1, N_H) * math.sqrt(3.0 / N_H)
    # inputs 162..191 are zero padding: their weights stay zero
    w1 = p[O_W1:O_B1].reshape(N_H, N_IN)
    w1[:, 162:] = 0.0
    return p


@dataclass
class LearnedStats:
    mae: float          # mean |predicted dE - exact dE| of the chosen candidates
    proposals: int
    accepted: int
    mean_accepted_dE: float
    loss: float         # mean squared error (in units of (dE/16)^2) of the last training batch


_lib.register("n3_check_bounded_wait", [ctypes.c_uint32, _P, _P])

ERR_TIMEOUT = 8  # device error bit: a bounded wait gave up


def check_bounded_wait(tries: int = 256) -> None:
    """Runs the tensor-core pipeline's bounded mbarrier wait on a barrier that
    nothing arrives on; the wait gives up after ``tries`` attempts and the
    device reports it.  Raises TimeoutError, as a stalled pipeline would."""
    t = _lib.torch()
    dev = _lib.require_device()
    err = t.zeros(1, dtype=t.int32, device=dev)
    _lib.call("n3_check_bounded_wait", int(tries), err.data_ptr(), _lib.stream_ptr())
    bits = int(err.item())
    if bits & ERR_TIMEOUT:
        raise TimeoutError(f"a bounded device wait gave up after {tries} tries (error bits {bits:#x})")


class LearnedProposal:
    """Learned proposals driving a TemperingChains object's chains."""

    def __init__(self, chains: TemperingChains, *, seed: int = 1, ring_capacity: int = 1 << 21,
                 batch: int = 4096, lr: float = 1e-3, params: np.ndarray | None = None, moves: int = 1,
                 bad_bias: int = 0, threads_per_chain: int = 0):
        t = _lib.torch()
        if not 0 <= bad_bias <= 100:
            raise ValueError("bad_bias must lie in [0,100]")
        if threads_per_chain not in (0, 32, 64):
            raise ValueError("threads_per_chain must be 0 (the default), 32 or 64")
        self.bad_bias = int(bad_bias)
        # width of the team that makes one chain's exact moves (0: the library's default)
        self.threads_per_chain = int(threads_per_chain)
        self.ch = chains
        dev = chains.device
        C = chains.cols.shape[0]
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.batch = batch
        self.lr = lr
        self.moves = int(moves)
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        count = int(_lib.lib().n3_mlp_param_count())
        if p.shape != (count,):
            raise ValueError(f"params must have {count} floats")
        self.params = t.from_numpy(p.copy()).to(dev)
        self.adam_m = t.zeros(count, dtype=t.float32, device=dev)
        self.adam_v = t.zeros(count, dtype=t.float32, device=dev)
        self.grads = t.zeros(count, dtype=t.float32, device=dev)
        self.scratch = t.zeros(int(_lib.lib().n3_mlp_scratch_floats(batch)), dtype=t.float32, device=dev)
        self.w2_img = t.zeros(131072, dtype=t.uint8, device=dev)
        self.w1a_img = t.zeros(8192, dtype=t.uint8, device=dev)
        self.a1_img = t.zeros(C * 4096, dtype=t.uint8, device=dev)
        self.badn = t.zeros((C, 150), dtype=t.float32, device=dev)
        self.c1 = t.zeros((C, N_H), dtype=t.float32, device=dev)
        self.cand = t.zeros((C, N_CAND), dtype=t.int32, device=dev)
        self.pred = t.zeros((C, N_CAND), dtype=t.float32, device=dev)
        self.rb_capacity = int(ring_capacity)
        self.rb_feat = t.zeros((self.rb_capacity, 12), dtype=t.int16, device=dev)
        self.rb_bad = t.zeros((self.rb_capacity, 150), dtype=t.uint8, device=dev)
        self.rb_dE = t.zeros(self.rb_capacity, dtype=t.int16, device=dev)
        self.stats = t.zeros(4, dtype=t.float32, device=dev)
        self.counters = t.zeros(2, dtype=t.int64, device=dev)
        self.loss = t.zeros(1, dtype=t.float32, device=dev)
        self.error_word = t.zeros(1, dtype=t.int32, device=dev)
        self.temps = t.from_numpy(np.asarray(chains.ladder_temperatures, np.float32)).to(dev)
        self._desc = self._descriptor()
        _lib.check(_lib.lib().n3_mlp_pack(ctypes.byref(self._desc), _lib.stream_ptr()), "n3_mlp_pack")
        self._graphs = {}

    def _descriptor(self) -> N3Mlp:
        d = N3Mlp()
        for name in ("params", "w2_img", "w1a_img", "a1_img", "badn", "c1", "cand", "pred", "rb_feat", "rb_bad",
                     "rb_dE", "stats", "counters", "error_word"):
            setattr(d, name, getattr(self, name).data_ptr())
        d.loss_out = self.loss.data_ptr()
        d.rb_capacity = self.rb_capacity
        return d

    # -- single operations (stream-ordered) ------------------------------------------
    def propose_scores(self, stream=None):
        """Draw this step's candidates and predict their dE (tcgen05 MLP)."""
        L = _lib.lib()
        cd = self.ch._descriptor()
        s = _lib.stream_ptr(stream)
        _lib.check(L.n3_mlp_candidates(ctypes.byref(cd), ctypes.byref(self._desc), self.seed, self.bad_bias, s),
                   "n3_mlp_candidates")
        _lib.check(L.n3_mlp_infer(ctypes.byref(self._desc), self.ch.cols.shape[0], s), "n3_mlp_infer")

    def step(self, stream=None):
        """One learned step on every chain."""
        self.propose_scores(stream)
        cd = self.ch._descriptor()
        _lib.check(_lib.lib().n3_mlp_step_team(ctypes.byref(cd), ctypes.byref(self._desc), self.temps.data_ptr(),
                                               self.seed, self.moves, self.threads_per_chain,
                                               _lib.stream_ptr(stream)), "n3_mlp_step_team")
        self.ch._moved(False)

    def train(self, stream=None):
        """One Adam step on a batch from the ring buffer."""
        _lib.check(_lib.lib().n3_mlp_train(ctypes.byref(self._desc), self.ch.cols.shape[0] * self.moves,
                                           self.batch, self.lr,
                                           self.seed ^ 0x5A5A5A5A, self.scratch.data_ptr(), self.grads.data_ptr(),
                                           self.adam_m.data_ptr(), self.adam_v.data_ptr(), _lib.stream_ptr(stream)),
                   "n3_mlp_train")

    def exchange(self, stream=None):
        cfg = self.ch._config(rounds=1, round_sweeps=0, round_proposals=0, exchange=True)
        self.ch._launch(cfg, stream=stream)

    def read_stats(self, reset: bool = True) -> LearnedStats:
        s = self.stats.cpu().numpy().astype(np.float64)
        loss = float(self.loss.item()) / max(1, self.batch)
        if reset:
            self.stats.zero_()
        n = max(1.0, s[1])
        return LearnedStats(s[0] / n, int(s[1]), int(s[2]), s[3] / max(1.0, s[2]), loss)

    # -- blocks of steps in CUDA graphs ------------------------------------------------
    def _capture(self, steps: int, train_every: int, exchange: bool):
        t = _lib.torch()
        # warm-up outside capture: kernel attributes and device tables
        cur = t.cuda.current_stream()
        side = t.cuda.Stream(device=self.ch.device)
        side.wait_stream(cur)
        handle = ctypes.c_void_p()
        with t.cuda.stream(side):
            _lib.call("n3_graph_begin", _lib.stream_ptr(side))
            try:
                for k in range(steps):
                    self.step(stream=side)
                    if train_every and (k + 1) % train_every == 0:
                        self.train(stream=side)
                if exchange:
                    self.exchange(stream=side)
            finally:
                _lib.call("n3_graph_end", _lib.stream_ptr(side), ctypes.byref(handle))
        cur.wait_stream(side)
        return handle

    def run(self, steps: int, *, exchange_every: int = 1500, train_every: int = 10, block: int = 50,
            target: int | None = None, max_seconds: float | None = None, warm: bool = True,
            graph: bool = True) -> RunResult:
        """``steps`` learned steps per chain with a neighbour exchange every
        ``exchange_every`` steps (10 sweeps of 2n = 150 proposals at n = 75)
        and an Adam step every ``train_every`` steps.  Stops at the first block
        boundary after some chain reaches E <= target (then ``hit`` holds the
        device time of the first block that saw it)."""
        t = _lib.torch()
        if exchange_every % block or steps % block:
            raise ValueError("steps and exchange_every must be multiples of block")
        if warm:  # one eager step + training step sets kernel attributes outside any capture
            self.step()
            self.train()
            t.cuda.synchronize()
        start_ev, end_ev = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        stream = t.cuda.current_stream()
        wall0 = time.perf_counter()
        start_ev.record(stream)
        done = 0
        hit = None
        while done < steps:
            with_exchange = (done + block) % exchange_every == 0
            if graph:
                key = (block, train_every, with_exchange)
                if key not in self._graphs:
                    self._graphs[key] = self._capture(block, train_every, with_exchange)
                _lib.call("n3_graph_launch", self._graphs[key], _lib.stream_ptr(stream))
            else:
                for k in range(block):
                    self.step()
                    if train_every and (k + 1) % train_every == 0:
                        self.train()
                if with_exchange:
                    self.exchange()
            done += block
            if target is not None or max_seconds is not None:
                best = int(self.ch.energy.min().item())
                if target is not None and best <= target:
                    hit = (int(t.argmin(self.ch.energy).item()), done, time.perf_counter() - wall0)
                    break
                if max_seconds is not None and time.perf_counter() - wall0 > max_seconds:
                    break
        end_ev.record(stream)
        end_ev.synchronize()
        seconds = start_ev.elapsed_time(end_ev) / 1e3
        if hit is not None:
            hit = (hit[0], hit[1], seconds)
        C = self.ch.cols.shape[0]
        return RunResult(done // 150, done // 150, done * C * self.moves, seconds, int(self.ch.best_energy.min().item()),
                         hit)

    def release_graphs(self):
        for h in self._graphs.values():
            _lib.lib().n3_graph_destroy(h)
        self._graphs.clear()

    def __del__(self):
        try:
            self.release_graphs()
        except Exception:  # interpreter shutdown
            pass
