"""Exact swap deltas on the B200 (drop-in for ``no_three_75.gpu_delta``).

``score_two_switches_gpu`` keeps the reference plugin's signature and result
(src/no_three_75/gpu_delta.py:86-116): the full score after exchanging the
selected slot's column with each partner slot, int32[2n], illegal partners
marked 1<<30.  It is the ``move_evaluator`` hook of the reference's
``local_search`` (src/no_three_75/search.py:94,124).  The batched functions
below work on device-resident populations (slot-layout columns) and take any
number of moves or anchors per launch.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from .state import pq_to_columns

SENTINEL = _lib.SENTINEL


def _t():
    return _lib.torch()


def _columns(p, q, device):
    t = _t()
    if _lib.is_tensor(p):
        c = t.empty(p.shape[:-1] + (2 * p.shape[-1],), dtype=t.int16, device=device)
        c[..., 0::2] = p
        c[..., 1::2] = q
        return c
    return t.from_numpy(pq_to_columns(p, q)).to(device)


def score_two_switches_gpu(p, q, selected_index: int, current_score: int, badness) -> np.ndarray:
    """Replaces src/no_three_75/gpu_delta.py:86-116 (kernel gpu_delta.py:19-75)."""
    p_host = np.ascontiguousarray(p, dtype=np.int32)
    q_host = np.ascontiguousarray(q, dtype=np.int32)
    bad_host = np.ascontiguousarray(badness, dtype=np.int32)
    if p_host.ndim != 1 or q_host.shape != p_host.shape or bad_host.shape != (2 * len(p_host),):
        raise ValueError("invalid P/Q/badness shapes")
    n = len(p_host)
    if not 2 <= n <= _lib.MAX_N:
        raise ValueError(f"n={n} outside [2, {_lib.MAX_N}]")
    if not 0 <= int(selected_index) < 2 * n:
        raise ValueError("selected index outside [0, 2n)")
    t = _t()
    device = _lib.require_device()
    cols = t.from_numpy(pq_to_columns(p_host, q_host)[None]).to(device)
    bad = t.from_numpy(bad_host[None]).to(device)
    cur = t.tensor([int(current_score)], dtype=t.int32, device=device)
    anchors = t.tensor([[0, int(selected_index)]], dtype=t.int32, device=device)
    out = t.empty((1, 2 * n), dtype=t.int32, device=device)
    _lib.call("n3_two_switch_scores", _lib.ptr(cols), _lib.ptr(bad), _lib.ptr(cur), 1, n, _lib.ptr(anchors), 1,
              _lib.ptr(out), _lib.stream_ptr())
    return out[0].cpu().numpy()


def two_switch_scores(columns, badness, scores, anchors, *, stream=None):
    """Batched partner scores on device tensors: columns int16 [B, 2n], badness
    int32 [B, 2n], scores int32 [B], anchors int32 [A, 2] (state, slot) ->
    int32 [A, 2n] (SENTINEL where illegal)."""
    t = _t()
    B, m = columns.shape
    A = anchors.shape[0]
    out = t.empty((A, m), dtype=t.int32, device=columns.device)
    _lib.call("n3_two_switch_scores", _lib.ptr(columns), _lib.ptr(badness), _lib.ptr(scores), B, m // 2,
              _lib.ptr(anchors), A, _lib.ptr(out), _lib.stream_ptr(stream))
    return out


def transposition_scores(columns, badness, scores, anchors, *, stream=None):
    """Batched same-layer transposition scores -> int32 [A, n] (by partner row)."""
    t = _t()
    B, m = columns.shape
    A = anchors.shape[0]
    out = t.empty((A, m // 2), dtype=t.int32, device=columns.device)
    _lib.call("n3_transposition_scores", _lib.ptr(columns), _lib.ptr(badness), _lib.ptr(scores), B, m // 2,
              _lib.ptr(anchors), A, _lib.ptr(out), _lib.stream_ptr(stream))
    return out


def swap_deltas(columns, moves, *, badness: bool = False, pairs: bool = False, stream=None):
    """Exact dE of each move (state, u, v) -> int32 [M] (SENTINEL if illegal);
    with ``badness=True`` also the per-slot badness change int32 [M, 2n].
    ``pairs=True`` runs the reference's literal pair-by-pair formulation
    (an independent cross-check of the default direction-class kernel)."""
    t = _t()
    device = _lib.require_device()
    host = not _lib.is_tensor(columns)
    c = _lib.as_device(columns, t.int16, device)
    mv = _lib.as_device(moves, t.int32, device)
    if c.ndim != 2 or c.shape[1] % 2 or mv.ndim != 2 or mv.shape[1] != 3:
        raise ValueError("columns must be (B, 2n) and moves (M, 3)")
    B, m = c.shape
    M = mv.shape[0]
    dE = t.empty(M, dtype=t.int32, device=device)
    db = t.empty((M, m), dtype=t.int32, device=device) if badness else None
    name = "n3_swap_delta_pairs" if pairs else "n3_swap_delta"
    _lib.call(name, _lib.ptr(c), B, m // 2, _lib.ptr(mv), M, _lib.ptr(dE), _lib.ptr(db), _lib.stream_ptr(stream))
    if host:
        return (dE.cpu().numpy(), db.cpu().numpy()) if badness else dE.cpu().numpy()
    return (dE, db) if badness else dE


@dataclass(frozen=True)
class DeltaBenchmark:
    """Fields of src/no_three_75/gpu_delta.py:122-131."""

    cpu_seconds: float
    gpu_seconds: float
    repeats: int
    exact_match: bool

    @property
    def speedup(self) -> float:
        return self.cpu_seconds / max(self.gpu_seconds, 1e-12)


def benchmark_delta(p, q, selected_index: int, current_score: int, badness, *, repeats: int,
                    cpu_expected=None, cpu_seconds: float = float("nan")) -> DeltaBenchmark:
    """Harness of src/no_three_75/gpu_delta.py:134-157; the CPU side
    (``cpu_expected``, ``cpu_seconds``) is supplied by the caller."""
    gpu_actual = score_two_switches_gpu(p, q, selected_index, current_score, badness)
    exact = True
    if cpu_expected is not None:
        cpu_expected = np.asarray(cpu_expected)
        s_cpu = cpu_expected >= (1 << 59)
        s_gpu = gpu_actual >= (1 << 29)
        exact = bool(np.array_equal(s_cpu, s_gpu) and
                     np.array_equal(cpu_expected[~s_cpu].astype(np.int32), gpu_actual[~s_gpu]))
    started = time.perf_counter()
    for _ in range(repeats):
        score_two_switches_gpu(p, q, selected_index, current_score, badness)
    return DeltaBenchmark(cpu_seconds, (time.perf_counter() - started) / repeats, repeats, exact)
