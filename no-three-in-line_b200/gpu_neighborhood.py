"""Four-cycle and double-switch neighbourhood scans (drop-in for
``no_three_75.gpu_neighborhood``).

``best_four_cycle`` / ``best_double_switch`` keep the reference's signatures
and results (src/no_three_75/gpu_neighborhood.py:70-211): every candidate
through the anchor slot in the reference's enumeration order, the first
lowest-scoring legal one kept if it improves on the state, the same
``evaluated`` / ``legal`` counts.  The reference builds every candidate state
on the host (3.1 M states at n = 75 for a four-cycle scan) and rescores each in
full on the GPU; here one kernel scores every candidate exactly from direction
histograms of the 12 positions a slot set's candidates can take
(libn3 ``n3_neighborhood_scan``), and the host only decodes the winner and
checks it with the two independent device counts.  ``batch_size`` is accepted
for the reference's signature; the scan needs no batching.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass
from itertools import combinations, permutations

import numpy as np

from . import _lib
from .accelerated import score_and_badness
from .state import PairPermutations, points_to_permutations

_lib.register("n3_neighborhood_scan", [_lib._P, _lib._P, _lib._I, _lib._I, _lib._I64, _lib._P, _lib._P, _lib._P])


@dataclass(frozen=True)
class FourCycleResult:
    """gpu_neighborhood.py:14-21."""
    state: PairPermutations
    score: int
    anchor_index: int
    evaluated: int
    legal: int
    elapsed_seconds: float


@dataclass(frozen=True)
class DoubleSwitchResult:
    """gpu_neighborhood.py:24-31."""
    state: PairPermutations
    score: int
    anchor_index: int
    evaluated: int
    legal: int
    elapsed_seconds: float


def _values_state(values: np.ndarray) -> PairPermutations:
    """gpu_neighborhood.py:34-37."""
    n = values.shape[0]
    points = [(row, int(values[row, layer])) for row in range(n) for layer in range(2)]
    return points_to_permutations(points, n)


def bad_anchor_indices(state: PairPermutations, limit: int) -> list[int]:
    """gpu_neighborhood.py:128-132: slots by decreasing badness, then index."""
    _, badness = score_and_badness(np.asarray(state.P, dtype=np.int32), np.asarray(state.Q, dtype=np.int32))
    return sorted(range(2 * state.n), key=lambda index: (-int(badness[index]), index))[:limit]


def _scan(state: PairPermutations, anchor_index: int):
    state.validate()
    n = state.n
    if not (0 <= anchor_index < 2 * n):
        raise ValueError("anchor index outside point slots")
    if not 5 <= n <= _lib.MAX_N:
        raise ValueError(f"n={n} outside [5, {_lib.MAX_N}]")
    t = _lib.torch()
    device = _lib.require_device()
    p = np.asarray(state.P, dtype=np.int32)
    q = np.asarray(state.Q, dtype=np.int32)
    base_score = int(score_and_badness(p, q)[0])
    dp, dq = t.from_numpy(p).to(device), t.from_numpy(q).to(device)
    out = t.empty(4, dtype=t.int64, device=device)
    _lib.call("n3_neighborhood_scan", _lib.ptr(dp), _lib.ptr(dq), n, int(anchor_index), base_score, _lib.ptr(out),
              _lib.ptr(out) + 16, _lib.stream_ptr())
    best4, best2, legal4, legal2 = (int(x) for x in out.cpu().numpy().view(np.uint64))
    return n, p, q, base_score, (best4, legal4), (best2, legal2)


def _slot_set(n: int, anchor: int, combo_layers: int):
    """Decode (row triple, layer choice) number k of gpu_neighborhood.py:108-110."""
    others = [row for row in range(n) if row != anchor // 2]
    rows = list(combinations(others, 3))[combo_layers // 8]
    layers = combo_layers % 8
    return tuple(2 * r + ((layers >> (2 - i)) & 1) for i, r in enumerate(rows))


def _apply(base: np.ndarray, targets, sources) -> np.ndarray:
    flat = base.reshape(-1)
    changed = flat.copy()
    changed[list(targets)] = flat[list(sources)]
    return changed.reshape(base.shape)


def _verified(values: np.ndarray, score: int, what: str) -> None:
    """The reference re-scores the winner on the CPU (gpu_neighborhood.py:101-103);
    here both independent device counts (determinant and slope) must give it."""
    from .gpu import score_checked_gpu
    from .state import pq_to_columns

    checked = score_checked_gpu(pq_to_columns(values[None, :, 0], values[None, :, 1]), raise_on_mismatch=False)
    exact = int(checked.scores[0])
    if exact != score or checked.mismatches:
        raise AssertionError(f"GPU {what} score {score} != full score {exact}")


def best_four_cycle(state: PairPermutations, anchor_index: int, *, batch_size: int = 32768) -> FourCycleResult:
    """gpu_neighborhood.py:70-125."""
    started = time.perf_counter()
    n, p, q, base_score, (key, legal), _ = _scan(state, anchor_index)
    base = np.column_stack((p, q)).astype(np.int32)
    combos = (n - 1) * (n - 2) * (n - 3) // 6
    evaluated = combos * 8 * 6
    best_score, best_values = base_score, base
    if legal and (key >> 32) < base_score:
        idx = key & 0xFFFFFFFF
        order = list(permutations(_slot_set(n, anchor_index, idx // 6)))[idx % 6]
        targets = (anchor_index,) + tuple(order)
        best_score = int(key >> 32)
        best_values = _apply(base, targets, targets[1:] + targets[:1])
        _verified(best_values, best_score, "four-cycle")
    return FourCycleResult(_values_state(best_values), best_score, anchor_index, evaluated, legal,
                           time.perf_counter() - started)


def best_double_switch(state: PairPermutations, anchor_index: int, *, batch_size: int = 32768) -> DoubleSwitchResult:
    """gpu_neighborhood.py:135-211."""
    started = time.perf_counter()
    n, p, q, base_score, _, (key, legal) = _scan(state, anchor_index)
    base = np.column_stack((p, q)).astype(np.int32)
    combos = (n - 1) * (n - 2) * (n - 3) // 6
    evaluated = combos * 8 * 3
    best_score, best_values = base_score, base
    if legal and (key >> 32) < base_score:
        idx = key & 0xFFFFFFFF
        a, b, c = _slot_set(n, anchor_index, idx // 3)
        sources = ((a, anchor_index, c, b), (b, c, anchor_index, a), (c, b, a, anchor_index))[idx % 3]
        best_score = int(key >> 32)
        best_values = _apply(base, (anchor_index, a, b, c), sources)
        _verified(best_values, best_score, "double-switch")
    return DoubleSwitchResult(_values_state(best_values), best_score, anchor_index, evaluated, legal,
                              time.perf_counter() - started)
