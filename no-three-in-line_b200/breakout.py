"""Line-weighted energies of breakout search (drop-in for the scoring helpers of
``no_three_75.breakout``, src/no_three_75/breakout.py:39-86).

Breakout search raises the weight of lines that stay occupied at a plateau; a
line key ``(a, b, c)`` (the points with ``a*row + b*col + c == 0``, as
``geometry.canonical_line`` writes them) of weight ``w > 1`` adds
``(w - 1) * C(occupancy, 3)`` to the triple count.  ``weighted_candidate_scores``
re-weights the partner scores of a 2-switch evaluator (``evaluate_two_switches``)
and ``weighted_state_score`` a state's score; both run on the device
(``n3_weighted_switch_scores``, ``n3_weighted_state_scores``).
"""
from __future__ import annotations

import numpy as np

from . import _lib

_lib.register("n3_weighted_switch_scores", [_lib._P, _lib._P, _lib._I, _lib._I, _lib._P, _lib._P, _lib._P, _lib._I,
                                            _lib._P, _lib._P])
_lib.register("n3_weighted_state_scores", [_lib._P, _lib._P, _lib._I, _lib._I, _lib._P, _lib._P, _lib._P, _lib._I,
                                           _lib._P, _lib._P])

LineKey = tuple[int, int, int]


def _weight_arrays(weights: dict[LineKey, int]):
    keys = list(weights.items())
    lines = np.asarray([k for k, _ in keys], dtype=np.int64).reshape(-1, 3)
    if lines.size and (np.abs(lines) > np.iinfo(np.int32).max).any():
        raise ValueError("line coefficients must fit in int32")
    w = np.asarray([min(max(int(v), -(2**31)), 2**31 - 1) for _, v in keys], dtype=np.int32)
    return lines.astype(np.int32), w


def weighted_candidate_scores(p, q, selected_index: int, raw_scores, weights: dict[LineKey, int]) -> np.ndarray:
    """breakout.py:39-75: int64 [2n] raw partner scores plus the weighted extra of
    each partner's state."""
    raw = np.asarray(raw_scores).astype(np.int64, copy=True)
    if not weights or not any(int(w) > 1 for w in weights.values()):
        return raw
    t = _lib.torch()
    dev = _lib.require_device()
    p = np.ascontiguousarray(p, dtype=np.int32)
    q = np.ascontiguousarray(q, dtype=np.int32)
    n = len(p)
    if raw.shape != (2 * n,):
        raise ValueError("raw_scores must have 2n entries")
    lines, w = _weight_arrays(weights)
    d = lambda a: t.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    dp, dq, draw, dl, dw = d(p), d(q), d(raw), d(lines), d(w)
    out = t.empty(2 * n, dtype=t.int64, device=dev)
    _lib.call("n3_weighted_switch_scores", _lib.ptr(dp), _lib.ptr(dq), n, int(selected_index), _lib.ptr(draw),
              _lib.ptr(dl), _lib.ptr(dw), len(w), _lib.ptr(out), _lib.stream_ptr())
    return out.cpu().numpy()


def weighted_state_scores(p_batch, q_batch, raw_scores, weights: dict[LineKey, int]) -> np.ndarray:
    """weighted_state_score for every state of a P/Q batch [B, n]; int64 [B]."""
    p = np.ascontiguousarray(p_batch, dtype=np.int32)
    q = np.ascontiguousarray(q_batch, dtype=np.int32)
    raw = np.ascontiguousarray(raw_scores, dtype=np.int64)
    if p.ndim != 2 or q.shape != p.shape or raw.shape != (p.shape[0],):
        raise ValueError("P/Q must be [B, n] and raw scores [B]")
    if not weights:
        return raw.copy()
    t = _lib.torch()
    dev = _lib.require_device()
    lines, w = _weight_arrays(weights)
    d = lambda a: t.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    dp, dq, draw, dl, dw = d(p), d(q), d(raw), d(lines), d(w)  # held until the kernel has run
    out = t.empty(p.shape[0], dtype=t.int64, device=dev)
    _lib.call("n3_weighted_state_scores", _lib.ptr(dp), _lib.ptr(dq), p.shape[0], p.shape[1], _lib.ptr(draw),
              _lib.ptr(dl), _lib.ptr(dw), len(w), _lib.ptr(out), _lib.stream_ptr())
    return out.cpu().numpy()


def weighted_state_score(p, q, raw_score: int, weights: dict[LineKey, int]) -> int:
    """breakout.py:78-86."""
    if not weights:
        return int(raw_score)
    return int(weighted_state_scores(np.asarray(p)[None], np.asarray(q)[None], [int(raw_score)], weights)[0])
