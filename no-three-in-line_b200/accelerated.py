"""Drop-in for ``no_three_75.accelerated`` backed by the CUDA kernels.

Same names, arguments and return types as the reference's Numba functions
(src/no_three_75/accelerated.py:14-195): int64 results, illegal partners
marked 1<<60.  ``evaluate_two_switches`` therefore plugs straight into the
reference's ``local_search(move_evaluator=...)`` (src/no_three_75/search.py:94).
``score_and_badness`` also accepts a batch ([B, n] P/Q) and then returns
(int32[B], int64[B, 2n]).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .gpu import score_population_gpu

SENTINEL64 = 1 << 60


def score_and_badness(p, q):
    """Exact triple count and per-slot badness (accelerated.py:14-37)."""
    p = np.asarray(p)
    q = np.asarray(q)
    if p.ndim == 1:
        s, b = score_population_gpu(p[None], q[None], badness=True)
        return int(s[0]), b[0].astype(np.int64)
    s, b = score_population_gpu(p, q, badness=True)
    return s, b.astype(np.int64)


def _partner_scores(name: str, p, q, u: int, current_score: int, badness, width: int):
    t = _lib.torch()
    p = np.ascontiguousarray(p, dtype=np.int32)
    q = np.ascontiguousarray(q, dtype=np.int32)
    n = len(p)
    bad = np.ascontiguousarray(badness, dtype=np.int32)
    if p.ndim != 1 or q.shape != p.shape or bad.shape != (2 * n,):
        raise ValueError("invalid P/Q/badness shapes")
    if not 2 <= n <= _lib.MAX_N:
        raise ValueError(f"n={n} outside [2, {_lib.MAX_N}]")
    device = _lib.require_device()
    from .state import pq_to_columns

    cols = t.from_numpy(pq_to_columns(p, q)[None]).to(device)
    dbad = t.from_numpy(bad[None]).to(device)
    cur = t.tensor([int(current_score)], dtype=t.int32, device=device)
    anchors = t.tensor([[0, int(u)]], dtype=t.int32, device=device)
    out = t.empty((1, width), dtype=t.int32, device=device)
    _lib.call(name, _lib.ptr(cols), _lib.ptr(dbad), _lib.ptr(cur), 1, n, _lib.ptr(anchors), 1, _lib.ptr(out),
              _lib.stream_ptr())
    res = out[0].cpu().numpy().astype(np.int64)
    res[res >= _lib.SENTINEL] = SENTINEL64
    return res


def evaluate_two_switches(p, q, selected_index: int, current_score: int, badness) -> np.ndarray:
    """accelerated.py:122-195: scores of every degree-preserving 2-switch
    involving the selected slot, int64[2n] with sentinel 1<<60."""
    n = len(p)
    if not 0 <= int(selected_index) < 2 * n:
        raise ValueError("selected index outside [0, 2n)")
    return _partner_scores("n3_two_switch_scores", p, q, selected_index, current_score, badness, 2 * n)


def evaluate_transpositions(p, q, layer: int, selected_row: int, current_score: int, badness) -> np.ndarray:
    """accelerated.py:40-119: same-layer transpositions of (layer, row) with
    every partner row, int64[n] with sentinel 1<<60."""
    n = len(p)
    if layer not in (0, 1) or not 0 <= int(selected_row) < n:
        raise ValueError("layer must be 0/1 and row inside [0, n)")
    return _partner_scores("n3_transposition_scores", p, q, 2 * int(selected_row) + int(layer), current_score,
                           badness, n)


def legal_three_cycle_candidates(p, q, selected_index: int) -> np.ndarray:
    """search.py:38-65 (host enumeration): (selected, v, w, orientation) for
    v < w in two other distinct rows, three distinct columns, and no row left
    with a repeated column after the cycle; int32 [M, 4]."""
    n = len(p)
    cols = np.empty(2 * n, dtype=np.int64)
    cols[0::2], cols[1::2] = np.asarray(p), np.asarray(q)
    srow = int(selected_index) // 2
    su = int(selected_index)
    out = []
    for v in range(2 * n - 1):
        if v // 2 == srow:
            continue
        for w in range(v + 1, 2 * n):
            if w // 2 in (srow, v // 2):
                continue
            if len({int(cols[su]), int(cols[v]), int(cols[w])}) != 3:
                continue
            ou, ov, ow = su ^ 1, v ^ 1, w ^ 1
            if cols[v] != cols[ou] and cols[w] != cols[ov] and cols[su] != cols[ow]:
                out.append((su, v, w, 0))  # u <- v, v <- w, w <- u
            if cols[w] != cols[ou] and cols[v] != cols[ow] and cols[su] != cols[ov]:
                out.append((su, v, w, 1))  # u <- w, w <- v, v <- u
    return np.asarray(out, dtype=np.int32).reshape((-1, 4))


_lib.register("n3_three_cycle_scores", [_lib._P, _lib._P, _lib._I, _lib._P, _lib._I, _lib._I64, _lib._P, _lib._P])


def evaluate_three_cycles(p, q, candidates, current_score: int, badness=None) -> np.ndarray:
    """accelerated.py:196-276: score after each three-cycle candidate
    (u, v, w, orientation), int64; exact on the device (O(n) per candidate).
    ``badness`` is accepted for the reference's signature and not needed.
    Candidates that search.py:38-65 would not generate score 1<<60."""
    t = _lib.torch()
    p = np.ascontiguousarray(p, dtype=np.int32)
    q = np.ascontiguousarray(q, dtype=np.int32)
    cand = np.ascontiguousarray(np.asarray(candidates, dtype=np.int32).reshape(-1, 4))
    n = len(p)
    if p.ndim != 1 or q.shape != p.shape:
        raise ValueError("invalid P/Q shapes")
    if not 3 <= n <= _lib.MAX_N:
        raise ValueError(f"n={n} outside [3, {_lib.MAX_N}]")
    if len(cand) == 0:
        return np.empty(0, dtype=np.int64)
    device = _lib.require_device()
    dp, dq = t.from_numpy(p).to(device), t.from_numpy(q).to(device)
    dc = t.from_numpy(cand).to(device)
    out = t.empty(len(cand), dtype=t.int64, device=device)
    _lib.call("n3_three_cycle_scores", _lib.ptr(dp), _lib.ptr(dq), n, _lib.ptr(dc), len(cand), int(current_score),
              _lib.ptr(out), _lib.stream_ptr())
    return out.cpu().numpy()
