"""Conflict analysis of point sets (drop-in for ``no_three_75.conflicts``,
src/no_three_75/conflicts.py:13-83).

``analyze_points`` returns the reference's ``ConflictMetrics``: every line of
three or more points with its canonical key, its sorted points and C(k, 3),
each point's badness C(k - 1, 2) summed over its lines, the slope histogram
and the summary counts.  The lines are found on the device (``n3_analyze_lines``:
one warp per point set, direction histograms, no pair loop); the host decodes
the records, sorts the lines as the reference does (by -triples, then key) and
sums the histogram and the optional line-weighted score from them.
``analyze_population`` analyses many point sets of one size in one launch.
"""
from __future__ import annotations

import ctypes
from collections import Counter
from dataclasses import dataclass
from math import comb

import numpy as np

from . import _lib
from .geometry import LineKey, Point, primitive_slope

_lib.register("n3_analyze_lines", [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p])

MAX_POINTS = 160
GRID = 75
_LINE_WORDS = 9
_ERR_CAPACITY = 32


@dataclass(frozen=True)
class ViolatingLine:
    key: LineKey
    points: tuple[Point, ...]
    triples: int


@dataclass(frozen=True)
class ConflictMetrics:
    triples: int
    violating_lines: int
    max_line_occupancy: int
    max_point_badness: int
    weighted_score: int
    badness: tuple[int, ...]
    lines: tuple[ViolatingLine, ...]
    slope_histogram: dict[tuple[int, int], int]

    @property
    def lexicographic(self) -> tuple[int, int, int, int]:
        return self.triples, self.violating_lines, self.max_point_badness, self.weighted_score


def _max_lines(m: int) -> int:
    """Every pair lies on one line and a line of k >= 3 points holds C(k, 2) >= 3
    pairs, so a set of m points has at most C(m, 2) / 3 such lines."""
    return max(1, comb(m, 2) // 3)


def _device_lines(sets: np.ndarray, capacity: int):
    t = _lib.torch()
    dev = _lib.require_device()
    B, m = sets.shape[0], sets.shape[1]
    pts = t.from_numpy(np.ascontiguousarray(sets, np.int16)).to(dev)
    badness = t.zeros((B, m), dtype=t.int32, device=dev)
    count = t.zeros(B, dtype=t.int32, device=dev)
    lines = t.empty((B, capacity, _LINE_WORDS), dtype=t.int32, device=dev)
    err = t.zeros(1, dtype=t.int32, device=dev)
    _lib.call("n3_analyze_lines", pts.data_ptr(), B, m, badness.data_ptr(), count.data_ptr(), lines.data_ptr(),
              capacity, err.data_ptr(), _lib.stream_ptr())
    return badness.cpu().numpy(), count.cpu().numpy(), lines.cpu().numpy(), int(err.item())


def _metrics(points: list[Point], badness, records, line_weights) -> ConflictMetrics:
    lines = []
    hist: Counter = Counter()
    triples = weighted = 0
    for rec in records:
        key = (int(rec[0]), int(rec[1]), int(rec[2]))
        k = int(rec[3])
        words = rec[4:].astype(np.uint32)
        idx = [32 * w + b for w in range(5) for b in range(32) if (int(words[w]) >> b) & 1]
        if len(idx) != k:
            raise AssertionError(f"line {key}: {len(idx)} members recorded for occupancy {k}")
        line_triples = comb(k, 3)
        triples += line_triples
        weighted += (line_weights.get(key, 1) if line_weights else 1) * line_triples
        lines.append(ViolatingLine(key, tuple(sorted(points[i] for i in idx)), line_triples))
        hist[primitive_slope(key)] += line_triples
    lines.sort(key=lambda line: (-line.triples, line.key))
    bad = tuple(int(x) for x in badness)
    return ConflictMetrics(triples=triples, violating_lines=len(lines),
                           max_line_occupancy=max((len(line.points) for line in lines), default=2),
                           max_point_badness=max(bad, default=0), weighted_score=weighted, badness=bad,
                           lines=tuple(lines), slope_histogram=dict(hist))


def analyze_population(point_sets, line_weights: dict[LineKey, int] | None = None,
                       capacity: int = 1024) -> list[ConflictMetrics]:
    """``analyze_points`` of B point sets of equal size m (array [B, m, 2] or a
    list of point lists), in one device launch.  Sets with more than
    ``capacity`` lines are run again with room for the most a set can have."""
    sets = np.asarray(point_sets, dtype=np.int64)
    if sets.size == 0 and sets.ndim < 3:
        sets = sets.reshape(len(point_sets), 0, 2)
    if sets.ndim != 3 or sets.shape[2] != 2:
        raise ValueError("point sets must have shape (B, m, 2)")
    B, m = sets.shape[0], sets.shape[1]
    if m > MAX_POINTS:
        raise ValueError(f"at most {MAX_POINTS} points per set")
    if np.any(sets < 0) or np.any(sets >= GRID):
        raise ValueError(f"coordinates must lie in [0, {GRID})")
    if B == 0:
        return []
    capacity = max(1, min(capacity, _max_lines(m)))
    badness, count, lines, err = _device_lines(sets, capacity)
    out: list[ConflictMetrics | None] = [None] * B
    redo = []
    for b in range(B):
        if count[b] >= 0:
            continue
        pts = [tuple(p) for p in sets[b].tolist()]
        if len(set(pts)) != len(pts):
            raise ValueError("two distinct points are required")
        redo.append(b)
    if redo:
        if not err & _ERR_CAPACITY:
            raise RuntimeError(f"n3_analyze_lines: device error bits {err:#x}")
        badness_r, count_r, lines_r, err_r = _device_lines(sets[redo], _max_lines(m))
        if np.any(count_r < 0):
            raise RuntimeError(f"n3_analyze_lines: device error bits {err_r:#x}")
        for k, b in enumerate(redo):
            out[b] = _metrics([tuple(p) for p in sets[b].tolist()], badness_r[k], lines_r[k, :count_r[k]],
                              line_weights)
    for b in range(B):
        if out[b] is None:
            out[b] = _metrics([tuple(p) for p in sets[b].tolist()], badness[b], lines[b, :count[b]], line_weights)
    return out  # type: ignore[return-value]


def analyze_points(points: list[Point], line_weights: dict[LineKey, int] | None = None) -> ConflictMetrics:
    """conflicts.py:36-72 for one point list."""
    pts = [(int(r), int(c)) for r, c in points]
    return analyze_population(np.asarray(pts, np.int64).reshape(1, len(pts), 2), line_weights)[0]


def full_triple_score(points: list[Point]) -> int:
    """Number of collinear triples of a point list (conflicts.py:75-76): the
    sum of C(k, 3) over its lines, counted on the device."""
    return analyze_points(points).triples


def reference_swap_delta(state, layer: int, row_a: int, row_b: int) -> int:
    """Full-recompute delta of a same-layer row swap (conflicts.py:79-83),
    both states scored on the device."""
    from . import gpu

    candidate = state.swapped(layer, row_a, row_b)
    p = np.asarray([state.P, candidate.P], np.int32)
    q = np.asarray([state.Q, candidate.Q], np.int32)
    scores = gpu.score_population_gpu(p, q)
    return int(scores[1]) - int(scores[0])
