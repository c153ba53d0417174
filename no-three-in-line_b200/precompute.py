"""Line tables of the n x n grid and the two table scorers (drop-in for
``no_three_75.precompute``, src/no_three_75/precompute.py:18-127).

``build_geometry_tables`` builds the reference's tables on the device
(``n3_line_tables_count``, ``n3_line_tables_build``): every line with three or
more grid points that is neither a row nor a column (the lines that
``cp_sat._multi_point_lines`` finds on the whole grid, cp_sat.py:129-157),
numbered in the reference's order, with

* ``pair_to_line``: int32, the line of each unordered pair of grid points in
  ``triangular_pair_index`` order, or -1;
* ``offsets`` (int64) and ``indices`` (int32): the lines' members as CSR, each
  line in row-major order.

The arrays come back as host NumPy arrays, as the reference returns them, and a
device copy stays attached for the scorers.  ``score_pair_table`` and
``score_csr`` score a point list from the tables on the device
(``n3_lines_score_pairs``, ``n3_lines_score_csr``); the ``*_population``
forms score a P/Q batch.  Results equal the reference's for the same inputs,
exceptions included: ``score_pair_table`` raises ValueError for a repeated or
out-of-range point, ``score_csr`` indexes like NumPy (a negative id wraps, an id
beyond the grid raises IndexError).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib

_lib.register("n3_line_tables_count", [_lib._I, _lib._P, _lib._P, _lib._P, _lib._P])
_lib.register("n3_line_tables_build", [_lib._I, _lib._P, _lib._P, _lib._I64, _lib._P, _lib._P, _lib._P, _lib._P])
_lib.register("n3_lines_score_pairs", [_lib._P, _lib._P, _lib._I, _lib._I, _lib._P, _lib._P, _lib._P, _lib._P])
_lib.register("n3_lines_score_csr", [_lib._P, _lib._P, _lib._I, _lib._I, _lib._I64, _lib._P, _lib._P, _lib._P,
                                     _lib._P, _lib._P, _lib._P])

MAX_PAIR_POINTS = 512  # points per list that the device pair-table scorer takes
_ERR_RANGE, _ERR_TWICE, _ERR_HASH = 1, 2, 4  # error-word bits of n3_lines_score_pairs


@dataclass(frozen=True)
class DeviceTables:
    """The tables in device memory (torch tensors)."""

    pair_to_line: object
    offsets: object
    indices: object


@dataclass(frozen=True)
class GeometryTables:
    """precompute.py:18-25, plus the device copy the scorers read."""

    n: int
    pair_to_line: np.ndarray
    offsets: np.ndarray
    indices: np.ndarray
    line_count: int
    build_seconds: float
    device: DeviceTables | None = field(default=None, repr=False, compare=False)


def triangular_pair_index(left: int, right: int, point_count: int) -> int:
    """precompute.py:28-33: index of the unordered pair {left, right} in the
    row-major upper triangle of a point_count x point_count matrix."""
    if left > right:
        left, right = right, left
    if left == right or left < 0 or right >= point_count:
        raise ValueError("pair index requires two distinct in-range points")
    return left * (2 * point_count - left - 1) // 2 + right - left - 1


def _check_n(n) -> int:
    if type(n) is not int or n < 1 or n > _lib.MAX_N:
        raise ValueError(f"n must be an integer in [1, {_lib.MAX_N}]")
    return n


def build_geometry_tables(n: int) -> GeometryTables:
    """precompute.py:35-57, built on the device; build_seconds includes the
    copies back to the host."""
    started = time.perf_counter()
    n = _check_n(n)
    t = _lib.torch()
    dev = _lib.require_device()
    N = n * n
    pairs = N * (N - 1) // 2
    line_at = t.empty(N + 1, dtype=t.int64, device=dev)
    incidence_at = t.empty(N + 1, dtype=t.int64, device=dev)
    totals = np.zeros(2, dtype=np.int64)
    s = _lib.stream_ptr()
    _lib.call("n3_line_tables_count", n, _lib.ptr(line_at), _lib.ptr(incidence_at), totals.ctypes.data, s)
    line_count, incidences = int(totals[0]), int(totals[1])
    offsets = t.empty(line_count + 1, dtype=t.int64, device=dev)
    indices = t.empty(max(incidences, 1), dtype=t.int32, device=dev)[:incidences]
    pair_to_line = t.empty(max(pairs, 1), dtype=t.int32, device=dev)[:pairs]
    _lib.call("n3_line_tables_build", n, _lib.ptr(line_at), _lib.ptr(incidence_at), line_count, _lib.ptr(offsets),
              _lib.ptr(indices), _lib.ptr(pair_to_line), s)
    host = (pair_to_line.cpu().numpy(), offsets.cpu().numpy(), indices.cpu().numpy())
    return GeometryTables(n, host[0], host[1], host[2], line_count, time.perf_counter() - started,
                          DeviceTables(pair_to_line, offsets, indices))


def _device_tables(tables: GeometryTables) -> DeviceTables:
    """The attached device copy, or a fresh upload of tables built elsewhere."""
    if tables.device is not None:
        return tables.device
    t = _lib.torch()
    dev = _lib.require_device()
    up = lambda a, dt: t.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(dev)  # noqa: E731
    return DeviceTables(up(tables.pair_to_line, np.int32), up(tables.offsets, np.int64),
                        up(tables.indices, np.int32))


def _run_pairs(id_lists: list[np.ndarray], n: int, tables: GeometryTables) -> np.ndarray:
    t = _lib.torch()
    dev = _lib.require_device()
    d = _device_tables(tables)
    starts = np.zeros(len(id_lists) + 1, dtype=np.int64)
    np.cumsum([len(x) for x in id_lists], out=starts[1:])
    flat = np.concatenate(id_lists).astype(np.int32) if id_lists else np.zeros(0, np.int32)
    d_ids = t.from_numpy(np.ascontiguousarray(flat)).to(dev) if flat.size else t.zeros(1, dtype=t.int32, device=dev)
    d_starts = t.from_numpy(starts).to(dev)
    scores = t.empty(len(id_lists), dtype=t.int64, device=dev)
    err = t.zeros(1, dtype=t.int32, device=dev)
    _lib.call("n3_lines_score_pairs", _lib.ptr(d_ids), _lib.ptr(d_starts), len(id_lists), n,
              _lib.ptr(d.pair_to_line) if d.pair_to_line.numel() else None, _lib.ptr(scores), _lib.ptr(err),
              _lib.stream_ptr())
    code = int(err.item())
    if code & (_ERR_RANGE | _ERR_TWICE):
        raise ValueError("pair index requires two distinct in-range points")
    if code:
        raise RuntimeError(f"pair-table scorer: error word {code:#x}")
    return scores.cpu().numpy()


def _run_csr(id_lists: list[np.ndarray], n: int, tables: GeometryTables) -> np.ndarray:
    t = _lib.torch()
    dev = _lib.require_device()
    d = _device_tables(tables)
    starts = np.zeros(len(id_lists) + 1, dtype=np.int64)
    np.cumsum([len(x) for x in id_lists], out=starts[1:])
    flat = np.concatenate(id_lists).astype(np.int32) if id_lists else np.zeros(0, np.int32)
    d_ids = t.from_numpy(np.ascontiguousarray(flat)).to(dev) if flat.size else t.zeros(1, dtype=t.int32, device=dev)
    d_starts = t.from_numpy(starts).to(dev)
    groups = (len(id_lists) + 31) // 32
    occupancy = t.empty(groups * n * n, dtype=t.int32, device=dev)
    scores = t.empty(len(id_lists), dtype=t.int64, device=dev)
    err = t.zeros(1, dtype=t.int32, device=dev)
    _lib.call("n3_lines_score_csr", _lib.ptr(d_ids), _lib.ptr(d_starts), len(id_lists), n, int(tables.line_count),
              _lib.ptr(d.offsets), _lib.ptr(d.indices) if d.indices.numel() else None, _lib.ptr(occupancy),
              _lib.ptr(scores), _lib.ptr(err), _lib.stream_ptr())
    if int(err.item()):
        raise IndexError("a point id is out of bounds for the grid")
    return scores.cpu().numpy()


def score_pair_table(points, tables: GeometryTables) -> int:
    """precompute.py:60-81: sum of C(k, 3) over the table's lines, from the
    lines of the points' pairs (a CTA per list, a warp per anchor point)."""
    n = tables.n
    ids = sorted(row * n + column for row, column in points)
    if len(ids) < 2:
        return 0  # no pair: the reference's score is 0
    N = n * n
    if ids[0] < 0 or ids[-1] >= N or any(a == b for a, b in zip(ids, ids[1:])):
        raise ValueError("pair index requires two distinct in-range points")
    if len(ids) > MAX_PAIR_POINTS:
        raise ValueError(f"the device pair-table scorer takes at most {MAX_PAIR_POINTS} points")
    return int(_run_pairs([np.asarray(ids, dtype=np.int32)], n, tables)[0])


def _csr_ids(points, n: int) -> np.ndarray:
    """NumPy index semantics of ``occupied[ids] = 1``: negative ids wrap."""
    N = n * n
    ids = [row * n + column for row, column in points]
    for v in ids:
        if v >= N or v < -N:
            raise IndexError(f"index {v} is out of bounds for axis 0 with size {N}")
    return np.asarray([v + N if v < 0 else v for v in ids], dtype=np.int32)


def score_csr(points, tables: GeometryTables) -> int:
    """precompute.py:84-89: occupancy summed over every line's members (32
    point lists per occupancy word, bit-sliced counts)."""
    return int(_run_csr([_csr_ids(points, tables.n)], tables.n, tables)[0])


def _population_ids(p_batch, q_batch, n: int) -> list[np.ndarray]:
    p = np.asarray(p_batch, dtype=np.int64)
    q = np.asarray(q_batch, dtype=np.int64)
    if p.ndim != 2 or q.shape != p.shape or p.shape[1] != n:
        raise ValueError("P/Q must be [B, n] batches for the tables' n")
    if p.size and (p.min() < 0 or q.min() < 0 or p.max() >= n or q.max() >= n):
        raise ValueError("columns must lie in [0, n)")
    rows = np.arange(n) * n
    return [np.concatenate((rows + p[b], rows + q[b])).astype(np.int32) for b in range(p.shape[0])]


def score_pair_table_population(p_batch, q_batch, tables: GeometryTables) -> np.ndarray:
    """score_pair_table of every state of a P/Q batch [B, n]; int64 [B]."""
    ids = _population_ids(p_batch, q_batch, tables.n)
    if 2 * tables.n > MAX_PAIR_POINTS:
        raise ValueError(f"the device pair-table scorer takes at most {MAX_PAIR_POINTS} points")
    return _run_pairs(ids, tables.n, tables) if ids else np.zeros(0, np.int64)


def score_csr_population(p_batch, q_batch, tables: GeometryTables) -> np.ndarray:
    """score_csr of every state of a P/Q batch [B, n]; int64 [B]."""
    ids = _population_ids(p_batch, q_batch, tables.n)
    return _run_csr(ids, tables.n, tables) if ids else np.zeros(0, np.int64)


def _timed(score, calls: int) -> tuple[int, float]:
    """Calls ``score`` ``calls`` times back to back; returns its last result
    and the mean wall time of one call."""
    result = 0
    t0 = time.perf_counter()
    for _ in range(calls):
        result = score()
    return int(result), (time.perf_counter() - t0) / calls


def benchmark_precomputation(n: int, points) -> dict[str, object]:
    """precompute.py:92-127 with the device scorers: A the determinant count
    (``accelerated.score_and_badness``), B the pair table, C the direction-class
    line count (the slope scorer, this engine's canonical-line form), D the CSR
    scan.  The four must agree (AssertionError otherwise)."""
    from .accelerated import score_and_badness
    from .gpu import score_slope_gpu
    from .state import pq_to_columns, points_to_permutations

    pq = points_to_permutations(points, n)
    p, q = np.asarray(pq.P, np.int32), np.asarray(pq.Q, np.int32)
    columns = pq_to_columns(p[None], q[None])
    tables = build_geometry_tables(n)
    scorers = {  # name in the result -> (scorer, calls timed)
        "A_numba_determinants": (lambda: score_and_badness(p, q)[0], 100),
        "B_pair_to_line": (lambda: score_pair_table(points, tables), 100),
        "C_canonical_line_dict": (lambda: score_slope_gpu(columns)[0][0], 5),
        "D_csr_line_scan": (lambda: score_csr(points, tables), 20),
    }
    score_and_badness(p, q)  # first launch outside the timing
    results = {name: _timed(fn, calls) for name, (fn, calls) in scorers.items()}
    scores = {score for score, _ in results.values()}
    if len(scores) != 1:
        raise AssertionError("precompute scorers disagree: " + ", ".join(f"{k}={v[0]}" for k, v in results.items()))
    return {
        "n": n,
        "score": scores.pop(),
        "line_count": tables.line_count,
        "line_incidences": int(len(tables.indices)),
        "build_seconds": tables.build_seconds,
        "memory_bytes": {
            "pair_to_line_triangular": int(tables.pair_to_line.nbytes),
            "csr_offsets": int(tables.offsets.nbytes),
            "csr_indices": int(tables.indices.nbytes),
        },
        "seconds_per_score": {name: seconds for name, (_, seconds) in results.items()},
    }
