"""Exhaustive 2-switch beam search (drop-in for ``no_three_75.gpu_exhaustive_beam``).

``gpu_exhaustive_beam_search`` keeps the reference's signature, validation,
callback and result (src/no_three_75/gpu_exhaustive_beam.py:91-325) and
follows the same search trajectory: the same candidate order, scores, stable
score order, random.Random(seed) shuffle of the candidates within
``energy_window`` of the best, prospect ranking, signature and ``seen`` rules,
and elite ranking.  Where it runs differs (libn3 ``n3_exh_*``):

* every candidate of a generation, all legal 2-switches of all elites that
  touch a bad slot (all slots every ``global_every`` generations), is scored on
  the device exactly from its parent (two direction histograms per partner),
  without building the child; the reference builds every child and rescores
  it in full;
* the quality pool (the first 24 x elite_size candidates of the stable score
  order), the diverse pool (legal candidates within the window, in order), its
  CPython shuffle, the prospect list and the prospects' states are made on the
  device;
* the host keeps the retention rules, which read and grow the set of seen
  state signatures, over the prospects only (at most 48 x elite_size states).

``candidate_descriptors`` is the reference's host enumeration, kept for callers
that use it directly.
"""
from __future__ import annotations

import ctypes
import time
from typing import Callable

import numpy as np

from . import _lib
from .gpu_device_search import (GpuSearchResult, GpuSearchSnapshot, _normalize_raw, elite_key, normalize_rows,
                                 rank_elites)
from .state import PairPermutations

_P = ctypes.c_void_p
_I = ctypes.c_int

_lib.register("n3_exh_candidates", [_P, _P, _P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P])
_lib.register("n3_exh_select", [_P, _P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P])
_lib.register("n3_exh_build_prospects", [_P, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P])
_lib.register("n3_exh_gather_rows", [_P, _P, _P, _I, _I, _P, _P, _P, _P])

INVALID = 1 << 29
ST_ANCHORS, ST_CANDIDATES, ST_LEGAL, ST_QUALITY, ST_DIVERSE, ST_PROSPECTS, ST_ERROR = range(7)
MAX_ELITES = 2048


def candidate_descriptors(badness: np.ndarray, *, global_anchors: bool = False) -> np.ndarray:
    """Every unordered switch touching a bad slot (or every switch), as
    (parent, u, v) rows in the reference's order (gpu_exhaustive_beam.py:67-82)."""
    badness = np.asarray(badness)
    parent_count, edge_count = badness.shape
    rows = []
    for parent in range(parent_count):
        anchors = list(range(edge_count)) if global_anchors else list(map(int, np.flatnonzero(badness[parent])))
        anchor_set = set(anchors)
        for u in anchors:
            for v in range(edge_count):
                if v == u or (v >> 1) == (u >> 1) or (v in anchor_set and v < u):
                    continue
                rows.append((parent, u, v))
    return np.asarray(rows, dtype=np.int32).reshape((-1, 3))


def _signature(p: np.ndarray, q: np.ndarray) -> bytes:
    """The reference's state signature (gpu_exhaustive_beam.py:85-88)."""
    values = np.column_stack((p, q))
    values.sort(axis=1)
    return values.astype(np.int16, copy=False).tobytes()


def _signatures(p: np.ndarray, q: np.ndarray) -> list[bytes]:
    """_signature of every row pair (p[k], q[k]), the rows sorted all at once."""
    p, q = np.asarray(p), np.asarray(q)
    values = np.stack((np.minimum(p, q), np.maximum(p, q)), axis=2)  # each row's pair sorted
    width = values.shape[1] * 4  # bytes of one row's int16 signature
    whole = values.astype(np.int16).tobytes()
    return [whole[k * width:(k + 1) * width] for k in range(len(values))]


class _Buffers:
    """Device buffers of one search, sized for elite_size + 1 elites (the
    reference's retention can keep one elite more than elite_size when
    elite_size is 1)."""

    def __init__(self, n: int, elite_size: int, dev):
        t = _lib.torch()
        m = 2 * n
        E = elite_size + 1
        self.E = E
        C = E * m * (m - 2)
        P = 48 * elite_size
        z = lambda *shape, dtype=t.int32: t.zeros(shape, dtype=dtype, device=dev)  # noqa: E731
        self.elite_p, self.elite_q = z(E, n), z(E, n)
        self.elite_cols = z(E, m, dtype=t.int16)
        self.elite_scores, self.elite_bad = z(E), z(E, m)
        self.tmp_p, self.tmp_q, self.tmp_cols = z(E, n), z(E, n), z(E, m, dtype=t.int16)
        self.anchors, self.start = z(E * m, 2), z(E * m)
        self.partner = z(E * m, m)
        self.cand_score, self.cand_code = z(C), z(C)
        self.quality, self.diverse = z(24 * elite_size), z(C)
        self.in_quality = z(C, dtype=t.uint8)
        self.dpos = z(C)
        self.prospects, self.p_pos, self.p_score = z(P), z(P), z(P)
        self.pp, self.pq, self.parent_of = z(P, n), z(P, n), z(P)
        self.p_scores2, self.p_bad = z(P), z(P, m)
        self.status = z(8, dtype=t.int64)
        self.rng = z(625)
        self.index = z(E)


def _score(buf: _Buffers, p, q, count: int, n: int, scores, bad, stream) -> None:
    _lib.call("n3_score_population", p.data_ptr(), q.data_ptr(), count, n, scores.data_ptr(), bad.data_ptr(), stream)


def _gather(buf: _Buffers, src_p, src_q, idx: np.ndarray, n: int, stream):
    """Rows idx of (src_p, src_q) into the elite buffers (through tmp rows)."""
    t = _lib.torch()
    k = len(idx)
    buf.index[:k].copy_(t.from_numpy(np.ascontiguousarray(idx, np.int32)))
    _lib.call("n3_exh_gather_rows", src_p.data_ptr(), src_q.data_ptr(), buf.index.data_ptr(), k, n,
              buf.tmp_p.data_ptr(), buf.tmp_q.data_ptr(), buf.tmp_cols.data_ptr(), stream)
    buf.elite_p[:k].copy_(buf.tmp_p[:k])
    buf.elite_q[:k].copy_(buf.tmp_q[:k])
    buf.elite_cols[:k].copy_(buf.tmp_cols[:k])


def gpu_exhaustive_beam_search(
    initial: PairPermutations,
    *,
    seed: int,
    generations: int,
    elite_size: int,
    energy_window: int,
    initial_elites: np.ndarray | None = None,
    global_every: int = 25,
    report_every: int = 5,
    callback: Callable[[GpuSearchSnapshot], None] | None = None,
) -> GpuSearchResult:
    """Walk a diverse beam through complete bad-edge 2-switch neighborhoods."""
    initial.validate()
    if initial.n > 75:
        raise ValueError("CUDA kernels support n <= 75")
    if elite_size < 1 or generations < 1:
        raise ValueError("elite_size and generations must be positive")
    if elite_size > MAX_ELITES:
        raise ValueError(f"elite_size must not exceed {MAX_ELITES}")
    t = _lib.torch()
    dev = _lib.require_device()
    stream = _lib.stream_ptr()
    n = initial.n
    base = np.column_stack((initial.P, initial.Q)).astype(np.int32)[None, :, :]
    if initial_elites is not None:
        supplied = np.ascontiguousarray(initial_elites, dtype=np.int32)
        if supplied.ndim != 3 or supplied.shape[1:] != (n, 2):
            raise ValueError("initial_elites must have shape (count,n,2)")
        for values in supplied:
            _normalize_raw(values[:, 0], values[:, 1]).validate()
        base = np.concatenate((base, supplied), axis=0)
    base = base[:elite_size]
    buf = _Buffers(n, elite_size, dev)
    count = len(base)
    host_p, host_q = np.ascontiguousarray(base[:, :, 0]), np.ascontiguousarray(base[:, :, 1])
    buf.tmp_p[:count].copy_(t.from_numpy(host_p))
    buf.tmp_q[:count].copy_(t.from_numpy(host_q))
    _score(buf, buf.tmp_p, buf.tmp_q, count, n, buf.elite_scores, buf.elite_bad, stream)
    scores = buf.elite_scores[:count].cpu().numpy()
    bad = buf.elite_bad[:count].cpu().numpy()
    order = rank_elites(scores, bad)
    staged_p, staged_q = buf.tmp_p.clone(), buf.tmp_q.clone()
    _gather(buf, staged_p, staged_q, order, n, stream)
    _score(buf, buf.elite_p, buf.elite_q, count, n, buf.elite_scores, buf.elite_bad, stream)
    elite_scores = scores[order]
    elite_bad_host = bad[order]
    best_score = int(elite_scores[0])
    best_key = elite_key(best_score, elite_bad_host[0])
    best_p, best_q = host_p[order[0]].copy(), host_q[order[0]].copy()
    seen = {_signature(host_p[i], host_q[i]) for i in range(count)}
    evaluations = count
    _lib.call("n3_py_random_seed", buf.rng.data_ptr(), abs(int(seed)) & (2 ** 64 - 1), stream)
    started = time.perf_counter()
    completed = 0

    for generation in range(1, generations + 1):
        completed = generation
        glob = bool(global_every and generation % global_every == 0)
        _lib.call("n3_exh_candidates", buf.elite_cols.data_ptr(), buf.elite_bad.data_ptr(),
                  buf.elite_scores.data_ptr(), count, n, int(glob), buf.anchors.data_ptr(), buf.start.data_ptr(),
                  buf.partner.data_ptr(), buf.cand_score.data_ptr(), buf.cand_code.data_ptr(),
                  buf.status.data_ptr(), stream)
        if int(buf.status[ST_ANCHORS].item()) == 0:
            break
        _lib.call("n3_exh_select", buf.cand_score.data_ptr(), buf.status.data_ptr(), elite_size, best_score,
                  energy_window, buf.rng.data_ptr(), buf.quality.data_ptr(), buf.diverse.data_ptr(),
                  buf.in_quality.data_ptr(), buf.dpos.data_ptr(), buf.prospects.data_ptr(), buf.p_pos.data_ptr(),
                  buf.p_score.data_ptr(), int(buf.cand_score.numel()), stream)
        status = buf.status.cpu().numpy()
        if status[ST_ERROR]:
            raise RuntimeError("exhaustive beam: the quality pool's scores span more than 8192 energy levels")
        legal, prospects = int(status[ST_LEGAL]), int(status[ST_PROSPECTS])
        evaluations += legal
        if legal == 0:
            break
        _lib.call("n3_exh_build_prospects", buf.elite_cols.data_ptr(), n, buf.anchors.data_ptr(),
                  buf.cand_code.data_ptr(), buf.prospects.data_ptr(), buf.status.data_ptr(), prospects,
                  buf.pp.data_ptr(), buf.pq.data_ptr(), buf.parent_of.data_ptr(), stream)
        # the prospects' own full counts: their badness, and an audit of the exact scores
        _score(buf, buf.pp, buf.pq, prospects, n, buf.p_scores2, buf.p_bad, stream)
        p_score = buf.p_score[:prospects].cpu().numpy()
        if not np.array_equal(buf.p_scores2[:prospects].cpu().numpy(), p_score):
            raise AssertionError("exhaustive beam: incremental candidate scores differ from full recount")
        p_bad = buf.p_bad[:prospects].cpu().numpy()
        pp = buf.pp[:prospects].cpu().numpy()
        pq = buf.pq[:prospects].cpu().numpy()
        p_pos = buf.p_pos[:prospects].cpu().numpy()
        sigs = _signatures(pp, pq)
        ranked = [int(k) for k in rank_elites(p_score, p_bad)]
        diverse_order = [int(k) for k in np.argsort(np.where(p_pos >= 0, p_pos, np.iinfo(np.int32).max),
                                                    kind="stable")[:int(np.count_nonzero(p_pos >= 0))]]
        quality_count = max(1, elite_size // 4)
        selected: list[int] = []
        selected_signatures: set[bytes] = set()

        def retain(k: int, *, require_unseen: bool) -> bool:
            signature = sigs[k]
            if signature in selected_signatures or (require_unseen and signature in seen):
                return False
            selected.append(k)
            selected_signatures.add(signature)
            return True

        for k in ranked:
            retain(k, require_unseen=True)
            if len(selected) == quality_count:
                break
        for k in diverse_order:
            retain(k, require_unseen=True)
            if len(selected) == elite_size:
                break
        if len(selected) < elite_size:
            for k in ranked + diverse_order:
                retain(k, require_unseen=False)
                if len(selected) == elite_size:
                    break
        if not selected:
            seen.clear()
            selected = ranked[:elite_size]
            selected_signatures = {sigs[k] for k in selected}
        seen.update(selected_signatures)
        if len(seen) > 500000:
            seen = set(selected_signatures)

        sel = np.asarray(selected, dtype=np.int32)
        count = len(sel)
        new_scores = p_score[sel]
        new_bad = p_bad[sel]
        rank = rank_elites(new_scores, new_bad)
        order_in_prospects = sel[rank]
        _gather(buf, buf.pp, buf.pq, order_in_prospects, n, stream)
        _score(buf, buf.elite_p, buf.elite_q, count, n, buf.elite_scores, buf.elite_bad, stream)
        elite_scores = new_scores[rank]
        elite_bad_host = new_bad[rank]
        generation_best = int(elite_scores[0])
        generation_key = elite_key(generation_best, elite_bad_host[0])
        improved = generation_key < best_key
        if improved:
            best_score, best_key = generation_best, generation_key
            best_p, best_q = pp[order_in_prospects[0]].copy(), pq[order_in_prospects[0]].copy()
        if callback is not None and (improved or generation % max(1, report_every) == 0):
            npp, nqq = normalize_rows(pp[order_in_prospects], pq[order_in_prospects])
            normalized = [np.column_stack((a, c)) for a, c in zip(npp, nqq)]
            callback(GpuSearchSnapshot(generation, time.perf_counter() - started, evaluations, generation_best,
                                       best_score, tuple(map(int, elite_scores)), np.asarray(normalized, np.int32),
                                       _normalize_raw(best_p, best_q)))
        if best_score == 0:
            from .gpu import score_checked_gpu
            from .state import pq_to_columns

            state = _normalize_raw(best_p, best_q)
            checked = score_checked_gpu(pq_to_columns(np.asarray([state.P], np.int32),
                                                      np.asarray([state.Q], np.int32)))
            if int(checked.scores[0]) != 0:
                raise AssertionError("beam E=0 failed verification by both device counts")
            break

    return GpuSearchResult(_normalize_raw(best_p, best_q), best_score, completed, evaluations,
                           time.perf_counter() - started, seed)
