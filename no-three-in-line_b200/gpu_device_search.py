"""Device-resident beam search (drop-in for ``no_three_75.gpu_device_search``).

``gpu_device_beam_search`` keeps the reference's signature, validation and
result (src/no_three_75/gpu_device_search.py:254-432) and produces the same
search trajectory: the same mutation draws (xorshift64* per child), the same
scores, the same stable score order, the same random.Random(seed) shuffle of
the children within ``energy_window`` of the best, the same rank_elites order
and elite_key best-so-far rule.  The difference is where it runs: every
generation is five kernel launches on one stream (libn3 ``n3_beam_generation``)
with no copy back to the host, where the reference copies every child's score
to the host, sorts and shuffles in Python and copies the elites back.  Each
child is scored from its parent by the exact delta of each of its swaps (the
reference rescores every child in full); the result is the same integer.  Without
a callback the host synchronises only to stop early (every ``report_every``
generations) and at the end; with a callback it reads an 8-word status after
each generation (the reference's reporting rule needs to know whether the
generation improved) and the elites only on the generations it reports.

``elite_size`` must be at least 2 (the reference's selection loop appends past
``elite_size`` when it is 1) and ``population`` at most 65536.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass
from typing import Callable

import numpy as np

from . import _lib
from .state import PairPermutations

_P = ctypes.c_void_p
_I = ctypes.c_int

STATUS_WORDS = 8


class BeamDesc(ctypes.Structure):
    _fields_ = [("n", _I), ("population", _I), ("elite_size", _I), ("energy_window", _I), ("max_strength", _I),
                ("bad_bias", _I), ("seed", ctypes.c_uint64)] + \
               [(name, _P) for name in ("elite_p", "elite_q", "elite_badness", "elite_scores", "child_p", "child_q",
                                        "child_scores", "pick_p", "pick_q", "pick_badness", "pick_scores",
                                        "selected", "rng", "status", "best_p", "best_q", "history")] + \
               [("history_len", _I)] + \
               [(name, _P) for name in ("child_parent", "child_moves", "child_nmoves", "child_badness",
                                        "error_word")]


_lib.register("n3_beam_mutate", [_P, _P, _P] + [_I] * 7 + [ctypes.c_uint64, _I, _P, _P, _P])
_lib.register("n3_py_random_seed", [_P, ctypes.c_uint64, _P])
_lib.register("n3_py_random_shuffle", [_P, _P, _I, _P])
_lib.register("n3_py_shuffle_steps", [_P, _I, _P, _P])
_lib.register("n3_normalize_pairs", [_P, _P, _I, _I, _P, _P])
_lib.register("n3_beam_init", [ctypes.POINTER(BeamDesc), _I, _P])
_lib.register("n3_beam_generation", [ctypes.POINTER(BeamDesc), _I, _P])


@dataclass(frozen=True)
class GpuSearchSnapshot:
    """src/no_three_75/gpu_search.py:16-25."""
    generation: int
    elapsed_seconds: float
    evaluations: int
    generation_best: int
    best_score: int
    elite_scores: tuple[int, ...]
    elite_values: np.ndarray
    state: PairPermutations


@dataclass(frozen=True)
class GpuSearchResult:
    """src/no_three_75/gpu_search.py:28-35."""
    state: PairPermutations
    score: int
    generations: int
    evaluations: int
    elapsed_seconds: float
    seed: int


def normalize_rows(p, q) -> tuple[np.ndarray, np.ndarray]:
    """Canonical P/Q of every state given as raw rows p[b], q[b] (the columns
    of each row in either order): points_to_permutations of each, by the
    library's host routine n3_normalize_pairs (the same augmenting-path search,
    so the same result).  ValueError if a state is not a row/column 2-factor."""
    p = np.ascontiguousarray(np.atleast_2d(p), dtype=np.int32)
    q = np.ascontiguousarray(np.atleast_2d(q), dtype=np.int32)
    if p.shape != q.shape:
        raise ValueError("P and Q rows must have the same shape")
    po, qo = np.empty_like(p), np.empty_like(q)
    _lib.call("n3_normalize_pairs", p.ctypes.data, q.ctypes.data, p.shape[0], p.shape[1], po.ctypes.data,
              qo.ctypes.data)
    return po, qo


def _normalize_raw(p: np.ndarray, q: np.ndarray) -> PairPermutations:
    """gpu_device_search.py:178-182: raw P/Q rows back to a canonical state."""
    po, qo = normalize_rows(p, q)
    return PairPermutations(tuple(int(x) for x in po[0]), tuple(int(x) for x in qo[0]))


def elite_key(score: int, badness: np.ndarray) -> tuple[int, int, int]:
    """gpu_device_search.py:200-203."""
    values = np.asarray(badness).astype(np.int64)
    return int(score), int(values.max()), int(np.dot(values, values))


def rank_elites(scores: np.ndarray, badness: np.ndarray) -> np.ndarray:
    """gpu_device_search.py:185-197: stable order by (E, max badness, sum of
    squared badness), ties in index order.  The three keys of every row are
    formed at once (int64) and ordered by one stable lexicographic sort, the
    same order as the reference's Python sort by elite_key."""
    scores = np.asarray(scores).astype(np.int64).reshape(-1)
    if len(scores) == 0:
        return np.zeros(0, dtype=np.int32)
    values = np.asarray(badness).astype(np.int64).reshape(len(scores), -1)
    return np.lexsort((np.einsum("ij,ij->i", values, values), values.max(axis=1), scores)).astype(np.int32)


def mutate_population_device(parent_p, parent_q, *, population: int, active_strength: int, max_strength: int,
                             seed: int, generation: int, bad_bias: int = 85, stream=None):
    """gpu_device_search.py:206-251: score the parents' badness, then mutate
    them into ``population`` children on the device; returns host arrays."""
    pp = np.ascontiguousarray(parent_p, dtype=np.int32)
    pq = np.ascontiguousarray(parent_q, dtype=np.int32)
    if pp.ndim != 2 or pq.shape != pp.shape or pp.shape[1] > _lib.MAX_N:
        raise ValueError("P/Q batches must match and n must not exceed 75")
    t = _lib.torch()
    dev = _lib.require_device()
    B, n = pp.shape
    dp, dq = t.from_numpy(pp).to(dev), t.from_numpy(pq).to(dev)
    scores = t.empty(B, dtype=t.int32, device=dev)
    bad = t.empty((B, 2 * n), dtype=t.int32, device=dev)
    s = _lib.stream_ptr(stream)
    _lib.call("n3_score_population", _lib.ptr(dp), _lib.ptr(dq), B, n, _lib.ptr(scores), _lib.ptr(bad), s)
    cp_ = t.empty((population, n), dtype=t.int32, device=dev)
    cq_ = t.empty_like(cp_)
    quality = max(1, min(B, B // 4))
    _lib.call("n3_beam_mutate", _lib.ptr(dp), _lib.ptr(dq), _lib.ptr(bad), B, quality, n, population,
              active_strength, max_strength, bad_bias, seed & (2**64 - 1), generation, _lib.ptr(cp_), _lib.ptr(cq_),
              s)
    return cp_.cpu().numpy(), cq_.cpu().numpy()


def py_random_shuffle_device(values, seed: int):
    """random.Random(seed).shuffle(values) computed on the device (the RNG
    walk the beam search uses); returns the shuffled host array."""
    t = _lib.torch()
    dev = _lib.require_device()
    v = t.from_numpy(np.ascontiguousarray(values, dtype=np.int32)).to(dev)
    state = t.empty(625, dtype=t.int32, device=dev)
    _lib.call("n3_py_random_seed", _lib.ptr(state), abs(int(seed)) & (2**64 - 1), None)
    _lib.call("n3_py_random_shuffle", _lib.ptr(state), _lib.ptr(v), int(v.numel()), None)
    return v.cpu().numpy()


def py_shuffle_steps_device(counts, seed: int):
    """The j of every step of random.Random(seed).shuffle over each count in
    ``counts`` in turn (one generator), resolved on the device as the beam
    selection resolves its shuffle; returns one int32 array per count
    (entry s = the j of step s, entry 0 = 0)."""
    t = _lib.torch()
    dev = _lib.require_device()
    state = t.empty(625, dtype=t.int32, device=dev)
    _lib.call("n3_py_random_seed", _lib.ptr(state), abs(int(seed)) & (2**64 - 1), None)
    out = []
    for count in counts:
        js = t.empty(max(1, int(count)), dtype=t.int32, device=dev)
        _lib.call("n3_py_shuffle_steps", _lib.ptr(state), int(count), _lib.ptr(js), None)
        out.append(js[:int(count)].cpu().numpy())
    return out


class DeviceBeam:
    """Device buffers and descriptor of one beam search."""

    def __init__(self, n: int, *, seed: int, population: int, elite_size: int, max_strength: int,
                 energy_window: int, bad_bias: int, history_len: int):
        t = _lib.torch()
        self.device = dev = _lib.require_device()
        i32 = t.int32
        self.n, self.population, self.elite_size = n, population, elite_size
        z = lambda *shape, dtype=i32: t.zeros(shape, dtype=dtype, device=dev)  # noqa: E731
        self.elite_p, self.elite_q = z(elite_size, n), z(elite_size, n)
        self.elite_badness, self.elite_scores = z(elite_size, 2 * n), z(elite_size)
        self.child_p, self.child_q, self.child_scores = z(population, n), z(population, n), z(population)
        self.pick_p, self.pick_q = z(elite_size, n), z(elite_size, n)
        self.pick_badness, self.pick_scores = z(elite_size, 2 * n), z(elite_size)
        self.selected = z(elite_size)
        self.rng = z(625)
        self.status = z(STATUS_WORDS, dtype=t.int64)
        self.best_p, self.best_q = z(n), z(n)
        self.history = z(max(1, history_len), 2)
        self.child_parent, self.child_nmoves = z(population), z(population)
        self.child_moves = z(population, max_strength)
        self.child_badness = z(population, 2 * n)
        self.error_word = z(1)
        self.desc = BeamDesc(n, population, elite_size, energy_window, max_strength, bad_bias,
                             seed & (2**64 - 1),
                             *[_lib.ptr(x) for x in (self.elite_p, self.elite_q, self.elite_badness,
                                                     self.elite_scores, self.child_p, self.child_q,
                                                     self.child_scores, self.pick_p, self.pick_q, self.pick_badness,
                                                     self.pick_scores, self.selected, self.rng, self.status,
                                                     self.best_p, self.best_q, self.history)],
                             history_len,
                             *[_lib.ptr(x) for x in (self.child_parent, self.child_moves, self.child_nmoves,
                                                     self.child_badness, self.error_word)])

    def init(self, base: np.ndarray, stream=None) -> None:
        t = _lib.torch()
        count = base.shape[0]
        self.elite_p[:count] = t.from_numpy(np.ascontiguousarray(base[:, :, 0], dtype=np.int32)).to(self.device)
        self.elite_q[:count] = t.from_numpy(np.ascontiguousarray(base[:, :, 1], dtype=np.int32)).to(self.device)
        _lib.call("n3_beam_init", ctypes.byref(self.desc), count, _lib.stream_ptr(stream))

    def generation(self, g: int, stream=None) -> None:
        _lib.call("n3_beam_generation", ctypes.byref(self.desc), g, _lib.stream_ptr(stream))

    def read_status(self) -> np.ndarray:
        """The 8 status words; raises AssertionError if a child's maintained
        badness failed its re-check (device error bit 16)."""
        st = self.status.cpu().numpy()
        if int(self.error_word.item()):
            raise AssertionError(f"beam search: device error bits {int(self.error_word.item()):#x}")
        return st


def gpu_device_beam_search(
    initial: PairPermutations,
    *,
    seed: int,
    generations: int,
    population: int,
    elite_size: int,
    max_strength: int,
    energy_window: int,
    initial_elites: np.ndarray | None = None,
    report_every: int = 5,
    bad_bias: int = 85,
    callback: Callable[[GpuSearchSnapshot], None] | None = None,
) -> GpuSearchResult:
    """Generate mutations, score, and retain the beam without population transfers
    (gpu_device_search.py:254-432; validation :269-278)."""
    initial.validate()
    if initial.n > _lib.MAX_N:
        raise ValueError("device badness kernel currently supports n <= 75")
    if not (1 <= elite_size <= population):
        raise ValueError("elite_size must be between one and population")
    if elite_size < 2:
        raise ValueError("the device beam search needs elite_size >= 2")
    if population > 65536:
        raise ValueError("the device beam search supports population <= 65536")
    if max_strength < 1:
        raise ValueError("max_strength must be positive")
    if not 0 <= bad_bias <= 100:
        raise ValueError("bad_bias must be between zero and 100")
    base = np.column_stack((initial.P, initial.Q)).astype(np.int32)[None, :, :]
    if initial_elites is not None:
        supplied = np.ascontiguousarray(initial_elites, dtype=np.int32)
        if supplied.ndim != 3 or supplied.shape[1:] != (initial.n, 2):
            raise ValueError("initial_elites must have shape (count,n,2)")
        for values in supplied:
            _normalize_raw(values[:, 0], values[:, 1]).validate()
        base = np.concatenate((base, supplied), axis=0)
    base = base[:elite_size]
    beam = DeviceBeam(initial.n, seed=seed, population=population, elite_size=elite_size,
                      max_strength=max_strength, energy_window=energy_window, bad_bias=bad_bias,
                      history_len=generations)
    beam.init(base)
    evaluations = len(base)
    started = time.perf_counter()
    completed = 0
    check_every = max(1, report_every)
    for generation in range(1, generations + 1):
        beam.generation(generation)
        if callback is None and generation % check_every and generation != generations:
            continue
        st = beam.read_status()
        completed = int(st[5])
        if callback is not None and (st[7] or generation % max(1, report_every) == 0):
            count = int(st[0])
            ep = beam.elite_p[:count].cpu().numpy()
            eq = beam.elite_q[:count].cpu().numpy()
            scores = beam.elite_scores[:count].cpu().numpy()
            npp, nqq = normalize_rows(ep, eq)
            normalized = [np.column_stack((a, c)) for a, c in zip(npp, nqq)]
            best_state = _normalize_raw(beam.best_p.cpu().numpy(), beam.best_q.cpu().numpy())
            callback(GpuSearchSnapshot(generation, time.perf_counter() - started,
                                       evaluations + population * completed, int(st[6]), int(st[1]),
                                       tuple(map(int, scores)), np.asarray(normalized, dtype=np.int32),
                                       best_state))
        if st[1] == 0:
            break
    st = beam.read_status()
    completed = int(st[5])
    best_score = int(st[1])
    state = _normalize_raw(beam.best_p.cpu().numpy(), beam.best_q.cpu().numpy())
    if best_score == 0:  # gpu_device_search.py:412-418: both independent counts must agree on E = 0
        from .gpu import score_checked_gpu
        from .state import pq_to_columns

        checked = score_checked_gpu(pq_to_columns(np.asarray(state.P, np.int32)[None],
                                                  np.asarray(state.Q, np.int32)[None]), raise_on_mismatch=False)
        if int(checked.scores[0]) != 0 or checked.mismatches:
            raise AssertionError("device GPU E=0 failed verification: determinant and slope counts disagree")
    return GpuSearchResult(state, best_score, completed, evaluations + population * completed,
                           time.perf_counter() - started, seed)
