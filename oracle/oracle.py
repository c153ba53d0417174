"""ctypes front end of the C oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline / reference arm, never by the product package.  Every
function restates a reference function (file:line given on each) and is
pinned against the reference's own outputs by tests/test_oracle_golden.py.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
SENTINEL64 = 1 << 60

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_lib = None


def build() -> Path:
    """Compile liboracle.so with the Makefile next to this file."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.n3o_score_and_badness.restype = ctypes.c_int64
        L.n3o_score_and_badness.argtypes = [_i32p, _i32p, ctypes.c_int, _i64p]
        for name in ("n3o_score_population", "n3o_slope_population"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [_i32p, _i32p, ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_void_p, ctypes.c_int]
        for name in ("n3o_slope_score_points", "n3o_det_score_points"):
            f = getattr(L, name)
            f.restype = ctypes.c_int64
            f.argtypes = [_i32p, _i32p, ctypes.c_int, _i64p]
        L.n3o_two_switches.restype = None
        L.n3o_two_switches.argtypes = [_i32p, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int64, _i64p, _i64p]
        L.n3o_transpositions.restype = None
        L.n3o_transpositions.argtypes = [_i32p, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                         _i64p, _i64p]
        L.n3o_walk_delta.restype = ctypes.c_int
        L.n3o_walk_delta.argtypes = [_i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32),
                                     ctypes.c_void_p]
        L.n3o_score_columns.restype = ctypes.c_int32
        L.n3o_score_columns.argtypes = [_i32p, ctypes.c_int, ctypes.c_void_p]
        L.n3o_max_threads.restype = ctypes.c_int
        L.n3o_three_cycles.restype = None
        L.n3o_three_cycles.argtypes = [_i32p, _i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int64, _i64p, _i64p]
        L.n3o_beam_mutate.restype = None
        L.n3o_beam_mutate.argtypes = [_i32p, _i32p, _i32p] + [ctypes.c_int] * 7 + [ctypes.c_uint64, ctypes.c_int,
                                                                                    _i32p, _i32p]
        _lib = L
    return _lib


def _c32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def max_threads() -> int:
    return int(lib().n3o_max_threads())


def score_and_badness(p, q) -> tuple[int, np.ndarray]:
    """accelerated.py:14-37."""
    p, q = _c32(p), _c32(q)
    bad = np.zeros(2 * len(p), np.int64)
    s = lib().n3o_score_and_badness(p, q, len(p), bad)
    return int(s), bad


def score_population(p, q, *, badness: bool = False, threads: int = 1):
    """Batched accelerated.py:14-37 over P/Q [B, n] (gpu.py:108's CPU loop)."""
    p, q = _c32(p), _c32(q)
    B, n = p.shape
    scores = np.zeros(B, np.int32)
    bad = np.zeros((B, 2 * n), np.int32) if badness else None
    lib().n3o_score_population(p, q, B, n, scores, bad.ctypes.data if bad is not None else None, threads)
    return (scores, bad) if badness else scores


def slope_population(p, q, *, threads: int = 1):
    """Normalised-direction line count (verifier_b.py:8-33 counted, conflicts.py:36-72 sums)."""
    p, q = _c32(p), _c32(q)
    B, n = p.shape
    scores = np.zeros(B, np.int32)
    bad = np.zeros((B, 2 * n), np.int32)
    lib().n3o_slope_population(p, q, B, n, scores, bad.ctypes.data, threads)
    return scores, bad


def slope_score_points(points) -> tuple[int, np.ndarray]:
    pts = np.asarray(points, dtype=np.int32).reshape(-1, 2)
    rows, cols = _c32(pts[:, 0]), _c32(pts[:, 1])
    bad = np.zeros(len(pts), np.int64)
    return int(lib().n3o_slope_score_points(rows, cols, len(pts), bad)), bad


def det_score_points(points) -> tuple[int, np.ndarray]:
    """verifier_a.py:8-16 counted over all triples."""
    pts = np.asarray(points, dtype=np.int32).reshape(-1, 2)
    rows, cols = _c32(pts[:, 0]), _c32(pts[:, 1])
    bad = np.zeros(len(pts), np.int64)
    return int(lib().n3o_det_score_points(rows, cols, len(pts), bad)), bad


def two_switches(p, q, u: int, score: int, badness) -> np.ndarray:
    """accelerated.py:122-195 (sentinel 1<<60)."""
    p, q = _c32(p), _c32(q)
    out = np.zeros(2 * len(p), np.int64)
    lib().n3o_two_switches(p, q, len(p), int(u), int(score), np.ascontiguousarray(badness, np.int64), out)
    return out


def transpositions(p, q, layer: int, row: int, score: int, badness) -> np.ndarray:
    """accelerated.py:40-119 (sentinel 1<<60)."""
    p, q = _c32(p), _c32(q)
    out = np.zeros(len(p), np.int64)
    lib().n3o_transpositions(p, q, len(p), int(layer), int(row), int(score),
                             np.ascontiguousarray(badness, np.int64), out)
    return out


def walk_delta(cols, u: int, v: int):
    """tempering.py:58,68-89: (legal, dE, dbad[2n])."""
    c = _c32(cols)
    dE = ctypes.c_int32(0)
    dbad = np.zeros(len(c), np.int32)
    ok = lib().n3o_walk_delta(c, len(c) // 2, int(u), int(v), ctypes.byref(dE), dbad.ctypes.data)
    return bool(ok), int(dE.value), dbad


_MASK64 = (1 << 64) - 1


def next_u64(state: int) -> tuple[int, int]:
    """xorshift64* (Vigna) as the reference's next_u64 (gpu_device_search.py:18-25):
    returns (new state, output)."""
    x = state
    x ^= x >> 12
    x ^= (x << 25) & _MASK64
    x ^= x >> 27
    return x, (x * 2685821657736338717) & _MASK64


def bias_slot(badness, m: int, target: int) -> int:
    """The reference's badness-weighted slot (tempering.py:52-54)."""
    u = 0
    while u < m - 1 and target >= int(badness[u]):
        target -= int(badness[u])
        u += 1
    return u


def distance_delta(reference, u: int, v: int, cu: int, cv: int) -> int:
    """Change of the distance to the reference state (tempering.py:59-63)."""
    ur, vr = (u >> 1) * 2, (v >> 1) * 2
    return (int(cu in (reference[ur], reference[ur + 1])) + int(cv in (reference[vr], reference[vr + 1]))
            - int(cv in (reference[ur], reference[ur + 1])) - int(cu in (reference[vr], reference[vr + 1])))


def walk_with_reference_rng(cols, bad, score: int, rng: int, best_cols, best_score: int, temperature: float,
                            accepted: int, reference, removed: int, center: float, strength: float, steps: int,
                            bad_bias: int) -> dict:
    """One replica of the reference's walk kernel (tempering.py:29-115) with
    its own xorshift64* draws and double-precision acceptance, restated from
    this oracle's pieces: ``bias_slot``, ``distance_delta`` and the pair-form
    delta ``walk_delta``.  Used to pin those pieces against the reference's
    kernel; the device engine draws with Philox instead (``temper_run``)."""
    import math

    cols = np.array(cols, np.int32)
    bad = np.array(bad, np.int32)
    best_cols = np.array(best_cols, np.int32)
    m = len(cols)
    T = float(np.float32(temperature))
    c32, s32 = float(np.float32(center)), float(np.float32(strength))
    for _ in range(steps):
        rng, x = next_u64(rng)
        u = x % m
        if bad_bias > 0 and score > 0:
            rng, x = next_u64(rng)
            if x % 100 < bad_bias:
                rng, x = next_u64(rng)
                u = bias_slot(bad, m, x % (3 * score))
        rng, x = next_u64(rng)
        v = x % m
        cu, cv = int(cols[u]), int(cols[v])
        valid = score > 0 and (u >> 1) != (v >> 1) and cu != cv and cols[u ^ 1] != cv and cols[v ^ 1] != cu
        if not valid:
            continue
        dd = distance_delta(reference, u, v, cu, cv)
        _, delta, dbad = walk_delta(cols, u, v)
        rng, x = next_u64(rng)
        uniform = ((x >> 11) + 0.5) / 9007199254740992.0
        offset = removed - c32
        energy = delta + s32 * (2 * offset * dd + dd * dd)
        if energy <= 0 or math.log(uniform) < -energy / T:
            cols[u], cols[v] = cv, cu
            bad += dbad
            score += delta
            removed += dd
            accepted += 1
            if score < best_score:
                best_score = score
                best_cols = cols.copy()
    return {"columns": cols, "badness": bad, "scores": score, "rngs": rng, "best_columns": best_cols,
            "best_scores": best_score, "accepted": accepted, "removed": removed}


def score_columns(cols) -> tuple[int, np.ndarray]:
    c = _c32(cols)
    bad = np.zeros(len(c), np.int32)
    return int(lib().n3o_score_columns(c, len(c) // 2, bad.ctypes.data)), bad


def philox4x32_10(ctr, key0: int, key1: int) -> list[int]:
    """Philox4x32-10 (Salmon et al., SC'11) restated in oracle.c."""
    L = lib()
    f = L.n3o_philox4x32_10
    f.restype = None
    f.argtypes = [np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS"), ctypes.c_uint32, ctypes.c_uint32,
                  np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")]
    out = np.zeros(4, np.uint32)
    f(np.ascontiguousarray(ctr, dtype=np.uint32), key0 & 0xFFFFFFFF, key1 & 0xFFFFFFFF, out)
    return [int(x) for x in out]


def temper_run(state: dict, *, ladder_size: int, acc, exch, seed: int, rounds: int = 0, round_sweeps: int = 0,
               round_proposals: int = 0, exchange: bool = True, ladder_rounds=None, threads: int = 0,
               bad_bias: int = 0, reference=None, umbrella=None, frac=None) -> dict:
    """CPU replay of the device tempering kernel (see n3o_temper_run in oracle.c).

    ``state`` holds numpy arrays in the layout of the device chains (columns
    [C, stride]); a replayed copy is returned.  With ``umbrella`` ([C, 2] int64
    per replica position) the state also needs ``removed`` [C]; ``reference``
    is the reference state's slot columns and ``frac`` the [L, 768] factors."""
    L = lib()
    f = L.n3o_temper_run
    f.restype = None
    P = ctypes.c_void_p
    f.argtypes = ([ctypes.c_int, ctypes.c_int, ctypes.c_int] + [P] * 13 + [ctypes.c_int, P, ctypes.c_int,
                                                                          ctypes.c_uint64] + [ctypes.c_int] * 4 +
                  [P, ctypes.c_int, ctypes.c_int, P, P, P, P])
    s = {k: np.array(v, copy=True) for k, v in state.items()}
    conv = {"cols": np.int32, "bad": np.int32, "E": np.int32, "bestE": np.int32, "best_cols": np.int32,
            "temp_of": np.int32, "chain_at": np.int32, "counter": np.uint64, "accepted": np.uint32,
            "ladder_n": np.int32, "ladder_round": np.uint32, "ladder_exch": np.uint32}
    for k, dt in conv.items():
        s[k] = np.ascontiguousarray(s[k], dtype=dt)
    acc = np.ascontiguousarray(acc, dtype=np.uint32)
    exch = np.ascontiguousarray(exch, dtype=np.uint32)
    lr = None if ladder_rounds is None else np.ascontiguousarray(ladder_rounds, dtype=np.int32)
    C, stride = s["cols"].shape
    ref = umb = fr = None
    if umbrella is not None:
        s["removed"] = np.ascontiguousarray(s["removed"], dtype=np.int32)
        ref = np.ascontiguousarray(reference, dtype=np.int32)
        umb = np.ascontiguousarray(umbrella, dtype=np.int64)
        fr = np.ascontiguousarray(frac, dtype=np.uint32)
    f(C, ladder_size, stride, *(s[k].ctypes.data for k in ["cols", "bad", "E", "bestE", "best_cols", "temp_of",
                                                            "chain_at", "counter", "accepted", "ladder_n",
                                                            "ladder_round", "ladder_exch"]),
      acc.ctypes.data, acc.shape[1], exch.ctypes.data, exch.shape[1], seed & 0xFFFFFFFFFFFFFFFF, rounds,
      round_sweeps, round_proposals, int(exchange), lr.ctypes.data if lr is not None else None, threads,
      int(bad_bias), None if ref is None else ref.ctypes.data,
      None if umb is None else s["removed"].ctypes.data, None if umb is None else umb.ctypes.data,
      None if fr is None else fr.ctypes.data)
    return s


# --------------------------------------------------------------------------
# Device beam search (gpu_device_search.py:185-432), restated on the CPU.
# --------------------------------------------------------------------------
def beam_mutate(parent_p, parent_q, parent_badness, *, quality_count: int, population: int, active_strength: int,
                max_strength: int, bad_bias: int, seed: int, generation: int):
    """The CUDA kernel ``mutate_population`` (gpu_device_search.py:17-114)."""
    pp, pq, pb = _c32(parent_p), _c32(parent_q), _c32(parent_badness)
    n = pp.shape[1]
    cp_ = np.empty((population, n), np.int32)
    cq_ = np.empty((population, n), np.int32)
    lib().n3o_beam_mutate(pp, pq, pb, pp.shape[0], quality_count, n, population, active_strength, max_strength,
                          bad_bias, seed & ((1 << 64) - 1), generation, cp_, cq_)
    return cp_, cq_


def elite_key(score: int, badness) -> tuple[int, int, int]:
    """gpu_device_search.py:200-203."""
    v = np.asarray(badness, dtype=np.int64)
    return int(score), int(v.max()), int(np.dot(v, v))


def rank_elites(scores, badness) -> np.ndarray:
    """gpu_device_search.py:185-197: stable sort by (score, max badness, sum of squares)."""
    return np.asarray(sorted(range(len(scores)), key=lambda i: elite_key(scores[i], badness[i])), dtype=np.int32)


def beam_search(initial_p, initial_q, extra=None, *, seed: int, generations: int, population: int, elite_size: int,
                max_strength: int, energy_window: int, bad_bias: int = 85, threads: int = 0) -> dict:
    """The generation loop of gpu_device_beam_search (gpu_device_search.py:254-432):
    mutate, score, keep the best quarter plus a seeded random.Random shuffle of the
    children within ``energy_window`` of the best, rank by elite_key."""
    from random import Random

    rng = Random(seed)
    base = np.column_stack((initial_p, initial_q)).astype(np.int32)[None]
    if extra is not None:
        base = np.concatenate((base, np.asarray(extra, np.int32)), axis=0)
    base = base[:elite_size]
    ep, eq = base[:, :, 0].copy(), base[:, :, 1].copy()
    es, eb = score_population(ep, eq, badness=True, threads=threads)
    order = rank_elites(es, eb)
    ep, eq, eb, es = ep[order], eq[order], eb[order], es[order]
    best_score = int(es[0])
    best_key = elite_key(best_score, eb[0])
    best_p, best_q = ep[0].copy(), eq[0].copy()
    last_improvement, completed = 0, 0
    out = {"generation_best": [], "best_history": [], "elite_scores": [], "elite_p": [], "elite_q": []}
    for generation in range(1, generations + 1):
        completed = generation
        active = min(max_strength, 2 + (generation - last_improvement) // 10)
        qc = max(1, min(len(es), elite_size // 4))
        cp_, cq_ = beam_mutate(ep, eq, eb, quality_count=qc, population=population, active_strength=active,
                               max_strength=max_strength, bad_bias=bad_bias, seed=seed, generation=generation)
        scores = score_population(cp_, cq_, threads=threads)
        order = np.argsort(scores, kind="stable")
        selected = list(map(int, order[:max(1, elite_size // 4)]))
        chosen = set(selected)
        diverse = list(map(int, np.flatnonzero(scores <= best_score + energy_window)))
        rng.shuffle(diverse)
        for index in diverse:
            if index not in chosen:
                selected.append(index)
                chosen.add(index)
                if len(selected) == elite_size:
                    break
        if len(selected) < elite_size:
            for index in map(int, order):
                if index not in chosen:
                    selected.append(index)
                    chosen.add(index)
                    if len(selected) == elite_size:
                        break
        sel = np.asarray(selected, np.int64)
        ep, eq, es = cp_[sel], cq_[sel], scores[sel]
        _, eb = score_population(ep, eq, badness=True, threads=threads)
        rank = rank_elites(es, eb)
        ep, eq, eb, es = ep[rank], eq[rank], eb[rank], es[rank]
        key = elite_key(int(es[0]), eb[0])
        if key < best_key:
            best_score, best_key = int(es[0]), key
            best_p, best_q = ep[0].copy(), eq[0].copy()
            last_improvement = generation
        out["generation_best"].append(int(es[0]))
        out["best_history"].append(best_score)
        out["elite_scores"].append(es.copy())
        out["elite_p"].append(ep.copy())
        out["elite_q"].append(eq.copy())
        if best_score == 0:
            break
    out.update(completed=completed, best_score=best_score, best_p_raw=best_p, best_q_raw=best_q,
               evaluations=len(base) + completed * population)
    return out


# --------------------------------------------------------------------------
# Multi-point moves.
# --------------------------------------------------------------------------
def three_cycles(p, q, candidates, score: int, badness) -> np.ndarray:
    """accelerated.py:196-276 (candidates int32 [M, 4]: u, v, w, orientation)."""
    p, q = _c32(p), _c32(q)
    cand = _c32(np.asarray(candidates).reshape(-1, 4))
    out = np.zeros(cand.shape[0], np.int64)
    lib().n3o_three_cycles(p, q, len(p), cand, cand.shape[0], int(score),
                           np.ascontiguousarray(badness, dtype=np.int64), out)
    return out


def legal_three_cycle_candidates(p, q, selected: int) -> np.ndarray:
    """search.py:38-65: (selected, v, w, orientation) for v < w in other, distinct
    rows with three distinct columns and no row left with a repeated column."""
    n = len(p)
    cols = np.empty(2 * n, np.int64)
    cols[0::2], cols[1::2] = p, q
    srow = selected // 2
    out = []
    for v in range(2 * n - 1):
        if v // 2 == srow:
            continue
        for w in range(v + 1, 2 * n):
            if w // 2 in (srow, v // 2):
                continue
            if len({int(cols[selected]), int(cols[v]), int(cols[w])}) != 3:
                continue
            ou, ov, ow = selected ^ 1, v ^ 1, w ^ 1
            if cols[v] != cols[ou] and cols[w] != cols[ov] and cols[selected] != cols[ow]:
                out.append((selected, v, w, 0))
            if cols[w] != cols[ou] and cols[v] != cols[ow] and cols[selected] != cols[ov]:
                out.append((selected, v, w, 1))
    return np.asarray(out, np.int32).reshape(-1, 4)


def neighborhood_scan(p, q, anchor: int, *, kind: str, threads: int = 0):
    """gpu_neighborhood.py:70-211 restated: every four-cycle (kind "four") or
    double switch (kind "double") through ``anchor``, enumerated in the
    reference's order (row triples, layer choices, orderings), each scored in
    full; returns (best score, evaluated, legal, best P, best Q) with the first
    strictly improving minimum, the base state when nothing improves."""
    from itertools import combinations, permutations, product

    p, q = _c32(p), _c32(q)
    n = len(p)
    base = np.column_stack((p, q)).astype(np.int32)
    flat = base.reshape(-1)
    best = int(score_and_badness(p, q)[0])
    best_values = base.copy()
    targets, sources = [], []
    others = [r for r in range(n) if r != anchor // 2]
    for rows in combinations(others, 3):
        for layers in product((0, 1), repeat=3):
            slots = tuple(2 * r + l for r, l in zip(rows, layers))
            if kind == "four":
                for order in permutations(slots):
                    t = (anchor,) + order
                    targets.append(t)
                    sources.append(t[1:] + t[:1])
            else:
                a, b, c = slots
                for src in ((a, anchor, c, b), (b, c, anchor, a), (c, b, a, anchor)):
                    targets.append((anchor, a, b, c))
                    sources.append(src)
    targets = np.asarray(targets, np.int64)
    sources = np.asarray(sources, np.int64)
    new_cols = flat[sources]
    legal = np.all(new_cols != flat[targets ^ 1], axis=1)
    lt, lc = targets[legal], new_cols[legal]
    cand = np.broadcast_to(flat, (len(lt), flat.size)).copy()
    cand[np.arange(len(lt))[:, None], lt] = lc
    scores = score_population(np.ascontiguousarray(cand[:, 0::2]), np.ascontiguousarray(cand[:, 1::2]),
                              threads=threads) if len(lt) else np.empty(0, np.int32)
    if len(scores) and int(scores.min()) < best:
        i = int(np.argmin(scores))
        best = int(scores[i])
        best_values = cand[i].reshape(n, 2)
    return best, int(len(targets)), int(legal.sum()), best_values[:, 0].copy(), best_values[:, 1].copy()


# --------------------------------------------------------------------------
# Line weights of breakout search (breakout.py:39-86), restated with NumPy.
# --------------------------------------------------------------------------
def _c3(k):
    k = np.asarray(k, np.int64)
    return np.where(k >= 3, k * (k - 1) * (k - 2) // 6, 0)


def weighted_switch_scores(p, q, u: int, raw, keys, vals) -> np.ndarray:
    """breakout.py:39-75 with weights as parallel arrays (keys [L, 3], vals [L])."""
    p, q = np.asarray(p, np.int64), np.asarray(q, np.int64)
    n = len(p)
    rows = np.repeat(np.arange(n, dtype=np.int64), 2)
    cols = np.empty(2 * n, np.int64)
    cols[0::2], cols[1::2] = p, q
    out = np.asarray(raw, np.int64).copy()
    keys = np.asarray(keys, np.int64).reshape(-1, 3)
    vals = np.asarray(vals, np.int64)
    for (a, b, c), w in zip(keys, vals):
        if w <= 1:
            continue
        member = a * rows + b * cols + c == 0
        occ = int(member.sum())
        new_u = a * rows[u] + b * cols + c == 0          # u to (row u, column v)
        new_v = a * rows + b * cols[u] + c == 0          # v to (row v, column u)
        k = occ - int(member[u]) - member.astype(np.int64) + new_u + new_v
        out += (w - 1) * _c3(k)
    return out


def weighted_state_score(p, q, raw_score: int, keys, vals) -> int:
    """breakout.py:78-86."""
    p, q = np.asarray(p, np.int64), np.asarray(q, np.int64)
    n = len(p)
    rows = np.concatenate([np.arange(n), np.arange(n)])
    cols = np.concatenate([p, q])
    value = int(raw_score)
    for (a, b, c), w in zip(np.asarray(keys, np.int64).reshape(-1, 3), np.asarray(vals, np.int64)):
        if w <= 1:
            continue
        value += int((w - 1) * _c3(int(np.count_nonzero(a * rows + b * cols + c == 0))))
    return value


# --------------------------------------------------------------------------
# Line tables (precompute.py:18-94).  Pure NumPy restatements.
# --------------------------------------------------------------------------
def triangular_pair_index(left: int, right: int, point_count: int) -> int:
    """precompute.py:28-33: index of the unordered pair {left, right} in the
    row-major upper triangle of point_count x point_count."""
    if left > right:
        left, right = right, left
    if left == right or left < 0 or right >= point_count:
        raise ValueError("pair index requires two distinct in-range points")
    return left * (2 * point_count - left - 1) // 2 + right - left - 1


def geometry_tables(n: int) -> dict:
    """build_geometry_tables (precompute.py:35-57) over the lines that
    _multi_point_lines (cp_sat.py:129-157) finds on the whole grid: every line
    with three or more grid points that is neither a row nor a column (pairs in
    one row or column are skipped there).  A line enters the reference's dict at
    its second pair, (first member, third member) in the row-major pair loop, so
    the line ids follow (first member, third member).  For one first member the
    third is (r0 + 2a, c0 + 2b) for the line's primitive step (a >= 1, b != 0),
    so the order is that of (a, b).  Members are listed in row-major order."""
    from math import gcd

    N = n * n
    rr, cc = np.divmod(np.arange(N), n)
    recs = []  # (first member, a, b, length)
    for a in range(1, n):
        for b in range(-(n - 1), n):
            if b == 0 or gcd(a, abs(b)) != 1:
                continue
            start = ~((rr - a >= 0) & (cc - b >= 0) & (cc - b < n))  # no grid point before
            third = (rr + 2 * a < n) & (cc + 2 * b >= 0) & (cc + 2 * b < n)
            sel = np.nonzero(start & third)[0]
            if len(sel) == 0:
                continue
            steps_r = (n - 1 - rr[sel]) // a
            steps_c = (n - 1 - cc[sel]) // b if b > 0 else cc[sel] // (-b)
            length = 1 + np.minimum(steps_r, steps_c)
            recs.append(np.stack([sel, np.full_like(sel, a), np.full_like(sel, b), length], 1))
    if recs:
        lines = np.concatenate(recs)
        lines = lines[np.lexsort((lines[:, 2], lines[:, 1], lines[:, 0]))]
    else:
        lines = np.zeros((0, 4), np.int64)
    lengths = lines[:, 3]
    offsets = np.zeros(len(lines) + 1, np.int64)
    np.cumsum(lengths, out=offsets[1:])
    indices = np.empty(int(offsets[-1]), np.int32)
    pair_to_line = np.full(N * (N - 1) // 2, -1, np.int32)
    for k in np.unique(lengths):
        ids = np.nonzero(lengths == k)[0]
        t = np.arange(k)
        r = rr[lines[ids, 0]][:, None] + lines[ids, 1][:, None] * t
        c = cc[lines[ids, 0]][:, None] + lines[ids, 2][:, None] * t
        members = r * n + c  # increasing along the line (a >= 1)
        indices[(offsets[ids][:, None] + t).ravel()] = members.ravel()
        i, j = np.triu_indices(k, 1)
        left, right = members[:, i], members[:, j]
        tri = left * (2 * N - left - 1) // 2 + right - left - 1
        pair_to_line[tri.ravel()] = np.repeat(ids, len(i)).astype(np.int32)
    return {"n": n, "pair_to_line": pair_to_line, "offsets": offsets, "indices": indices, "line_count": len(lines)}


def score_pair_table(points, tables: dict) -> int:
    """precompute.py:60-81: sum of C(k, 3) over the table's lines from the
    pair counts of the points' pairs."""
    from itertools import combinations
    from math import comb, isqrt

    n = tables["n"]
    ids = sorted(row * n + column for row, column in points)
    N = n * n
    pairs = np.fromiter((triangular_pair_index(a, b, N) for a, b in combinations(ids, 2)), dtype=np.int64)
    line_ids = tables["pair_to_line"][pairs]
    line_ids = line_ids[line_ids >= 0]
    score = 0
    for count in np.unique(line_ids, return_counts=True)[1]:
        d = 1 + 8 * int(count)
        root = isqrt(d)
        if root * root != d:
            raise AssertionError("selected pair count is not triangular")
        k = (1 + root) // 2
        score += comb(k, 3) if k >= 3 else 0
    return score


def score_csr(points, tables: dict) -> int:
    """precompute.py:84-89: occupancy summed over each line's members."""
    n = tables["n"]
    occupied = np.zeros(n * n, dtype=np.int8)
    occupied[[row * n + column for row, column in points]] = 1
    if tables["line_count"] == 0:
        return 0
    counts = np.add.reduceat(occupied[tables["indices"]], tables["offsets"][:-1]).astype(np.int64)
    counts = counts[counts >= 3]
    return int(np.sum(counts * (counts - 1) * (counts - 2) // 6))


# --------------------------------------------------------------------------
# Conflict analysis (conflicts.py:36-72 over geometry.py:14-40), restated.
# --------------------------------------------------------------------------
def canonical_line(a, b) -> tuple[int, int, int]:
    """geometry.py:14-28: primitive (A, B, C) with A*row + B*col + C = 0."""
    from math import gcd

    if tuple(a) == tuple(b):
        raise ValueError("two distinct points are required")
    A, B = int(b[1]) - int(a[1]), int(a[0]) - int(b[0])
    C = -(A * int(a[0]) + B * int(a[1]))
    g = gcd(gcd(abs(A), abs(B)), abs(C))
    A, B, C = A // g, B // g, C // g
    if A < 0 or (A == 0 and B < 0):
        A, B, C = -A, -B, -C
    return A, B, C


def primitive_slope(key) -> tuple[int, int]:
    """geometry.py:31-40."""
    from math import gcd

    dx, dy = int(key[1]), -int(key[0])
    g = gcd(abs(dx), abs(dy))
    dx, dy = dx // g, dy // g
    if dx < 0 or (dx == 0 and dy < 0):
        dx, dy = -dx, -dy
    return dx, dy


def analyze_points(points, line_weights=None) -> dict:
    """conflicts.py:36-72: lines of three or more points (key, sorted points,
    C(k,3)) sorted by (-triples, key), per-point badness, slope histogram and
    the summary counts, as plain Python values."""
    from itertools import combinations
    from math import comb

    pts = [(int(r), int(c)) for r, c in points]
    members: dict = {}
    for i, j in combinations(range(len(pts)), 2):
        s = members.setdefault(canonical_line(pts[i], pts[j]), set())
        s.add(i)
        s.add(j)
    badness = [0] * len(pts)
    lines, hist = [], {}
    triples = weighted = 0
    for key, idx in members.items():
        k = len(idx)
        if k < 3:
            continue
        t = comb(k, 3)
        triples += t
        weighted += (line_weights.get(key, 1) if line_weights else 1) * t
        for i in idx:
            badness[i] += comb(k - 1, 2)
        lines.append((key, tuple(sorted(pts[i] for i in idx)), t))
        s = primitive_slope(key)
        hist[s] = hist.get(s, 0) + t
    lines.sort(key=lambda x: (-x[2], x[0]))
    return {"triples": triples, "violating_lines": len(lines),
            "max_line_occupancy": max((len(x[1]) for x in lines), default=2),
            "max_point_badness": max(badness, default=0), "weighted_score": weighted, "badness": badness,
            "lines": lines, "slope_histogram": hist}
