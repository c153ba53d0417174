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
               round_proposals: int = 0, exchange: bool = True, ladder_rounds=None, threads: int = 0) -> dict:
    """CPU replay of the device tempering kernel (see n3o_temper_run in oracle.c).

    ``state`` holds numpy arrays in the layout of the device chains (columns
    [C, stride]); a replayed copy is returned."""
    L = lib()
    f = L.n3o_temper_run
    f.restype = None
    P = ctypes.c_void_p
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + [P] * 13 + [ctypes.c_int, P, ctypes.c_int,
                                                                         ctypes.c_uint64] + [ctypes.c_int] * 4 + [P, ctypes.c_int]
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
    f(C, ladder_size, stride, *(s[k].ctypes.data for k in ["cols", "bad", "E", "bestE", "best_cols", "temp_of",
                                                            "chain_at", "counter", "accepted", "ladder_n",
                                                            "ladder_round", "ladder_exch"]),
      acc.ctypes.data, acc.shape[1], exch.ctypes.data, exch.shape[1], seed & 0xFFFFFFFFFFFFFFFF, rounds,
      round_sweeps, round_proposals, int(exchange), lr.ctypes.data if lr is not None else None, threads)
    return s
