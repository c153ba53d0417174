"""Generate the walk golden fixture (walk_golden.npz) from the reference itself.

Run once, in a container that has the reference checked out, numba and g++:

    NUMBA_CACHE_DIR=/tmp/n3_numba python tests/golden/make_golden_walk.py /path/to/reference

(or set N3_REFERENCE to the checkout instead of passing it).

What is the reference's own code here:

* the persistent walk kernel: the CUDA C source string ``SOURCE`` of
  tempering.py:19-116 (with the xorshift64* ``next_u64`` of
  gpu_device_search.py:18-25 that it embeds) is read from the imported module
  at run time and compiled for the CPU (g++, into a temporary directory)
  behind a small shim: one thread per block, so every block-strided loop runs
  sequentially, ``__syncthreads`` does nothing and ``atomicAdd`` is a plain
  add.  The kernel's result does not depend on its thread count (its atomics
  only sum integers), so this is the reference's walk, step for step, with its
  own RNG, its badness-biased slot draw, its umbrella restraint and its
  double-precision ``log`` acceptance.  Its source is never copied into this
  repository;
* ``accelerated.score_and_badness`` for the initial scores and badness and
  ``state.random_state`` for the seeded initial states, as
  ``TemperingChains.__init__`` (tempering.py:130-152) sets them up.

Each case runs the walk in chunks of ``steps`` proposals and records every
array the kernel updates after every chunk.  The GPU box never runs this
script; tests read the fixture.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
import tempfile
from pathlib import Path
from random import Random

import numpy as np

HERE = Path(__file__).resolve().parent
if len(sys.argv) > 1:
    REFERENCE = Path(sys.argv[1])
elif os.environ.get("N3_REFERENCE"):
    REFERENCE = Path(os.environ["N3_REFERENCE"])
else:
    raise SystemExit("usage: make_golden_walk.py /path/to/reference  (or set N3_REFERENCE)")
sys.path.insert(0, str(REFERENCE / "src"))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/n3_numba_cache")

from no_three_75 import accelerated, state, tempering  # noqa: E402

SHIM = r"""
#include <math.h>
#define __device__
#define __global__
#define __forceinline__ inline
#define __shared__ static
struct shim_dim3 { unsigned int x; };
static shim_dim3 blockIdx, blockDim, threadIdx;
static inline void __syncthreads() {}
static inline int atomicAdd(int* p, int v) { const int o = *p; *p = o + v; return o; }
"""

DRIVER = r"""
extern "C" void run_walk(int replicas, int* columns, int* badness, int* scores, unsigned long long* rngs,
                         int* best_columns, int* best_scores, const float* temperatures, int* accepted,
                         const int* reference, int* removed_points, const float* centers, const float* strengths,
                         int n, int steps, int bad_bias) {
  blockDim.x = 1;
  threadIdx.x = 0;
  for (int r = 0; r < replicas; ++r) {
    blockIdx.x = r;
    walk(columns, badness, scores, rngs, best_columns, best_scores, temperatures, accepted, reference,
         removed_points, centers, strengths, n, steps, bad_bias);
  }
}
"""


def build_walk(tmp: Path):
    src = tmp / "walk.cpp"
    src.write_text(SHIM + tempering.SOURCE + DRIVER)
    lib = tmp / "walk.so"
    # no -march: plain SSE2 doubles, no fused multiply-adds, as Python's floats
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-o", str(lib), str(src)], check=True)
    dll = ctypes.CDLL(str(lib))
    P = ctypes.c_void_p
    I = ctypes.c_int
    dll.run_walk.argtypes = [I] + [P] * 12 + [I, I, I]
    dll.run_walk.restype = None
    return dll


def initial(n: int, replicas: int, base_seed: int):
    rows = []
    for i in range(replicas):
        s = state.random_state(n, Random(base_seed + i))
        rows.append(np.column_stack((s.P, s.Q)).flatten())
    columns = np.asarray(rows, np.int32)
    scores, badness = [], []
    for row in columns:
        e, b = accelerated.score_and_badness(row[0::2].copy(), row[1::2].copy())
        scores.append(e)
        badness.append(b)
    return columns, np.asarray(scores, np.int32), np.asarray(badness, np.int32)


CASES = {
    # name: n, replicas, base seed, rng seed, bad_bias, strength, chunks, steps per chunk
    "n20_plain": dict(n=20, replicas=4, base=91001, rng=5, bad_bias=0, strength=0.0, chunks=20, steps=25),
    "n20_bias50": dict(n=20, replicas=4, base=91001, rng=6, bad_bias=50, strength=0.0, chunks=20, steps=25),
    "n20_bias85": dict(n=20, replicas=4, base=91101, rng=7, bad_bias=85, strength=0.0, chunks=20, steps=25),
    "n20_bias100": dict(n=20, replicas=4, base=91201, rng=8, bad_bias=100, strength=0.0, chunks=20, steps=25),
    "n20_umbrella": dict(n=20, replicas=4, base=91301, rng=9, bad_bias=0, strength=0.5, chunks=20, steps=25),
    "n20_umbrella_bias85": dict(n=20, replicas=4, base=91401, rng=10, bad_bias=85, strength=0.75, chunks=20,
                                steps=25),
    "n75_bias85_umbrella": dict(n=75, replicas=2, base=91001, rng=11, bad_bias=85, strength=0.2, chunks=6, steps=50),
}


def run_case(dll, cfg) -> dict:
    n, R = cfg["n"], cfg["replicas"]
    columns, scores, badness = initial(n, R, cfg["base"])
    temperatures = np.geomspace(0.3, 3.0, R).astype(np.float32)
    host = np.random.default_rng(cfg["rng"])
    rngs = host.integers(1, 2 ** 64 - 1, size=R, dtype=np.uint64)
    reference = columns[0].copy()
    ref_pts = set((i // 2, int(c)) for i, c in enumerate(reference))
    removed = np.asarray([len(ref_pts - set((i // 2, int(c)) for i, c in enumerate(row))) for row in columns],
                         np.int32)
    centers = np.linspace(0, 3 * R, R).astype(np.float32)
    strengths = np.full(R, cfg["strength"], np.float32)
    best_columns, best_scores = columns.copy(), scores.copy()
    accepted = np.zeros(R, np.int32)
    start = {"columns": columns.copy(), "badness": badness.copy(), "scores": scores.copy(), "rngs": rngs.copy(),
             "removed": removed.copy()}
    hist = {k: [] for k in ("columns", "badness", "scores", "rngs", "best_columns", "best_scores", "accepted",
                            "removed")}
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    for _ in range(cfg["chunks"]):
        dll.run_walk(R, ptr(columns), ptr(badness), ptr(scores), ptr(rngs), ptr(best_columns), ptr(best_scores),
                     ptr(temperatures), ptr(accepted), ptr(reference), ptr(removed), ptr(centers), ptr(strengths),
                     n, cfg["steps"], cfg["bad_bias"])
        for k, v in (("columns", columns), ("badness", badness), ("scores", scores), ("rngs", rngs),
                     ("best_columns", best_columns), ("best_scores", best_scores), ("accepted", accepted),
                     ("removed", removed)):
            hist[k].append(v.copy())
    # every recorded energy is the full recount of its state (the reference's validate, tempering.py:193-201)
    for row, e, b in zip(columns, scores, badness):
        fe, fb = accelerated.score_and_badness(row[0::2].copy(), row[1::2].copy())
        assert fe == e and np.array_equal(fb, b)
    out = {f"start_{k}": v for k, v in start.items()}
    out.update({f"hist_{k}": np.stack(v) for k, v in hist.items()})
    out.update(temperatures=temperatures, reference=reference, centers=centers, strengths=strengths,
               n=np.asarray(n), steps=np.asarray(cfg["steps"]), bad_bias=np.asarray(cfg["bad_bias"]))
    return out


def main():
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        dll = build_walk(Path(tmp))
        for name, cfg in CASES.items():
            res = run_case(dll, cfg)
            acc = int(res["hist_accepted"][-1].sum())
            print(f"{name}: accepted {acc}, scores {res['start_scores'].tolist()} -> "
                  f"{res['hist_scores'][-1].tolist()}, removed -> {res['hist_removed'][-1].tolist()}")
            out.update({f"{name}/{k}": v for k, v in res.items()})
    np.savez_compressed(HERE / "walk_golden.npz", **out)


if __name__ == "__main__":
    main()
