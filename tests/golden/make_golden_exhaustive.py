"""Generate the exhaustive-beam golden fixture (exhaustive_golden.npz) from the
reference itself.

Run once, in a container that has the reference checked out, numba and g++:

    NUMBA_CACHE_DIR=/tmp/n3_numba python tests/golden/make_golden_exhaustive.py /path/to/reference

(or set N3_REFERENCE to the checkout instead of passing it).

The reference's own ``gpu_exhaustive_beam_search`` (gpu_exhaustive_beam.py:91-325)
runs unmodified, with its CuPy module and kernels swapped for CPU stand-ins:

* ``cp`` is NumPy (the function uses asarray, asnumpy, empty, empty_like and
  fancy indexing, which NumPy provides with the same meaning);
* its enumeration kernel is the reference's own CUDA C source
  ``ENUMERATE_SOURCE`` (gpu_exhaustive_beam.py:17-58), read from the imported
  module and compiled for the CPU by g++ behind a small shim that loops over
  the grid (into a temporary directory; the source is never copied here);
* its score and score-with-badness kernels count the same collinear triples
  with ``accelerated.score_and_badness`` (accelerated.py:14-37), the
  reference's CPU count; at n = 75 the batch of children is counted by the
  repository's C restatement of that function on all host threads (pinned to
  the reference by tests/test_oracle_golden.py), for time.

Every generation's snapshot (best scores, elite scores and normalised elites)
is recorded through the function's callback.  The GPU box never runs this
script; tests read the fixture.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
import tempfile
import types
from pathlib import Path
from random import Random

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
if len(sys.argv) > 1:
    REFERENCE = Path(sys.argv[1])
elif os.environ.get("N3_REFERENCE"):
    REFERENCE = Path(os.environ["N3_REFERENCE"])
else:
    raise SystemExit("usage: make_golden_exhaustive.py /path/to/reference  (or set N3_REFERENCE)")
sys.path.insert(0, str(REFERENCE / "src"))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/n3_numba_cache")

from no_three_75 import accelerated, gpu_exhaustive_beam, state  # noqa: E402

SHIM = r"""
#define __device__
#define __global__
#define __forceinline__ inline
struct shim_dim3 { unsigned int x; };
static shim_dim3 blockIdx, blockDim, threadIdx;
"""

DRIVER = r"""
extern "C" void run_enumerate(const int* parent_p, const int* parent_q, const int* descriptors, int candidate_count,
                              int n, int* child_p, int* child_q, unsigned char* valid) {
  blockDim.x = 256;
  for (int c = 0; c < candidate_count; ++c) {
    blockIdx.x = c / 256;
    threadIdx.x = c % 256;
    enumerate_switches(parent_p, parent_q, descriptors, candidate_count, n, child_p, child_q, valid);
  }
}
"""


def build_enumerate(tmp: Path):
    src = tmp / "enumerate.cpp"
    src.write_text(SHIM + gpu_exhaustive_beam.ENUMERATE_SOURCE.replace('extern "C" __global__', 'extern "C"')
                   + DRIVER)
    lib = tmp / "enumerate.so"
    subprocess.run(["g++", "-O2", "-shared", "-fPIC", "-o", str(lib), str(src)], check=True)
    dll = ctypes.CDLL(str(lib))
    P = ctypes.c_void_p
    dll.run_enumerate.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, P, P, P]
    dll.run_enumerate.restype = None
    return dll


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Kernel:
    """A callable with CuPy RawKernel's call form: kernel(grid, block, args)."""

    def __init__(self, fn):
        self.fn = fn

    def __call__(self, grid, block, args):
        self.fn(*args)


def count_batch(p, q, badness=None):
    """Scores (and badness) of a batch of P/Q rows."""
    p = np.ascontiguousarray(p, np.int32)
    q = np.ascontiguousarray(q, np.int32)
    if len(p) > 2000:  # the C restatement on every host thread
        sys.path.insert(0, str(ROOT))
        from oracle import oracle

        if badness is None:
            return oracle.score_population(p, q, threads=0), None
        return oracle.score_population(p, q, badness=True, threads=0)
    scores = np.empty(len(p), np.int32)
    bad = np.empty((len(p), 2 * p.shape[1]), np.int32)
    for i in range(len(p)):
        e, b = accelerated.score_and_badness(p[i].copy(), q[i].copy())
        scores[i], bad[i] = e, b
    return scores, bad


def make_kernels(dll):
    def score_badness(p, q, n, scores_out, badness_out):
        s, b = count_batch(p, q, badness=True)
        scores_out[...] = s
        badness_out[...] = b

    def score(p, q, n, scores_out):
        scores_out[...] = count_batch(p, q)[0]

    def enumerate_(parent_p, parent_q, descriptors, candidate_count, n, child_p, child_q, valid):
        for a in (parent_p, parent_q, descriptors, child_p, child_q, valid):
            assert a.flags["C_CONTIGUOUS"]
        dll.run_enumerate(ptr(parent_p), ptr(parent_q), ptr(descriptors), int(candidate_count), int(n),
                          ptr(child_p), ptr(child_q), ptr(valid))

    cp = types.SimpleNamespace(asarray=lambda x, dtype=None: np.ascontiguousarray(np.asarray(x, dtype=dtype)),
                               asnumpy=lambda x: np.asarray(x).copy(), empty=np.empty,
                               empty_like=np.empty_like, int32=np.int32, uint8=np.uint8)
    return cp, Kernel(score_badness), Kernel(score), Kernel(enumerate_)


CONFIGS = {
    "a": dict(n=20, seed=7, generations=14, elite_size=16, energy_window=12, global_every=5, extra=3),
    "b": dict(n=20, seed=31, generations=8, elite_size=8, energy_window=4, global_every=0, extra=0),
    "c": dict(n=75, seed=11, generations=3, elite_size=8, energy_window=12, global_every=3, extra=0),
}


def run(dll, cfg):
    cp, k_bad, k_score, k_enum = make_kernels(dll)
    gpu_exhaustive_beam._kernels = lambda: (cp, None, k_bad, k_score)
    gpu_exhaustive_beam._enumerate_kernel = lambda: k_enum
    n = cfg["n"]
    initial = state.random_state(n, Random(91001 + cfg["seed"]))
    extra = None
    if cfg["extra"]:
        rows = []
        for i in range(cfg["extra"]):
            s = state.random_state(n, Random(92001 + 17 * i + cfg["seed"]))
            rows.append(np.column_stack((s.P, s.Q)))
        extra = np.asarray(rows, np.int32)
    snaps = []
    result = gpu_exhaustive_beam.gpu_exhaustive_beam_search(
        initial, seed=cfg["seed"], generations=cfg["generations"], elite_size=cfg["elite_size"],
        energy_window=cfg["energy_window"], initial_elites=extra, global_every=cfg["global_every"],
        report_every=1, callback=snaps.append)
    E = cfg["elite_size"]
    elite_scores = np.full((len(snaps), E), -1, np.int32)
    elites = np.full((len(snaps), E, n, 2), -1, np.int8)
    for g, s in enumerate(snaps):
        elite_scores[g, :len(s.elite_scores)] = s.elite_scores
        elites[g, :len(s.elite_values)] = s.elite_values
    out = {"initial_p": np.asarray(initial.P, np.int32), "initial_q": np.asarray(initial.Q, np.int32),
           "extra": extra if extra is not None else np.zeros((0, n, 2), np.int32),
           "generation": np.asarray([s.generation for s in snaps], np.int32),
           "evaluations": np.asarray([s.evaluations for s in snaps], np.int64),
           "generation_best": np.asarray([s.generation_best for s in snaps], np.int32),
           "best_score": np.asarray([s.best_score for s in snaps], np.int32),
           "elite_scores": elite_scores, "elites": elites,
           "result_score": np.asarray(result.score), "result_generations": np.asarray(result.generations),
           "result_evaluations": np.asarray(result.evaluations),
           "result_p": np.asarray(result.state.P, np.int32), "result_q": np.asarray(result.state.Q, np.int32)}
    for k in ("n", "seed", "generations", "elite_size", "energy_window", "global_every"):
        out[k] = np.asarray(cfg[k])
    print(f"{cfg}: best {result.score} after {result.generations} generations, "
          f"{result.evaluations} evaluations; per generation {out['best_score'].tolist()}")
    return out


def main():
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        dll = build_enumerate(Path(tmp))
        for name, cfg in CONFIGS.items():
            res = run(dll, cfg)
            out.update({f"{name}/{k}": v for k, v in res.items()})
    np.savez_compressed(HERE / "exhaustive_golden.npz", **out)


if __name__ == "__main__":
    main()
