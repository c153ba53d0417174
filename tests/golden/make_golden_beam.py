"""Generate the device-beam-search golden fixture (beam_golden.npz) from the
reference itself.

Run once, in a container that has the reference checked out and numba and g++
installed:

    NUMBA_CACHE_DIR=/tmp/n3_numba python tests/golden/make_golden_beam.py [/path/to/reference]

What is the reference's own code here:

* the mutation kernel: the CUDA C source string ``MUTATION_SOURCE`` of
  gpu_device_search.py:17-114 is read from the imported module at run time and
  compiled for the CPU (g++, into a temporary directory) behind a small shim that
  maps ``blockIdx``/``threadIdx`` to a loop over children; its source is never
  copied into this repository;
* ``rank_elites`` and ``elite_key`` (gpu_device_search.py:185-203) and the
  standard library's ``random.Random`` used by the search for its diversity
  shuffle (gpu_device_search.py:280, 343);
* ``accelerated.score_and_badness`` (accelerated.py:14-37) for every count: the
  reference's CUDA score and badness kernels (gpu.py:13-42,
  gpu_device_search.py:118-161) count the same collinear triples.

The generation loop below follows ``gpu_device_beam_search``
(gpu_device_search.py:254-432) step by step, with its CuPy arrays replaced by
NumPy ones.  The GPU box never runs this script; tests read the fixture.
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
    raise SystemExit("usage: make_golden_beam.py /path/to/reference  (or set N3_REFERENCE)")
sys.path.insert(0, str(REFERENCE / "src"))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/n3_numba_cache")

from no_three_75 import accelerated, gpu_device_search, state  # noqa: E402

SHIM = r"""
#define __device__
#define __global__
#define __forceinline__ inline
struct shim_dim3 { unsigned int x; };
static shim_dim3 blockIdx, blockDim, threadIdx;
"""

DRIVER = r"""
extern "C" void run_mutation(const int* parent_p, const int* parent_q, const int* parent_badness, int elite_count,
                             int quality_count, int n, int population, int active_strength, int max_strength,
                             int bad_bias, unsigned long long base_seed, int generation, int* child_p, int* child_q) {
  blockDim.x = 256;
  for (int child = 0; child < population; ++child) {
    blockIdx.x = child / 256;
    threadIdx.x = child % 256;
    mutate_population(parent_p, parent_q, parent_badness, elite_count, quality_count, n, population,
                      active_strength, max_strength, bad_bias, base_seed, generation, child_p, child_q);
  }
}
"""


def build_mutation(tmp: Path):
    src = tmp / "mutation.cpp"
    src.write_text(SHIM + gpu_device_search.MUTATION_SOURCE + DRIVER)
    lib = tmp / "mutation.so"
    subprocess.run(["g++", "-O2", "-shared", "-fPIC", "-o", str(lib), str(src)], check=True)
    dll = ctypes.CDLL(str(lib))
    P = ctypes.c_void_p
    I = ctypes.c_int
    dll.run_mutation.argtypes = [P, P, P, I, I, I, I, I, I, I, ctypes.c_ulonglong, I, P, P]
    dll.run_mutation.restype = None
    return dll


def mutate(dll, ep, eq, eb, quality_count, population, active, max_strength, bad_bias, seed, generation):
    ep = np.ascontiguousarray(ep, dtype=np.int32)
    eq = np.ascontiguousarray(eq, dtype=np.int32)
    eb = np.ascontiguousarray(eb, dtype=np.int32)
    n = ep.shape[1]
    cp_ = np.empty((population, n), dtype=np.int32)
    cq_ = np.empty((population, n), dtype=np.int32)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    dll.run_mutation(ptr(ep), ptr(eq), ptr(eb), ep.shape[0], quality_count, n, population, active, max_strength,
                     bad_bias, seed, generation, ptr(cp_), ptr(cq_))
    return cp_, cq_


def score(p, q):
    """E and badness of every state (accelerated.score_and_badness)."""
    e = np.empty(p.shape[0], dtype=np.int32)
    b = np.empty((p.shape[0], 2 * p.shape[1]), dtype=np.int32)
    for i in range(p.shape[0]):
        s, bad = accelerated.score_and_badness(p[i].astype(np.int32), q[i].astype(np.int32))
        e[i], b[i] = s, bad
    return e, b


def normalize(p, q):
    n = p.shape[0]
    pts = [(r, int(p[r])) for r in range(n)] + [(r, int(q[r])) for r in range(n)]
    s = state.points_to_permutations(pts, n)
    return np.asarray(s.P, dtype=np.int32), np.asarray(s.Q, dtype=np.int32)


def beam_search(dll, initial_p, initial_q, extra, *, seed, generations, population, elite_size, max_strength,
                energy_window, bad_bias=85):
    """gpu_device_beam_search (gpu_device_search.py:254-432) with NumPy arrays."""
    n = initial_p.shape[0]
    rng = Random(seed)
    base = np.column_stack((initial_p, initial_q)).astype(np.int32)[None]
    if extra is not None:
        base = np.concatenate((base, extra.astype(np.int32)), axis=0)
    base = base[:elite_size]
    ep, eq = base[:, :, 0].copy(), base[:, :, 1].copy()
    es, eb = score(ep, eq)
    order = gpu_device_search.rank_elites(es, eb)
    ep, eq, eb, es = ep[order], eq[order], eb[order], es[order]
    best_score = int(es[0])
    best_key = gpu_device_search.elite_key(best_score, eb[0])
    best_p, best_q = ep[0].copy(), eq[0].copy()
    evaluations = len(base)
    last_improvement = 0
    hist = {"generation_best": [], "best_score": [], "elite_scores": [], "elite_p": [], "elite_q": []}
    completed = 0
    for generation in range(1, generations + 1):
        completed = generation
        active = min(max_strength, 2 + (generation - last_improvement) // 10)
        quality_count = max(1, min(len(es), elite_size // 4))
        cp_, cq_ = mutate(dll, ep, eq, eb, quality_count, population, active, max_strength, bad_bias, seed,
                          generation)
        scores, _ = score(cp_, cq_)
        evaluations += population
        order = np.argsort(scores, kind="stable")
        quality_keep = max(1, elite_size // 4)
        selected = list(map(int, order[:quality_keep]))
        selected_set = set(selected)
        diverse = list(map(int, np.flatnonzero(scores <= best_score + energy_window)))
        rng.shuffle(diverse)
        for index in diverse:
            if index not in selected_set:
                selected.append(index)
                selected_set.add(index)
                if len(selected) == elite_size:
                    break
        if len(selected) < elite_size:
            for raw in order:
                index = int(raw)
                if index not in selected_set:
                    selected.append(index)
                    selected_set.add(index)
                    if len(selected) == elite_size:
                        break
        sel = np.asarray(selected, dtype=np.int64)
        ep, eq = cp_[sel], cq_[sel]
        es = scores[sel]
        _, eb = score(ep, eq)
        rank = gpu_device_search.rank_elites(es, eb)
        ep, eq, eb, es = ep[rank], eq[rank], eb[rank], es[rank]
        generation_best = int(es[0])
        key = gpu_device_search.elite_key(generation_best, eb[0])
        if key < best_key:
            best_score, best_key = generation_best, key
            best_p, best_q = ep[0].copy(), eq[0].copy()
            last_improvement = generation
        hist["generation_best"].append(generation_best)
        hist["best_score"].append(best_score)
        hist["elite_scores"].append(es.copy())
        hist["elite_p"].append(ep.astype(np.int8))
        hist["elite_q"].append(eq.astype(np.int8))
        if best_score == 0:
            break
    np_, nq_ = normalize(best_p, best_q)
    return {"completed": completed, "evaluations": evaluations, "best_score": best_score,
            "best_p_raw": best_p, "best_q_raw": best_q, "best_p": np_, "best_q": nq_,
            "generation_best": np.asarray(hist["generation_best"], np.int32),
            "best_history": np.asarray(hist["best_score"], np.int32),
            "elite_scores": np.stack(hist["elite_scores"]).astype(np.int32),
            "elite_p": np.stack(hist["elite_p"]), "elite_q": np.stack(hist["elite_q"])}


CONFIGS = {
    "a": dict(n=20, seed=7, generations=25, population=512, elite_size=16, max_strength=6, energy_window=12,
              extra=3),
    "b": dict(n=75, seed=11, generations=6, population=1024, elite_size=64, max_strength=12, energy_window=12,
              extra=0),
}


def main():
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        dll = build_mutation(Path(tmp))
        # one direct call of the test-facing mutation wrapper (gpu_device_search.py:206-251 shape)
        par = [state.random_state(20, Random(91001 + i)) for i in range(8)]
        pp = np.asarray([s.P for s in par], np.int32)
        pq = np.asarray([s.Q for s in par], np.int32)
        _, pb = score(pp, pq)
        qc = max(1, min(8, 8 // 4))
        mp, mq = mutate(dll, pp, pq, pb, qc, 64, 3, 6, 85, 5, 2)
        out.update(mut_parent_p=pp, mut_parent_q=pq, mut_child_p=mp, mut_child_q=mq)
        for name, cfg in CONFIGS.items():
            n = cfg["n"]
            init = state.random_state(n, Random(91001))
            extra = None
            if cfg["extra"]:
                ex = [state.random_state(n, Random(91002 + i)) for i in range(cfg["extra"])]
                extra = np.asarray([np.column_stack((s.P, s.Q)) for s in ex], np.int32)
                out[f"{name}_extra"] = extra
            res = beam_search(dll, np.asarray(init.P, np.int32), np.asarray(init.Q, np.int32), extra,
                              seed=cfg["seed"], generations=cfg["generations"], population=cfg["population"],
                              elite_size=cfg["elite_size"], max_strength=cfg["max_strength"],
                              energy_window=cfg["energy_window"])
            out[f"{name}_initial_p"] = np.asarray(init.P, np.int32)
            out[f"{name}_initial_q"] = np.asarray(init.Q, np.int32)
            out[f"{name}_config"] = np.asarray([n, cfg["seed"], cfg["generations"], cfg["population"],
                                                cfg["elite_size"], cfg["max_strength"], cfg["energy_window"]],
                                               np.int64)
            for k, v in res.items():
                out[f"{name}_{k}"] = np.asarray(v)
            print(name, "best", res["best_score"], "completed", res["completed"], "gen_best",
                  res["generation_best"].tolist())
    np.savez_compressed(HERE / "beam_golden.npz", **out)


if __name__ == "__main__":
    main()
