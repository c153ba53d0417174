"""Generate the multi-point move fixtures (neighborhood_golden.npz) from the
reference itself.

Run once, in a container that has the reference checked out and numba installed:

    NUMBA_CACHE_DIR=/tmp/n3_numba python tests/golden/make_golden_neighborhood.py [/path/to/reference]

Every number below is an output of the reference's own functions:

* ``search.legal_three_cycle_candidates`` (search.py:38-65) and
  ``accelerated.evaluate_three_cycles`` (accelerated.py:196-276) on seeded states;
* ``gpu_neighborhood.best_four_cycle`` / ``best_double_switch``
  (gpu_neighborhood.py:70-211) and ``bad_anchor_indices`` (:128-132).  These
  score their candidate states with ``score_population_gpu`` (CuPy, absent here);
  the script replaces that one function by the reference's CPU count
  ``accelerated.score_and_badness`` (the same integer, accelerated.py:14-37)
  and runs the rest of the reference code unchanged, at grid sizes the CPU
  scores in seconds.

The GPU box never runs this script; tests read the fixture.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path
from random import Random

import numpy as np

HERE = Path(__file__).resolve().parent
if len(sys.argv) > 1:
    REFERENCE = Path(sys.argv[1])
elif os.environ.get("N3_REFERENCE"):
    REFERENCE = Path(os.environ["N3_REFERENCE"])
else:
    raise SystemExit("usage: make_golden_neighborhood.py /path/to/reference  (or set N3_REFERENCE)")
sys.path.insert(0, str(REFERENCE / "src"))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/n3_numba_cache")

from no_three_75 import accelerated, gpu_neighborhood, search, state  # noqa: E402


def cpu_score_population(p_batch, q_batch):
    p = np.ascontiguousarray(p_batch, dtype=np.int32)
    q = np.ascontiguousarray(q_batch, dtype=np.int32)
    return np.asarray([accelerated.score_and_badness(p[i], q[i])[0] for i in range(p.shape[0])], dtype=np.int32)


def main():
    out = {}
    # three-cycle scores (accelerated.py:196-276) over every legal candidate of a few anchors
    for n, seeds in ((20, range(3)), (75, range(2))):
        rows = []
        for k in seeds:
            s = state.random_state(n, Random(91001 + k))
            p, q = np.asarray(s.P, np.int32), np.asarray(s.Q, np.int32)
            score, bad = accelerated.score_and_badness(p, q)
            anchor = (7 * k + 3) % (2 * n)
            cand = search.legal_three_cycle_candidates(p, q, anchor)
            sc = accelerated.evaluate_three_cycles(p, q, cand, score, bad)
            out[f"tc_n{n}_s{k}_p"] = p
            out[f"tc_n{n}_s{k}_q"] = q
            out[f"tc_n{n}_s{k}_anchor"] = np.asarray(anchor)
            out[f"tc_n{n}_s{k}_cand"] = cand
            out[f"tc_n{n}_s{k}_scores"] = sc
            rows.append(len(cand))
        print("three-cycles", n, rows)
    # four-cycle / double-switch neighbourhood scans with the CPU count in place of CuPy
    gpu_neighborhood.score_population_gpu = cpu_score_population
    cases = []
    for n, seed, anchors in ((10, 91001, 2), (14, 91002, 2), (18, 91003, 1)):
        s = state.random_state(n, Random(seed))
        picks = gpu_neighborhood.bad_anchor_indices(s, anchors)
        for a in picks:
            r4 = gpu_neighborhood.best_four_cycle(s, a)
            r2 = gpu_neighborhood.best_double_switch(s, a)
            tag = f"nb_n{n}_a{a}"
            out[f"{tag}_p"] = np.asarray(s.P, np.int32)
            out[f"{tag}_q"] = np.asarray(s.Q, np.int32)
            out[f"{tag}_four"] = np.asarray([r4.score, r4.evaluated, r4.legal], np.int64)
            out[f"{tag}_four_P"] = np.asarray(r4.state.P, np.int32)
            out[f"{tag}_four_Q"] = np.asarray(r4.state.Q, np.int32)
            out[f"{tag}_double"] = np.asarray([r2.score, r2.evaluated, r2.legal], np.int64)
            out[f"{tag}_double_P"] = np.asarray(r2.state.P, np.int32)
            out[f"{tag}_double_Q"] = np.asarray(r2.state.Q, np.int32)
            cases.append((n, a))
            print("scan", n, a, "four", r4.score, r4.evaluated, r4.legal, "double", r2.score, r2.evaluated, r2.legal)
        out[f"nb_n{n}_anchors"] = np.asarray(picks, np.int32)
    out["nb_cases"] = np.asarray(cases, np.int32)
    np.savez_compressed(HERE / "neighborhood_golden.npz", **out)


if __name__ == "__main__":
    main()
