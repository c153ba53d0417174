"""Generate the line-weight fixture (breakout_golden.npz) from the reference itself.

Run once, in a container that has the reference checked out and numba installed:

    NUMBA_CACHE_DIR=/tmp/n3_numba python tests/golden/make_golden_breakout.py [/path/to/reference]

Outputs of the reference's ``breakout.weighted_candidate_scores`` and
``breakout.weighted_state_score`` (src/no_three_75/breakout.py:39-86) on seeded
states, with raw partner scores from ``accelerated.evaluate_two_switches`` and
weights on the state's own occupied lines (``conflicts.analyze_points``, as
breakout search adds them) plus seeded lines through random grid points
(``geometry.canonical_line``).  The GPU box never runs this script.
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
    raise SystemExit("usage: make_golden_breakout.py /path/to/reference  (or set N3_REFERENCE)")
sys.path.insert(0, str(REFERENCE / "src"))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/n3_numba_cache")

from no_three_75 import accelerated, breakout, conflicts, geometry, state  # noqa: E402


def main():
    out = {}
    k = 0
    for n, seeds in ((20, 4), (75, 3)):
        for s in range(seeds):
            st = state.random_state(n, Random(91001 + s))
            p, q = np.asarray(st.P, np.int32), np.asarray(st.Q, np.int32)
            raw_score, bad = accelerated.score_and_badness(p, q)
            rng = Random(500 + 17 * s + n)
            pts = [(r, int(p[r])) for r in range(n)] + [(r, int(q[r])) for r in range(n)]
            weights = {line.key: rng.randint(1, 6) for line in conflicts.analyze_points(pts).lines}
            for _ in range(10):
                a = (rng.randrange(n), rng.randrange(n))
                b = (rng.randrange(n), rng.randrange(n))
                if a != b:
                    weights[geometry.canonical_line(a, b)] = rng.randint(0, 5)
            keys = np.asarray(list(weights), np.int64).reshape(-1, 3)
            vals = np.asarray(list(weights.values()), np.int64)
            sel = [rng.randrange(2 * n) for _ in range(4)]
            scores = []
            for u in sel:
                raw = accelerated.evaluate_two_switches(p, q, u, raw_score, bad)
                scores.append(breakout.weighted_candidate_scores(p, q, u, raw, weights))
            tag = f"w{k}"
            out.update({f"{tag}_p": p, f"{tag}_q": q, f"{tag}_keys": keys, f"{tag}_vals": vals,
                        f"{tag}_sel": np.asarray(sel, np.int32),
                        f"{tag}_raw": np.stack([accelerated.evaluate_two_switches(p, q, u, raw_score, bad)
                                                for u in sel]),
                        f"{tag}_scores": np.stack(scores),
                        f"{tag}_state": np.asarray(breakout.weighted_state_score(p, q, int(raw_score), weights)),
                        f"{tag}_raw_score": np.asarray(int(raw_score))})
            print(tag, n, len(weights), "weighted state", int(out[f"{tag}_state"]), "raw", raw_score)
            k += 1
    out["count"] = np.asarray(k)
    np.savez_compressed(HERE / "breakout_golden.npz", **out)


if __name__ == "__main__":
    main()
