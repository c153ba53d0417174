"""Generate the line-table fixture (lines_golden.npz) from the reference itself.

Run once, in a container that has the reference checked out:

    python tests/golden/make_golden_lines.py [/path/to/reference]

``no_three_75.precompute`` imports ``cp_sat``, which imports ``ortools`` at the
top; ortools is not installed here and none of the functions used below touch
it, so an empty stand-in module satisfies the import.  Outputs of the
reference's ``build_geometry_tables`` (src/no_three_75/precompute.py:35-57):
the whole tables for small grids, and SHA-256 digests of the three arrays plus
the sizes for n = 20, 40 and 75 (the n = 75 pair table alone is 63 MB).  Scores
of ``score_pair_table`` and ``score_csr`` (:60-89) on seeded states and on
point lists that reach their edge cases: rows and columns with three or more
points (not in the tables), negative ids (wrapped by NumPy indexing in
score_csr), repeated points, empty and two-point lists.  The GPU box never runs
this script.
"""
from __future__ import annotations

import hashlib
import os
import sys
import types
from pathlib import Path
from random import Random

import numpy as np

HERE = Path(__file__).resolve().parent
if len(sys.argv) > 1:
    REFERENCE = Path(sys.argv[1])
elif os.environ.get("N3_REFERENCE"):
    REFERENCE = Path(os.environ["N3_REFERENCE"])
else:
    raise SystemExit("usage: make_golden_lines.py /path/to/reference  (or set N3_REFERENCE)")
sys.path.insert(0, str(REFERENCE / "src"))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/n3_numba_cache")

_stub = {name: types.ModuleType(name) for name in ("ortools", "ortools.sat", "ortools.sat.python",
                                                     "ortools.sat.python.cp_model")}
_stub["ortools"].sat = _stub["ortools.sat"]
_stub["ortools.sat"].python = _stub["ortools.sat.python"]
_stub["ortools.sat.python"].cp_model = _stub["ortools.sat.python.cp_model"]
for _name, _module in _stub.items():
    sys.modules.setdefault(_name, _module)

from no_three_75 import precompute, state  # noqa: E402


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    out = {}
    for n in (1, 2, 3, 4, 5, 7, 10, 13):
        t = precompute.build_geometry_tables(n)
        out.update({f"t{n}_pair_to_line": t.pair_to_line, f"t{n}_offsets": t.offsets, f"t{n}_indices": t.indices,
                    f"t{n}_line_count": np.asarray(t.line_count)})
    big = {}
    for n in (20, 40, 75):
        t = precompute.build_geometry_tables(n)
        big[n] = t
        out[f"h{n}"] = np.asarray([digest(t.pair_to_line), digest(t.offsets), digest(t.indices)])
        out[f"h{n}_sizes"] = np.asarray([t.line_count, len(t.indices), len(t.pair_to_line)], np.int64)
        print(n, t.line_count, len(t.indices), f"{t.build_seconds:.1f} s")

    # point lists: (n, points); score_pair_table may raise ValueError, score_csr IndexError
    lists = []
    for n, seeds in ((10, 3), (13, 3), (20, 2), (40, 2), (75, 3)):
        for s in range(seeds):
            st = state.random_state(n, Random(91001 + 7 * s + n))
            lists.append((n, [(r, int(st.P[r])) for r in range(n)] + [(r, int(st.Q[r])) for r in range(n)]))
    rng = Random(4242)
    for n in (7, 10, 13):
        grid = [(r, c) for r in range(n) for c in range(n)]
        lists.append((n, rng.sample(grid, 3 * n)))                         # rows with 3+ points
        lists.append((n, [(2, c) for c in range(n)] + [(k, k) for k in range(n) if k != 2]))
        lists.append((n, [(k, n - 1 - k) for k in range(n)] + [(0, 0), (n - 1, n - 1)]))
    lists.append((10, []))
    lists.append((10, [(3, 4)]))
    lists.append((10, [(3, 4), (5, 6)]))
    lists.append((10, [(0, 0), (1, 1), (2, 2), (2, 2)]))                    # a repeated point
    lists.append((10, [(0, -1), (1, 1), (2, 3), (3, 5), (9, 9)]))           # id -1 wraps in score_csr
    lists.append((10, [(1, 1), (2, 2), (3, 3), (10, 0)]))                   # id 100: out of range
    tables = {n: precompute.build_geometry_tables(n) for n in {n for n, _ in lists} if n not in big}
    tables.update(big)
    flat, starts, ns, pair_scores, csr_scores = [], [0], [], [], []
    for n, pts in lists:
        t = tables[n]
        try:
            ps = precompute.score_pair_table(pts, t)
        except ValueError:
            ps = -1
        try:
            cs = precompute.score_csr(pts, t)
        except IndexError:
            cs = -1
        flat.extend(pts)
        starts.append(len(flat))
        ns.append(n)
        pair_scores.append(ps)
        csr_scores.append(cs)
    out.update({"points": np.asarray(flat, np.int32).reshape(-1, 2), "starts": np.asarray(starts, np.int64),
                "n": np.asarray(ns, np.int32), "pair_scores": np.asarray(pair_scores, np.int64),
                "csr_scores": np.asarray(csr_scores, np.int64)})
    np.savez_compressed(HERE / "lines_golden.npz", **out)
    print("lists", len(ns), "pair", pair_scores, "csr", csr_scores)


if __name__ == "__main__":
    main()
