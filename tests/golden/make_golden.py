"""Generate the golden fixtures in this directory from the reference itself.

Run once, in a container that has the reference checked out (read-only is
fine) and numba installed:

    NUMBA_CACHE_DIR=/tmp/n3_numba python tests/golden/make_golden.py [/path/to/reference]

The reference (MilliganCo/no-three-in-line, package ``no_three_75``) is
imported from ``<reference>/src``; nothing here copies its code.  Every number
written below is an output of the reference's own functions:

* ``accelerated.score_and_badness`` (accelerated.py:14-37), the CPU
  determinant verifier for counts, and ``conflicts.full_triple_score``
  (conflicts.py:75-76) / ``conflicts.analyze_points`` (conflicts.py:36-72);
* ``accelerated.evaluate_two_switches`` / ``evaluate_transpositions``
  (accelerated.py:40-195), with the seeds and sizes of tests/test_delta.py;
* ``verifier_a`` / ``verifier_b`` witnesses (verifier_a.py:12-16,
  verifier_b.py:22-33) on the seeded small sets of
  tests/test_verifier_agreement.py;
* ``state.random_state`` (state.py:88-95) populations with seeds 91001+i
  (cli.py:203-204) and ``state.points_to_permutations`` (state.py:47-85);
* the reference's fixture results/best-near-solution-E10.json (E = 10).

The GPU box never runs this script; tests read the fixtures it wrote.
"""
from __future__ import annotations

import hashlib
import json
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
    raise SystemExit("usage: make_golden.py /path/to/reference  (or set N3_REFERENCE)")
sys.path.insert(0, str(REFERENCE / "src"))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/n3_numba_cache")

from no_three_75 import accelerated, conflicts, geometry, state, verifier_a, verifier_b  # noqa: E402


def population(n: int, count: int, base: int = 91001):
    p = np.empty((count, n), dtype=np.int32)
    q = np.empty((count, n), dtype=np.int32)
    for i in range(count):
        s = state.random_state(n, Random(base + i))
        p[i], q[i] = s.P, s.Q
    return p, q


def columns_of(p, q):
    c = np.empty(p.shape[:-1] + (2 * p.shape[-1],), dtype=np.int16)
    c[..., 0::2] = p
    c[..., 1::2] = q
    return c


def score_cols(cols):
    s, b = accelerated.score_and_badness(cols[0::2].astype(np.int32).copy(), cols[1::2].astype(np.int32).copy())
    return int(s), np.asarray(b, dtype=np.int64)


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.int32).tobytes())
    return h.hexdigest()


def make_c1():
    """n=20: 256 seeded states and 10^4 random row-pair column swaps, each
    scored by full recompute with the reference's score_and_badness."""
    n, count = 20, 256
    p, q = population(n, count)
    cols = columns_of(p, q)
    E = np.zeros(count, np.int32)
    bad = np.zeros((count, 2 * n), np.int16)
    E_lines = np.zeros(count, np.int32)
    for b in range(count):
        s, bb = score_cols(cols[b])
        E[b], bad[b] = s, bb
        E_lines[b] = conflicts.analyze_points(state.PairPermutations(tuple(p[b]), tuple(q[b])).points()).triples
        assert conflicts.full_triple_score(state.PairPermutations(tuple(p[b]), tuple(q[b])).points()) == s
    rng = Random(7)
    work = cols.copy()
    cur = [score_cols(work[b]) for b in range(count)]
    swaps = np.zeros((10000, 3), np.int32)
    valid = np.zeros(10000, np.int8)
    dE = np.zeros(10000, np.int32)
    E_after = np.zeros(10000, np.int32)
    dbad_sumsq = np.zeros(10000, np.int64)
    for t in range(10000):
        b, u, v = rng.randrange(count), rng.randrange(2 * n), rng.randrange(2 * n)
        swaps[t] = (b, u, v)
        c = work[b]
        cu, cv = int(c[u]), int(c[v])
        ok = (u >> 1) != (v >> 1) and cu != cv and int(c[u ^ 1]) != cv and int(c[v ^ 1]) != cu
        valid[t] = ok
        if not ok:
            E_after[t] = cur[b][0]
            continue
        moved = c.copy()
        moved[u], moved[v] = cv, cu
        s_new, b_new = score_cols(moved)
        dE[t] = s_new - cur[b][0]
        dbad = b_new - cur[b][1]
        dbad_sumsq[t] = int(np.dot(dbad, dbad))
        E_after[t] = s_new
        work[b] = moved
        cur[b] = (s_new, b_new)
    final_E = np.asarray([cur[b][0] for b in range(count)], np.int32)
    np.savez_compressed(HERE / "c1_n20.npz", p=p.astype(np.uint8), q=q.astype(np.uint8), E=E,
                        badness=bad, E_lines=E_lines, swaps=swaps, valid=valid, dE=dE,
                        E_after=E_after, dbad_sumsq=dbad_sumsq, final_cols=work.astype(np.uint8),
                        final_E=final_E)
    print("c1", E.mean(), valid.sum())


def make_c2():
    """n=75: 4096 seeded states; E and badness of every state."""
    n, count = 75, 4096
    p, q = population(n, count)
    cols = columns_of(p, q)
    E = np.zeros(count, np.int32)
    bad = np.zeros((count, 2 * n), np.int16)
    for b in range(count):
        s, bb = score_cols(cols[b])
        E[b], bad[b] = s, bb
    assert bad.max() < 256
    lines = []
    for b in range(16):
        m = conflicts.analyze_points(state.PairPermutations(tuple(p[b]), tuple(q[b])).points())
        assert m.triples == E[b] and tuple(m.badness) is not None
        lines.append([m.triples, m.violating_lines, m.max_line_occupancy, m.max_point_badness])
    np.savez_compressed(HERE / "c2_n75.npz", p256=p[:256].astype(np.uint8), q256=q[:256].astype(np.uint8),
                        E=E, badness=bad.astype(np.uint8), lines16=np.asarray(lines, np.int32),
                        pq_sha256=np.asarray(digest(p, q)))
    print("c2", E.mean(), E.min(), E.max())


def make_mixed():
    """Seed digests for the mixed-size chain sets: chain c of size n starts from
    random_state(n, Random(91001 + c)) with c counted inside each size."""
    out = {}
    for n, count in [(40, 1024), (52, 768), (60, 512), (68, 384), (75, 256)]:
        p, q = population(n, count)
        out[str(n)] = {"count": count, "pq_sha256": digest(p, q)}
    (HERE / "mixed_seeds.json").write_text(json.dumps(out, indent=1) + "\n")


def make_e10():
    sys.path.insert(0, str(REFERENCE / "src"))
    from no_three_75.io import load_candidate

    n, points, _ = load_candidate(REFERENCE / "results" / "best-near-solution-E10.json")
    st = state.points_to_permutations(points, n)
    p = np.asarray(st.P, np.int32)
    q = np.asarray(st.Q, np.int32)
    s, bb = accelerated.score_and_badness(p, q)
    m = conflicts.analyze_points(st.points())
    wa = verifier_a.find_collinear_triple(points)
    wb = verifier_b.find_collinear_triple(points)
    np.savez_compressed(HERE / "e10.npz", n=np.asarray(n), points=np.asarray(points, np.int16),
                        p=p.astype(np.uint8), q=q.astype(np.uint8), E=np.asarray(int(s)),
                        badness=np.asarray(bb, np.int16), full_triple_score=np.asarray(conflicts.full_triple_score(points)),
                        violating_lines=np.asarray(m.violating_lines), max_line_occupancy=np.asarray(m.max_line_occupancy),
                        line_badness=np.asarray(m.badness, np.int16),
                        witness_a=np.asarray(wa, np.int16), witness_b=np.asarray(wb, np.int16))
    print("e10", int(s), m.violating_lines, wa, wb)


def make_delta_pins():
    """Outputs of evaluate_two_switches / evaluate_transpositions with the seeds
    and sizes of the reference's tests/test_delta.py, plus n=75 anchors."""
    two, trans = [], []
    rng = Random(443)
    for n in range(4, 11):
        for _ in range(5):
            st = state.random_state(n, rng)
            p = np.asarray(st.P, np.int32)
            q = np.asarray(st.Q, np.int32)
            s, bad = accelerated.score_and_badness(p, q)
            u = rng.randrange(2 * n)
            out = accelerated.evaluate_two_switches(p, q, u, s, bad)
            two.append({"p": p.tolist(), "q": q.tolist(), "u": u, "score": int(s),
                        "badness": [int(x) for x in bad], "out": [int(x) for x in out]})
    rng = Random(9817)
    for n in range(4, 13):
        for _ in range(8):
            st = state.random_state(n, rng)
            p = np.asarray(st.P, np.int32)
            q = np.asarray(st.Q, np.int32)
            s, bad = accelerated.score_and_badness(p, q)
            for _ in range(4):
                layer, row = rng.randrange(2), rng.randrange(n)
                out = accelerated.evaluate_transpositions(p, q, layer, row, s, bad)
                trans.append({"p": p.tolist(), "q": q.tolist(), "layer": layer, "row": row, "score": int(s),
                              "badness": [int(x) for x in bad], "out": [int(x) for x in out]})
    p75, q75 = population(75, 8)
    big = []
    rng = Random(75)
    for b in range(8):
        s, bad = accelerated.score_and_badness(p75[b], q75[b])
        for _ in range(2):
            u = rng.randrange(150)
            out = accelerated.evaluate_two_switches(p75[b], q75[b], u, s, bad)
            big.append({"state": b, "u": u, "score": int(s), "out": [int(x) for x in out]})
    (HERE / "delta_pins.json").write_text(json.dumps({"two_switches": two, "transpositions": trans,
                                                       "two_switches_n75": big}) + "\n")
    print("delta", len(two), len(trans), len(big))


def make_geometry_pins():
    """Known answers of tests/test_geometry.py plus witness existence of both
    verifiers on the seeded sets of tests/test_verifier_agreement.py."""
    known = [[[0, 0], [3, 2], [6, 4]], [[0, 0], [3, 2], [6, 5]], [[2, 0], [2, 4], [2, 9]], [[0, 7], [4, 7], [9, 7]],
             [[0, 0], [2, 2], [5, 5]]]
    dets = [geometry.determinant(*map(tuple, t)) for t in known]
    rng = Random(20260904)
    sets = []
    for _ in range(3000):
        n = rng.randint(2, 9)
        grid = [(r, c) for r in range(n) for c in range(n)]
        size = rng.randint(0, min(14, len(grid)))
        pts = rng.sample(grid, size)
        wa = verifier_a.find_collinear_triple(pts)
        wb = verifier_b.find_collinear_triple(pts)
        assert (wa is None) == (wb is None)
        count = conflicts.full_triple_score(pts) if len(pts) >= 3 else 0
        sets.append({"points": [list(x) for x in pts], "collinear": wa is not None, "E": count})
    lines = {"canonical": [list(geometry.canonical_line((1, 2), (4, 8))), list(geometry.canonical_line((4, 8), (1, 2))),
                           list(geometry.canonical_line((7, 14), (1, 2)))]}
    (HERE / "geometry_pins.json").write_text(json.dumps({"known": known, "determinants": dets, "sets": sets,
                                                          **lines}) + "\n")
    print("geometry", sum(s["collinear"] for s in sets))


if __name__ == "__main__":
    make_geometry_pins()
    make_delta_pins()
    make_e10()
    make_c1()
    make_mixed()
    make_c2()
