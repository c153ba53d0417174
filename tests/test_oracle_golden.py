"""The CPU oracle against the reference's own outputs (tests/golden/*).

These pin the oracle before it is trusted as the checker of the CUDA path:
every fixture value below was produced by the reference package itself
(tests/golden/make_golden.py).
"""
from __future__ import annotations

import hashlib

import numpy as np

from no_three_in_line_b200 import state


def _digest(p, q):
    h = hashlib.sha256()
    for a in (p, q):
        h.update(np.ascontiguousarray(a, dtype=np.int32).tobytes())
    return h.hexdigest()


def test_random_state_reproduces_reference_populations(golden):
    c1 = golden("c1_n20.npz")
    p, q = state.seeded_population(20, 256)
    assert np.array_equal(p, c1["p"]) and np.array_equal(q, c1["q"])
    c2 = golden("c2_n75.npz")
    p, q = state.seeded_population(75, 4096)
    assert np.array_equal(p[:256], c2["p256"]) and np.array_equal(q[:256], c2["q256"])
    assert _digest(p, q) == str(c2["pq_sha256"])


def test_mixed_size_seed_digests(golden):
    seeds = golden("mixed_seeds.json")
    for n, rec in seeds.items():
        p, q = state.seeded_population(int(n), rec["count"])
        assert _digest(p, q) == rec["pq_sha256"], n


def test_oracle_scores_c1_n20(golden, oracle):
    c1 = golden("c1_n20.npz")
    s, b = oracle.score_population(c1["p"], c1["q"], badness=True, threads=0)
    assert np.array_equal(s, c1["E"])
    assert np.array_equal(b, c1["badness"])
    assert np.array_equal(s, c1["E_lines"])  # conflicts.analyze_points sum of C(k,3)
    s2, b2 = oracle.slope_population(c1["p"], c1["q"], threads=0)
    assert np.array_equal(s2, c1["E"]) and np.array_equal(b2, c1["badness"])


def test_oracle_scores_c2_n75(golden, oracle):
    c2 = golden("c2_n75.npz")
    p, q = state.seeded_population(75, 4096)
    s, b = oracle.score_population(p, q, badness=True, threads=0)
    assert np.array_equal(s, c2["E"])
    assert np.array_equal(b, c2["badness"].astype(np.int32))
    s2, b2 = oracle.slope_population(p[:512], q[:512], threads=0)
    assert np.array_equal(s2, c2["E"][:512]) and np.array_equal(b2, c2["badness"][:512].astype(np.int32))
    # analyze_points (conflicts.py:36-72) on the first states: triples and max point badness
    for i, (triples, _lines, _occ, max_bad) in enumerate(c2["lines16"]):
        assert s[i] == triples and b[i].max() == max_bad


def test_oracle_e10_fixture(golden, oracle):
    e = golden("e10.npz")
    assert int(e["E"]) == 10 and int(e["full_triple_score"]) == 10 and int(e["violating_lines"]) == 10
    s, b = oracle.score_and_badness(e["p"], e["q"])
    assert s == 10 and np.array_equal(b, e["badness"].astype(np.int64))
    assert int(b.sum()) == 30
    s2, b2 = oracle.det_score_points(e["points"])
    assert s2 == 10
    s3, _ = oracle.slope_score_points(e["points"])
    assert s3 == 10
    # the reference's witness ((2,62),(5,50),(6,46)) is collinear
    (a, bb, c) = [tuple(x) for x in e["witness_a"]]
    assert (bb[0] - a[0]) * (c[1] - a[1]) == (bb[1] - a[1]) * (c[0] - a[0])
    assert np.array_equal(e["witness_a"], e["witness_b"])
    # P/Q recovered by points_to_permutations matches the reference's
    st = state.points_to_permutations([tuple(map(int, x)) for x in e["points"]], int(e["n"]))
    assert st.P == tuple(int(x) for x in e["p"]) and st.Q == tuple(int(x) for x in e["q"])


def test_oracle_geometry_and_verifier_agreement(golden, oracle):
    g = golden("geometry_pins.json")
    for tri, det in zip(g["known"], g["determinants"]):
        (a, b, c) = tri
        assert (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0]) == det
    assert g["canonical"][0] == g["canonical"][1] == g["canonical"][2]
    for rec in g["sets"]:
        pts = rec["points"]
        if len(pts) < 3:
            assert not rec["collinear"]
            continue
        e_det, _ = oracle.det_score_points(pts)
        e_slope, _ = oracle.slope_score_points(pts)
        assert e_det == e_slope == rec["E"]
        assert (e_det > 0) == rec["collinear"]


def test_oracle_two_switches_and_transpositions(golden, oracle):
    d = golden("delta_pins.json")
    for rec in d["two_switches"]:
        out = oracle.two_switches(rec["p"], rec["q"], rec["u"], rec["score"], rec["badness"])
        assert out.tolist() == rec["out"]
    for rec in d["transpositions"]:
        out = oracle.transpositions(rec["p"], rec["q"], rec["layer"], rec["row"], rec["score"], rec["badness"])
        assert out.tolist() == rec["out"]
    p, q = state.seeded_population(75, 8)
    for rec in d["two_switches_n75"]:
        b = rec["state"]
        s, bad = oracle.score_and_badness(p[b], q[b])
        assert s == rec["score"]
        out = oracle.two_switches(p[b], q[b], rec["u"], s, bad)
        assert out.tolist() == rec["out"]


def test_oracle_walk_delta_replays_c1_swaps(golden, oracle):
    """The restated walk delta (tempering.py:68-89) reproduces the reference's
    full-recompute delta for the 10^4 seeded n=20 swaps, including badness."""
    c1 = golden("c1_n20.npz")
    cols = state.pq_to_columns(c1["p"], c1["q"]).astype(np.int32)
    cur = [oracle.score_columns(c) for c in cols]
    for t, (b, u, v) in enumerate(c1["swaps"]):
        ok, dE, dbad = oracle.walk_delta(cols[b], u, v)
        assert ok == bool(c1["valid"][t])
        if not ok:
            continue
        assert dE == c1["dE"][t]
        assert int(np.dot(dbad.astype(np.int64), dbad)) == c1["dbad_sumsq"][t]
        cols[b][u], cols[b][v] = cols[b][v], cols[b][u]
        s_new, b_new = oracle.score_columns(cols[b])
        assert s_new == c1["E_after"][t] and np.array_equal(b_new - cur[b][1], dbad)
        cur[b] = (s_new, b_new)
    assert np.array_equal(cols, c1["final_cols"].astype(np.int32))
