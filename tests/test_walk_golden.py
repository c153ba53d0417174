"""The walk's badness-biased slot draw and umbrella restraint (CPU).

* The oracle's pieces (``bias_slot``, ``distance_delta``, ``walk_delta``),
  driven by the reference's own xorshift64* draws and double-precision
  acceptance, reproduce the reference's walk kernel step for step
  (tests/golden/walk_golden.npz, made by make_golden_walk.py from the
  reference's kernel source, tempering.py:29-115).
* The device's forms of those rules equal the oracle's: the slot as a count of
  running badness sums, and the umbrella acceptance in 2^-24 fixed point
  against the reference's exp(-(dE + s((off + dd)^2 - off^2)) / T).
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "walk_golden.npz"


def cases(z):
    return sorted({k.split("/")[0] for k in z.files})


def test_walk_pieces_reproduce_the_reference_kernel(oracle):
    with np.load(GOLDEN) as z:
        names = cases(z)
        assert {"n20_bias85", "n20_umbrella_bias85", "n75_bias85_umbrella"} <= set(names)
        for name in names:
            g = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}
            R = len(g["start_scores"])
            steps, bias = int(g["steps"]), int(g["bad_bias"])
            for r in range(R):
                st = {"cols": g["start_columns"][r], "bad": g["start_badness"][r], "score": int(g["start_scores"][r]),
                      "rng": int(g["start_rngs"][r]), "best_cols": g["start_columns"][r],
                      "best": int(g["start_scores"][r]), "acc": 0, "removed": int(g["start_removed"][r])}
                for chunk in range(g["hist_scores"].shape[0]):
                    out = oracle.walk_with_reference_rng(
                        st["cols"], st["bad"], st["score"], st["rng"], st["best_cols"], st["best"],
                        float(g["temperatures"][r]), st["acc"], g["reference"], st["removed"],
                        float(g["centers"][r]), float(g["strengths"][r]), steps, bias)
                    for key in ("columns", "badness", "scores", "rngs", "best_columns", "best_scores", "accepted",
                                "removed"):
                        want = g["hist_" + key][chunk][r]
                        got = out[key]
                        assert np.array_equal(np.asarray(got, np.uint64 if key == "rngs" else np.int64),
                                              np.asarray(want, np.uint64 if key == "rngs" else np.int64)), \
                            (name, r, chunk, key)
                    st = {"cols": out["columns"], "bad": out["badness"], "score": out["scores"], "rng": out["rngs"],
                          "best_cols": out["best_columns"], "best": out["best_scores"], "acc": out["accepted"],
                          "removed": out["removed"]}


def device_bias_slot(badness, m, target):
    """The device's rule (chain_move.cuh bias_pick, the candidate kernel's
    binary search): the number of inclusive running sums not above the
    target, at most m - 1."""
    run = np.cumsum(np.asarray(badness[:m], np.int64))
    return min(int(np.sum(run <= target)), m - 1)


def test_device_bias_rule_equals_the_reference_loop(oracle):
    rng = np.random.default_rng(3)
    for trial in range(300):
        m = int(rng.integers(4, 151))
        bad = rng.integers(0, 6, m) * (rng.random(m) < 0.4)
        total = int(bad.sum())
        if total == 0:
            continue
        for target in range(total):
            assert device_bias_slot(bad, m, target) == oracle.bias_slot(bad, m, target)


def test_bias_draw_frequencies_follow_badness(oracle):
    """floor(r * 3E / 2^32) over 32-bit words r is uniform on [0, 3E), so slot u
    is drawn with probability badness[u] / 3E, as the reference intends."""
    bad = np.array([0, 3, 0, 0, 6, 1, 2, 0, 0, 0, 3, 0, 0, 0, 0, 0], np.int64)
    total = int(bad.sum())
    words = np.random.default_rng(1).integers(0, 2 ** 32, 200000, dtype=np.uint64)
    targets = (words * np.uint64(total)) >> np.uint64(32)
    counts = np.bincount([device_bias_slot(bad, len(bad), int(t)) for t in targets[:20000]], minlength=len(bad))
    freq = counts / counts.sum()
    assert np.all(counts[bad == 0] == 0)
    assert np.allclose(freq, bad / total, atol=0.01)


def fixed_point_threshold(dE, umb_q, acc_row, frac_row, W):
    e = (dE << 24) + umb_q
    if e <= 0:
        return 1 << 32
    a, b = e >> 24, e & 0xFFFFFF
    if a >= W:
        return 0
    t = int(acc_row[a])
    for j, idx in enumerate((b >> 16, (b >> 8) & 255, b & 255)):
        if idx:
            t = (t * int(frac_row[256 * j + idx])) >> 32
    return t


def test_umbrella_acceptance_in_fixed_point(lib_tempering):
    """Threshold of the device test = 2^32 exp(-(dE + restraint) / T) of the
    reference (tempering.py:93-95) to within a few units of 2^-32, over
    strengths, centres, distances and both signs of dd."""
    tp = lib_tempering
    temps = tp.geometric_ladder(0.05, 5.0, 8)
    acc, frac = tp.metropolis_table(temps), tp.fraction_table(temps)
    W = acc.shape[1]
    rng = np.random.default_rng(7)
    for _ in range(4000):
        t = int(rng.integers(0, 8))
        s = np.float32(rng.choice([0.05, 0.2, 0.5, 1.7]))
        c = np.float32(rng.uniform(0, 40))
        removed = int(rng.integers(0, 150))
        dd = int(rng.integers(-2, 3))
        dE = int(rng.integers(-20, 30))
        sq, c2 = tp.umbrella_coefficients([s], [c])[0]
        umb = int(sq) * (2 * removed * dd + dd * dd) - int(c2) * dd
        energy = dE + float(s) * (2 * (removed - float(c)) * dd + dd * dd)
        # each coefficient is rounded to 2^-25 at most
        bound = (abs(2 * removed * dd + dd * dd) + abs(dd)) * 2.0 ** -25 + 1e-12
        assert abs(dE + umb / 2.0 ** 24 - energy) <= bound
        got = fixed_point_threshold(dE, umb, acc[t], frac[t], W)
        e_fixed = dE + umb / 2.0 ** 24
        want = 2.0 ** 32 if e_fixed <= 0 else 2.0 ** 32 * math.exp(-e_fixed / temps[t])
        assert abs(got - min(want, 2.0 ** 32)) <= 5 + 1e-6 * want, (dE, umb, t, got, want)


@pytest.fixture
def lib_tempering():
    from no_three_in_line_b200 import tempering

    return tempering
