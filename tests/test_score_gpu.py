"""(a) Population scoring on the GPU, bit-exact against the pinned oracle and
the reference's golden vectors."""
from __future__ import annotations

from random import Random

import numpy as np
import pytest

from no_three_in_line_b200 import gpu, state

pytestmark = pytest.mark.gpu


def test_c1_n20_scores_and_badness(golden, cuda):
    c1 = golden("c1_n20.npz")
    s, b = gpu.score_population_gpu(c1["p"], c1["q"], badness=True)
    assert np.array_equal(s, c1["E"]) and np.array_equal(b, c1["badness"])
    cols = state.pq_to_columns(c1["p"], c1["q"])
    assert np.array_equal(gpu.score_columns_gpu(cols), c1["E"])
    s2, b2 = gpu.score_slope_gpu(cols)
    assert np.array_equal(s2, c1["E"]) and np.array_equal(b2, c1["badness"])
    chk = gpu.score_checked_gpu(cols)
    assert chk.mismatches == 0 and chk.error_word == 0
    assert np.array_equal(chk.scores, c1["E"]) and np.array_equal(chk.badness, c1["badness"])


def test_c2_n75_population(golden, cuda):
    c2 = golden("c2_n75.npz")
    p, q = state.seeded_population(75, 4096)
    s = gpu.score_population_gpu(p, q)
    assert np.array_equal(s, c2["E"])
    s, b = gpu.score_population_gpu(p, q, badness=True)
    assert np.array_equal(s, c2["E"]) and np.array_equal(b, c2["badness"].astype(np.int32))
    chk = gpu.score_checked_gpu(state.pq_to_columns(p, q))
    assert chk.mismatches == 0 and chk.error_word == 0
    assert np.array_equal(chk.scores, c2["E"]) and np.array_equal(chk.badness, c2["badness"].astype(np.int32))


def test_e10_fixture(golden, cuda):
    e = golden("e10.npz")
    p, q = e["p"][None].astype(np.int32), e["q"][None].astype(np.int32)
    s, b = gpu.score_population_gpu(p, q, badness=True)
    assert int(s[0]) == 10 and np.array_equal(b[0], e["badness"])
    chk = gpu.score_checked_gpu(state.pq_to_columns(p, q))
    assert int(chk.scores[0]) == 10 and int(chk.badness.sum()) == 30


@pytest.mark.parametrize("n", [2, 3, 4, 5, 7, 16, 31, 32, 33, 48, 63, 64, 65, 74, 75])
def test_every_size_matches_oracle(n, oracle, cuda):
    rng = Random(1000 + n)
    B = 37
    p = np.empty((B, n), np.int32)
    q = np.empty((B, n), np.int32)
    for i in range(B):
        st = state.random_state(n, rng)
        p[i], q[i] = st.P, st.Q
    ref_s, ref_b = oracle.score_population(p, q, badness=True, threads=0)
    s, b = gpu.score_population_gpu(p, q, badness=True)
    assert np.array_equal(s, ref_s) and np.array_equal(b, ref_b)
    cols = state.pq_to_columns(p, q)
    s2, b2 = gpu.score_slope_gpu(cols)
    assert np.array_equal(s2, ref_s) and np.array_equal(b2, ref_b)
    chk = gpu.score_checked_gpu(cols)
    assert np.array_equal(chk.scores, ref_s) and chk.mismatches == 0
    fwd = gpu.score_checked_gpu(cols, badness=False)  # forward slope count of E
    assert np.array_equal(fwd.scores, ref_s) and fwd.mismatches == 0 and fwd.badness is None


def test_degenerate_dense_collinear_states(oracle, cuda):
    """Highly collinear states (diagonal-like permutations) stress the count."""
    n = 75
    p = np.stack([np.arange(n), (np.arange(n) * 2) % n, (np.arange(n) * 3) % n]).astype(np.int32)
    q = np.stack([(np.arange(n) + 1) % n, (np.arange(n) * 2 + 1) % n, (np.arange(n) * 3 + 5) % n]).astype(np.int32)
    ref_s, ref_b = oracle.score_population(p, q, badness=True, threads=0)
    s, b = gpu.score_population_gpu(p, q, badness=True)
    assert np.array_equal(s, ref_s) and np.array_equal(b, ref_b)
    chk = gpu.score_checked_gpu(state.pq_to_columns(p, q))
    assert np.array_equal(chk.scores, ref_s) and np.array_equal(chk.badness, ref_b) and chk.mismatches == 0
    fwd = gpu.score_checked_gpu(state.pq_to_columns(p, q), badness=False)
    assert np.array_equal(fwd.scores, ref_s) and fwd.mismatches == 0


def test_long_lines_mixed_into_a_population(oracle, cuda):
    """States with 16 or more points on one line through a point (the slope
    count's 4-bit counters overflow and the state is recounted with 8-bit
    counters over each half of the directions) spread through a batch of random
    states, so that warps of one CTA take both paths."""
    n = 75
    pr, qr = state.seeded_population(n, 600)
    r = np.arange(n)
    dense_p = np.stack([r, r, (2 * r) % n, r, (r + 7) % n]).astype(np.int32)
    dense_q = np.stack([(r + 1) % n, (r + 37) % n, (2 * r + 1) % n, (n - 1 - r + (r == (n - 1) // 2)) % n,
                        (r + 8) % n]).astype(np.int32)
    keep = [k for k in range(len(dense_p)) if np.all(dense_p[k] != dense_q[k])
            and len(set(dense_q[k].tolist())) == n]
    p, q = pr.copy(), qr.copy()
    slots = [3, 97, 250, 251, 599][:len(keep)]
    for slot, k in zip(slots, keep):
        p[slot], q[slot] = dense_p[k], dense_q[k]
    ref_s, ref_b = oracle.score_population(p, q, badness=True, threads=0)
    cols = state.pq_to_columns(p, q)
    s2, b2 = gpu.score_slope_gpu(cols)
    assert np.array_equal(s2, ref_s) and np.array_equal(b2, ref_b)
    chk = gpu.score_checked_gpu(cols)
    assert np.array_equal(chk.scores, ref_s) and np.array_equal(chk.badness, ref_b) and chk.mismatches == 0
    fwd = gpu.score_checked_gpu(cols, badness=False)  # the forward count's own overflow path
    assert np.array_equal(fwd.scores, ref_s) and fwd.mismatches == 0
    assert max(ref_s[slot] for slot in slots) > 10000  # a line of 74 or 75 points is among them


def test_empty_batch_and_shape_errors(cuda):
    z = np.zeros((0, 10), np.int32)
    assert gpu.score_population_gpu(z, z).shape == (0,)
    with pytest.raises(ValueError):
        gpu.score_population_gpu(np.zeros((2, 5), np.int32), np.zeros((2, 6), np.int32))
    with pytest.raises(ValueError):
        gpu.score_population_gpu(np.zeros((2, 76), np.int32), np.zeros((2, 76), np.int32))


def test_checked_scoring_flags_invalid_states(cuda):
    """Out-of-range columns and duplicate points are caught by the kernel's own
    checks (it clamps its reads) and reported, never scored."""
    p, q = state.seeded_population(20, 4)
    cols = state.pq_to_columns(p, q)
    cols[1, 7] = 25          # column outside [0, 20)
    cols[2, 9] = cols[2, 8]  # duplicate point in row 4
    for badness in (True, False):
        chk = gpu.score_checked_gpu(cols, raise_on_mismatch=False, badness=badness)
        assert chk.error_word & 1 and chk.error_word & 2
        assert chk.mismatches == 2 and chk.scores[1] == -1 and chk.scores[2] == -1
    with pytest.raises(AssertionError):
        gpu.score_checked_gpu(cols)


def test_device_tensors_stay_on_device(cuda):
    import torch

    p, q = state.seeded_population(75, 8)
    dp = torch.from_numpy(p).cuda()
    dq = torch.from_numpy(q).cuda()
    out = gpu.score_population_gpu(dp, dq)
    assert out.is_cuda and out.dtype == torch.int32
    assert np.array_equal(out.cpu().numpy(), gpu.score_population_gpu(p, q))
