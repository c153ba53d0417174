"""(b) Exact swap deltas on the GPU, bit-exact against the reference's golden
outputs and the pinned oracle."""
from __future__ import annotations

from random import Random

import numpy as np
import pytest

from no_three_in_line_b200 import accelerated, gpu_delta, state

pytestmark = pytest.mark.gpu
SENT = gpu_delta.SENTINEL


def test_reference_two_switch_pins(golden, cuda):
    """Outputs of accelerated.evaluate_two_switches (tests/test_delta.py seeds)."""
    d = golden("delta_pins.json")
    for rec in d["two_switches"]:
        out = accelerated.evaluate_two_switches(np.array(rec["p"]), np.array(rec["q"]), rec["u"], rec["score"],
                                                np.array(rec["badness"]))
        assert out.tolist() == rec["out"]
        plug = gpu_delta.score_two_switches_gpu(rec["p"], rec["q"], rec["u"], rec["score"], rec["badness"])
        ref = np.array(rec["out"])
        legal = ref < (1 << 59)
        assert np.array_equal(plug >= (1 << 29), ~legal) and np.array_equal(plug[legal], ref[legal])
    p, q = state.seeded_population(75, 8)
    for rec in d["two_switches_n75"]:
        b = rec["state"]
        s, bad = accelerated.score_and_badness(p[b], q[b])
        assert s == rec["score"]
        out = accelerated.evaluate_two_switches(p[b], q[b], rec["u"], s, bad)
        assert out.tolist() == rec["out"]


def test_reference_transposition_pins(golden, cuda):
    d = golden("delta_pins.json")
    for rec in d["transpositions"]:
        out = accelerated.evaluate_transpositions(np.array(rec["p"]), np.array(rec["q"]), rec["layer"], rec["row"],
                                                  rec["score"], np.array(rec["badness"]))
        assert out.tolist() == rec["out"]


def _replay_rounds(swaps):
    """Split the swap sequence into rounds holding at most one swap per state,
    preserving each state's order."""
    per_state: dict[int, list[int]] = {}
    for t, (b, _u, _v) in enumerate(swaps):
        per_state.setdefault(int(b), []).append(t)
    rounds = []
    depth = max(len(v) for v in per_state.values())
    for r in range(depth):
        rounds.append([ts[r] for ts in per_state.values() if len(ts) > r])
    return rounds


@pytest.mark.parametrize("pairs", [False, True])
def test_c1_ten_thousand_swaps_against_full_recompute(golden, cuda, pairs):
    """The 10^4 seeded n=20 swaps: each incremental delta (and badness delta)
    equals the reference's full-recompute delta; the states end where the
    reference's did."""
    import torch

    c1 = golden("c1_n20.npz")
    cols = torch.from_numpy(state.pq_to_columns(c1["p"], c1["q"])).cuda()
    bad = torch.from_numpy(c1["badness"].astype(np.int32)).cuda()
    swaps = c1["swaps"]
    for rnd in _replay_rounds(swaps):
        idx = np.asarray(rnd)
        moves = torch.from_numpy(swaps[idx].astype(np.int32)).cuda()
        dE, dbad = gpu_delta.swap_deltas(cols, moves, badness=True, pairs=pairs)
        dE = dE.cpu().numpy()
        valid = c1["valid"][idx].astype(bool)
        assert np.array_equal(dE == SENT, ~valid)
        assert np.array_equal(dE[valid], c1["dE"][idx][valid])
        db = dbad.cpu().numpy().astype(np.int64)
        assert np.array_equal((db[valid] ** 2).sum(axis=1), c1["dbad_sumsq"][idx][valid])
        for k in np.nonzero(valid)[0]:
            b, u, v = (int(x) for x in swaps[idx[k]])
            cu, cv = cols[b, u].item(), cols[b, v].item()
            cols[b, u], cols[b, v] = cv, cu
            bad[b] += dbad[k]
    assert np.array_equal(cols.cpu().numpy(), c1["final_cols"].astype(np.int16))
    from no_three_in_line_b200 import gpu

    s, b = gpu.score_columns_gpu(cols, badness=True)
    assert np.array_equal(s.cpu().numpy(), c1["final_E"])
    assert torch.equal(b, bad)


def test_n75_moves_match_oracle_and_pairs_kernel(oracle, cuda):
    """4096 random n=75 moves: direction-class kernel == literal pair kernel ==
    the oracle's restatement of tempering.py:68-89, with badness deltas."""
    p, q = state.seeded_population(75, 256)
    cols = state.pq_to_columns(p, q)
    rng = Random(31337)
    moves = np.array([[rng.randrange(256), rng.randrange(150), rng.randrange(150)] for _ in range(4096)], np.int32)
    dE, db = gpu_delta.swap_deltas(cols, moves, badness=True)
    dE2, db2 = gpu_delta.swap_deltas(cols, moves, badness=True, pairs=True)
    assert np.array_equal(dE, dE2) and np.array_equal(db, db2)
    for k in range(0, 4096, 7):
        b, u, v = moves[k]
        ok, d, dbad = oracle.walk_delta(cols[b], u, v)
        if not ok:
            assert dE[k] == SENT
            continue
        assert dE[k] == d and np.array_equal(db[k], dbad)
        assert int(db[k].sum()) == 3 * d


def test_partner_scores_batched_match_oracle(oracle, cuda):
    import torch

    p, q = state.seeded_population(75, 16)
    s, bad = accelerated.score_and_badness(p, q)
    cols = torch.from_numpy(state.pq_to_columns(p, q)).cuda()
    anchors = torch.tensor([[b, (37 * b + 11) % 150] for b in range(16)], dtype=torch.int32).cuda()
    out = gpu_delta.two_switch_scores(cols, torch.from_numpy(bad.astype(np.int32)).cuda(),
                                      torch.from_numpy(s).cuda(), anchors).cpu().numpy()
    for b in range(16):
        u = (37 * b + 11) % 150
        ref = oracle.two_switches(p[b], q[b], u, int(s[b]), bad[b])
        legal = ref < (1 << 59)
        assert np.array_equal(out[b] >= SENT, ~legal) and np.array_equal(out[b][legal], ref[legal])


def test_illegal_and_out_of_range_moves(cuda):
    p, q = state.seeded_population(20, 2)
    cols = state.pq_to_columns(p, q)
    moves = np.array([[0, 4, 5],      # same row
                      [0, 3, 3],      # same slot
                      [5, 0, 2],      # state out of range
                      [1, 0, 99],     # slot out of range
                      [0, 0, 2]], np.int32)
    dE = gpu_delta.swap_deltas(cols, moves)
    assert (dE[:4] == SENT).all()
    assert gpu_delta.swap_deltas(cols, np.zeros((0, 3), np.int32)).shape == (0,)
