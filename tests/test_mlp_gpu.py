"""(d) Learned proposal: tcgen05 MLP inference against an fp64 reference of
the same bf16-rounded network, training gradients against torch autograd,
and exact energies through learned steps."""
from __future__ import annotations

import numpy as np
import pytest

from no_three_in_line_b200 import learned, state, tempering

pytestmark = pytest.mark.gpu


def bf16(x):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def inter16_offset(row, k):
    return (row >> 3) * 256 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2


def make(n=75, chains=32, L=16, seed=4):
    p, q = state.seeded_population(n, chains)
    temps = np.tile(tempering.geometric_ladder(0.05, 5.0, L), chains // L)
    ch = tempering.TemperingChains(state.pq_to_columns(p, q), temps, seed, ladder_size=L)
    return ch


def features(cols, bad, n, u, v):
    s = [u, v, u ^ 1, v ^ 1]
    return np.array([bad[x] / 16 for x in s] + [(x >> 1) / n for x in s] + [cols[x] / n for x in s])


def test_inference_matches_bf16_reference(cuda):
    # 480 chain tiles: more than one tile per SM, so the kernel's prefetch /
    # overlapped-MMA pipeline runs several iterations per CTA
    ch = make(chains=480, L=16)
    lp = learned.LearnedProposal(ch, seed=9, ring_capacity=1 << 12, batch=256)
    lp.propose_scores()
    P = lp.params.cpu().numpy().astype(np.float64)
    W1 = P[learned.O_W1:learned.O_B1].reshape(256, 192)
    b1 = P[learned.O_B1:learned.O_W2]
    W2 = P[learned.O_W2:learned.O_B2].reshape(256, 256)
    b2 = P[learned.O_B2:learned.O_W3]
    w3 = P[learned.O_W3:learned.O_B3]
    b3 = P[learned.O_B3]
    cols = ch.cols.cpu().numpy()
    bad = ch.badness_dev.cpu().numpy()
    cand = lp.cand.cpu().numpy()
    pred = lp.pred.cpu().numpy()
    img = lp.a1_img.cpu().numpy().reshape(-1, 4096)
    c1_dev = lp.c1.cpu().numpy()
    for c in list(range(0, cols.shape[0], 13)) + [cols.shape[0] - 1]:
        x_chain = bad[c] / 16.0
        # the chain part runs on the tensor cores: bf16 operands, fp32 accumulation
        c1 = b1 + bf16(W1[:, 12:162]) @ bf16(x_chain)
        assert np.allclose(c1_dev[c], c1, rtol=1e-5, atol=1e-5)
        F = np.zeros((128, 16))
        F[:, 12:14] = 1.0  # constant columns that carry the chain part (hi, lo) into layer 1
        for j in range(128):
            u, v = cand[c, j] & 0xFF, (cand[c, j] >> 8) & 0xFF
            F[j, :12] = features(cols[c], bad[c], 75, u, v)
            got = np.array([img[c, inter16_offset(j, k):inter16_offset(j, k) + 2].view(np.uint16)[0]
                            for k in range(16)], np.uint32)
            assert np.array_equal((got << 16).view(np.float32).astype(np.float64), bf16(F[j]))
        h1 = np.maximum(bf16(F) @ bf16(np.pad(W1[:, :12], ((0, 0), (0, 4)))).T + c1, 0)
        h2 = np.maximum(bf16(h1) @ bf16(W2).T + b2, 0)
        ref = (h2 @ w3 + b3) * 16.0
        assert np.allclose(pred[c], ref, rtol=1e-2, atol=5e-2), (c, np.abs(pred[c] - ref).max())


def test_training_gradients_match_autograd(cuda):
    """The five training GEMMs run on the tensor cores with bf16 operands and
    fp32 accumulation: each is checked against an fp64 product of the same
    bf16-rounded device operands (only the summation order differs); the head,
    bias sums and Adam in fp32 against fp64 formulas; and the whole gradient
    against fp64 autograd of the unrounded network within the bf16 tolerance."""
    import torch

    ch = make(chains=64, L=16)
    lp = learned.LearnedProposal(ch, seed=3, ring_capacity=1 << 14, batch=256, lr=1e-3)
    for _ in range(20):
        lp.step()
    p0 = lp.params.clone()
    lp.train()
    torch.cuda.synchronize()
    B, H = lp.batch, 256
    sc = lp.scratch.double().cpu().numpy()
    off = 0

    def take(size, shape):
        nonlocal off
        a = sc[off:off + size].reshape(shape)
        off += size
        return a

    X, y, d = take(B * 192, (B, 192)), take(B, (B,)), take(B, (B,))
    Z1, H1, Z2, H2, dZ2, dZ1 = (take(B * H, (B, H)) for _ in range(6))
    P = p0.double().cpu().numpy()
    W1 = P[learned.O_W1:learned.O_B1].reshape(H, 192)
    b1 = P[learned.O_B1:learned.O_W2]
    W2 = P[learned.O_W2:learned.O_B2].reshape(H, H)
    b2 = P[learned.O_B2:learned.O_W3]
    w3 = P[learned.O_W3:learned.O_B3]
    g = lp.grads.double().cpu().numpy()
    gW1 = g[learned.O_W1:learned.O_B1].reshape(H, 192)
    gW2 = g[learned.O_W2:learned.O_B2].reshape(H, H)

    def close(got, want, rtol=2e-4):
        scale = max(np.abs(want).max(), 1e-30)
        assert np.allclose(got, want, rtol=rtol, atol=rtol * scale), np.abs(got - want).max() / scale

    # tensor-core GEMMs against fp64 on the same bf16-rounded operands
    close(Z1, bf16(X) @ bf16(W1).T + b1)
    assert np.array_equal(H1, np.maximum(Z1, 0))
    close(Z2, bf16(H1) @ bf16(W2).T + b2)
    assert np.array_equal(H2, np.maximum(Z2, 0))
    close(gW2, bf16(dZ2).T @ bf16(H1))
    close(dZ1, (bf16(dZ2) @ bf16(W2)) * (Z1 > 0))
    close(gW1, bf16(dZ1).T @ bf16(X))
    # fp32 parts: bias sums and the head's gradients from the device activations
    close(g[learned.O_B1:learned.O_W2], dZ1.sum(0), rtol=1e-5)
    close(g[learned.O_B2:learned.O_W3], dZ2.sum(0), rtol=1e-5)
    close(g[learned.O_W3:learned.O_B3], H2.T @ d, rtol=1e-5)
    assert abs(g[learned.O_B3] - d.sum()) <= 1e-5 * (1 + np.abs(d).sum())
    close(dZ2, d[:, None] * w3[None, :] * (Z2 > 0), rtol=1e-5)
    # the whole gradient against autograd of the unrounded fp64 network
    Pt = p0.double().cpu().requires_grad_(True)
    tW1 = Pt[learned.O_W1:learned.O_B1].view(H, 192)
    tb1 = Pt[learned.O_B1:learned.O_W2]
    tW2 = Pt[learned.O_W2:learned.O_B2].view(H, H)
    tb2 = Pt[learned.O_B2:learned.O_W3]
    tw3 = Pt[learned.O_W3:learned.O_B3]
    tb3 = Pt[learned.O_B3]
    Xt, yt = torch.from_numpy(X), torch.from_numpy(y)
    h1 = torch.relu(Xt @ tW1.T + tb1)
    h2 = torch.relu(h1 @ tW2.T + tb2)
    out = h2 @ tw3 + tb3
    loss = ((out - yt) ** 2).mean()
    loss.backward()
    g_ref = Pt.grad.numpy()
    for lo, hi in ((learned.O_W1, learned.O_B1), (learned.O_W2, learned.O_B2), (learned.O_W3, learned.O_B3)):
        err = np.linalg.norm(g[lo:hi] - g_ref[lo:hi]) / max(np.linalg.norm(g_ref[lo:hi]), 1e-30)
        assert err < 3e-2, (lo, err)
    # the applied update is Adam's first step from these gradients
    m = 0.1 * g
    v = 0.001 * g * g
    p1_ref = P - 1e-3 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    assert np.allclose(lp.params.cpu().numpy(), p1_ref, rtol=1e-5, atol=1e-6)
    assert abs(float(lp.loss.item()) / B - float(loss)) < 2e-2 * (1 + float(loss))


def test_learned_steps_keep_energies_exact(cuda):
    ch = make(chains=64, L=16, seed=12)
    e0 = int(ch.energy.min().item())
    lp = learned.LearnedProposal(ch, seed=12, ring_capacity=1 << 16, batch=512)
    res = lp.run(600, exchange_every=300, train_every=10, block=50)
    ch.validate()
    assert int(ch.error_word.item()) == 0 and int(lp.error_word.item()) == 0
    st = lp.read_stats()
    assert st.proposals >= 64 * 600 and st.accepted > 0 and np.isfinite(st.mae)
    assert res.best < e0
    from no_three_in_line_b200 import gpu

    s = gpu.score_columns_gpu(ch.best_columns.cpu().numpy())
    assert np.array_equal(s, ch.best_energy.cpu().numpy())


def test_graph_and_eager_agree(cuda):
    runs = []
    for graph in (False, True):
        ch = make(chains=32, L=16, seed=21)
        lp = learned.LearnedProposal(ch, seed=21, ring_capacity=1 << 14, batch=256)
        lp.run(100, exchange_every=100, train_every=0, block=50, graph=graph, warm=False)
        runs.append((ch.cols.cpu().numpy(), ch.energy.cpu().numpy(), lp.params.cpu().numpy()))
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])


def test_several_moves_per_step_keep_energies_exact(cuda):
    """moves=4: four draws without replacement per scoring pass, each re-checked
    for legality on the current state and accepted by its exact delta."""
    ch = make(chains=64, L=16, seed=8)
    lp = learned.LearnedProposal(ch, seed=8, ring_capacity=1 << 16, batch=512, moves=4)
    lp.run(200, exchange_every=200, train_every=10, block=50)
    ch.validate()
    assert int(ch.error_word.item()) == 0
    st = lp.read_stats()
    assert st.proposals > 64 * 201 * 3 and st.accepted > 0


@pytest.mark.parametrize("moves", [1, 4])
def test_team_width_does_not_change_the_learned_run(cuda, moves):
    """One warp or a team of two per chain: the same draws, the same exact
    moves, the same ring-buffer tuples, bit for bit (64 chains: the last CTA
    of 14 chains is partly empty)."""
    runs = []
    for tpc in (32, 64):
        ch = make(chains=64, L=16, seed=31)
        lp = learned.LearnedProposal(ch, seed=31, ring_capacity=1 << 14, batch=256, moves=moves,
                                     threads_per_chain=tpc)
        lp.run(100, exchange_every=50, train_every=0, block=50, graph=tpc == 64, warm=False)
        ch.validate()
        assert int(ch.error_word.item()) == 0
        runs.append([x.cpu().numpy() for x in (ch.cols, ch.energy, ch.best_energy, ch.best_cols, ch.badness_dev,
                                               ch.accepted_dev, lp.rb_feat, lp.rb_bad, lp.rb_dE)])
        assert int(lp.read_stats().accepted) > 0
    for a, b in zip(*runs):
        assert np.array_equal(a, b)

