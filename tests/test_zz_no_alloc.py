"""The allocation-free training entry point, n3_mlp_train_noalloc.

It is for callers that cannot call cudaMalloc (a host application whose own
allocator owns all device memory, or a plug-in whose host forbids foreign
allocations): it keeps the batch activations and the gradient in a static
device array inside libn3.so instead of caller-provided scratch.  These tests
call it through the C ABI and compare it with n3_mlp_train, which takes the
same step with caller-allocated scratch, over two consecutive calls.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test.  It also passes on its own in a
fresh process.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from no_three_in_line_b200 import _lib, learned, state, tempering

pytestmark = pytest.mark.gpu

MAX_BATCH = 512


def _entry():
    f = _lib.lib().n3_mlp_train_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(learned.N3Mlp), ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_uint64,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return f


def _proposal(batch):
    p, q = state.seeded_population(75, 64)
    temps = np.tile(tempering.geometric_ladder(0.05, 5.0, 16), 4)
    ch = tempering.TemperingChains(state.pq_to_columns(p, q), temps, 31, ladder_size=16)
    lp = learned.LearnedProposal(ch, seed=31, ring_capacity=1 << 14, batch=batch)
    for _ in range(24):  # fill the ring buffer with exact (features, dE) tuples
        lp.step()
    return lp


def _snapshot(lp):
    return {k: getattr(lp, k).clone() for k in ("params", "adam_m", "adam_v", "counters")}


def _restore(lp, snap):
    for k, v in snap.items():
        getattr(lp, k).copy_(v)
    _lib.check(_lib.lib().n3_mlp_pack(ctypes.byref(lp._desc), _lib.stream_ptr()), "n3_mlp_pack")


def _noalloc_train(lp):
    rc = _entry()(ctypes.byref(lp._desc), lp.ch.cols.shape[0], lp.batch, lp.lr, lp.seed ^ 0x5A5A5A5A,
                  lp.adam_m.data_ptr(), lp.adam_v.data_ptr(), _lib.stream_ptr())
    _lib.check(rc, "n3_mlp_train_noalloc")


@pytest.mark.parametrize("batch", [256, MAX_BATCH])
def test_noalloc_training_matches_caller_scratch_over_two_calls(cuda, batch):
    import torch

    lp = _proposal(batch)
    # Both entry points reduce the gradient with float atomics, so its last bits
    # vary between calls.  A non-zero second moment keeps Adam's step linear in
    # the gradient (its first step from v = 0 is sign-like), so equal inputs give
    # outputs equal within the usual fp32 tolerance.
    lp.adam_v.fill_(1e-2)
    snap = _snapshot(lp)
    ref = []
    for _ in range(2):  # the existing entry point, caller-allocated scratch
        lp.train()
        torch.cuda.synchronize()
        ref.append((lp.params.cpu().numpy().copy(), float(lp.loss.item()), lp.w2_img.cpu().numpy().copy()))
    _restore(lp, snap)
    for k in range(2):  # the allocation-free entry point, same inputs
        _noalloc_train(lp)
        torch.cuda.synchronize()
        p, loss, img = lp.params.cpu().numpy(), float(lp.loss.item()), lp.w2_img.cpu().numpy()
        assert np.allclose(p, ref[k][0], rtol=1e-5, atol=1e-6), k
        assert abs(loss - ref[k][1]) <= 1e-4 * (1.0 + abs(ref[k][1])), k
        # the packed bf16 image follows the updated parameters
        assert np.mean(img != ref[k][2]) < 1e-3, k
    assert int(lp.counters[1].item()) == int(snap["counters"][1].item()) + 2


def test_noalloc_rejects_batches_beyond_its_static_capacity(cuda):
    lp = _proposal(256)
    lp.batch = MAX_BATCH + 1
    rc = _entry()(ctypes.byref(lp._desc), lp.ch.cols.shape[0], lp.batch, lp.lr, 1, lp.adam_m.data_ptr(),
                  lp.adam_v.data_ptr(), _lib.stream_ptr())
    assert rc == _lib.N3_ERR_RANGE
    assert str(MAX_BATCH) in _lib.last_error()
