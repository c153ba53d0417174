"""Failure detection without GPU faults: mistakes are planted on the host (in
device buffers written from the host, or in checkpoint files) and must be
caught by the device audit or the loaders."""
from __future__ import annotations

import numpy as np
import pytest

from no_three_in_line_b200 import gpu, state, tempering

pytestmark = pytest.mark.gpu


def _chains(seed=5):
    p, q = state.seeded_population(30, 16)
    temps = np.tile(tempering.geometric_ladder(0.1, 4.0, 8), 2)
    ch = tempering.TemperingChains(state.pq_to_columns(p, q), temps, seed, ladder_size=8)
    ch.run(20, exchange_every=10, graph=False)
    return ch


def test_audit_catches_a_wrong_energy(cuda):
    ch = _chains()
    ch.validate()
    ch.energy[3] += 1
    with pytest.raises(AssertionError):
        ch.validate()


def test_audit_catches_a_wrong_badness(cuda):
    ch = _chains()
    ch.badness_dev[5, 7] += 2
    with pytest.raises(AssertionError):
        ch.validate()


def test_audit_catches_a_moved_point(cuda):
    """A column changed behind the chains' back (energy no longer matches)."""
    ch = _chains()
    cols = ch.cols[2, :60].cpu().numpy()
    # swap two columns between rows so that the state stays a legal 2-factor
    for u in range(60):
        for v in range(u + 1, 60):
            if state.legal_swap(cols, u, v):
                c2 = cols.copy()
                c2[u], c2[v] = c2[v], c2[u]
                if gpu.score_columns_gpu(c2[None])[0] != gpu.score_columns_gpu(cols[None])[0]:
                    ch.cols[2, u], ch.cols[2, v] = int(cols[v]), int(cols[u])
                    with pytest.raises(AssertionError):
                        ch.validate()
                    return
    pytest.fail("no energy-changing swap found")


def test_truncated_checkpoint_is_rejected(cuda, tmp_path):
    ch = _chains()
    path = tmp_path / "ck.npz"
    ch.save(path)
    data = path.read_bytes()
    bad = tmp_path / "bad.npz"
    bad.write_bytes(data[: len(data) // 2])
    with pytest.raises(Exception):
        tempering.TemperingChains.restore(bad)


def test_checkpoint_with_corrupted_state_fails_validation(cuda, tmp_path):
    ch = _chains()
    path = tmp_path / "ck.npz"
    ch.save(path)
    with np.load(path) as z:
        arrays = {k: z[k] for k in z.files}
    arrays["energy"] = arrays["energy"] + 1
    np.savez(tmp_path / "bad.npz", **arrays)
    with pytest.raises(AssertionError):
        tempering.TemperingChains.restore(tmp_path / "bad.npz")


def test_bounded_device_wait_expires_without_hanging(cuda):
    """A device wait that can never complete gives up after its bound, reports
    it (TimeoutError on the host) and leaves the context usable."""
    import time

    from no_three_in_line_b200 import learned

    t0 = time.perf_counter()
    for tries in (1, 300, 1 << 16):
        with pytest.raises(TimeoutError):
            learned.check_bounded_wait(tries)
    assert time.perf_counter() - t0 < 60
    p, q = state.seeded_population(20, 4)
    assert gpu.score_population_gpu(p, q).shape == (4,)  # the context still works
    with pytest.raises(ValueError):
        learned.check_bounded_wait(0)
