"""Host logic of the exhaustive beam (CPU): the candidate order the device
kernels index by, checked against the reference's enumeration
(candidate_descriptors, gpu_exhaustive_beam.py:67-82)."""
from __future__ import annotations

import numpy as np

from no_three_in_line_b200 import gpu_exhaustive_beam as gx


def device_offsets(badness, global_anchors):
    """The anchors_kernel rule: anchor u of rank r among its elite's anchors
    keeps m - 2 - (r - [u odd and u - 1 an anchor]) partners; candidates follow
    elite by elite, anchor by anchor."""
    E, m = badness.shape
    out = []
    for p in range(E):
        flags = [global_anchors or badness[p, s] > 0 for s in range(m)]
        rank = 0
        for u in range(m):
            if not flags[u]:
                continue
            cnt = m - 2 - (rank - (1 if (u & 1) and flags[u - 1] else 0))
            out.append((p, u, cnt))
            rank += 1
    return out


def test_candidate_offsets_match_the_reference_enumeration():
    rng = np.random.default_rng(4)
    for trial in range(40):
        E, n = int(rng.integers(1, 6)), int(rng.integers(3, 12))
        bad = rng.integers(0, 3, (E, 2 * n)) * (rng.random((E, 2 * n)) < 0.5)
        for glob in (False, True):
            desc = gx.candidate_descriptors(bad, global_anchors=glob)
            offs = device_offsets(bad, glob)
            assert sum(c for _, _, c in offs) == len(desc)
            pos = 0
            for p, u, cnt in offs:
                block = desc[pos:pos + cnt]
                assert np.all(block[:, 0] == p) and np.all(block[:, 1] == u)
                # partners in ascending order, never u's row, never an earlier anchor
                vs = block[:, 2]
                assert np.all(np.diff(vs) > 0) and np.all((vs >> 1) != (u >> 1))
                pos += cnt


def test_signature_is_order_free_per_row():
    p = np.array([3, 0, 1, 2])
    q = np.array([1, 2, 3, 0])
    assert gx._signature(p, q) == gx._signature(q, p)
    assert gx._signature(p, q) != gx._signature(p[::-1].copy(), q[::-1].copy())
