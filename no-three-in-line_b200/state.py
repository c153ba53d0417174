"""Two-points-per-row/column state model (host side).

Mirrors the reference's ``no_three_75.state`` module
(src/no_three_75/state.py:10-95): a state of an n x n grid holds 2n points,
exactly two per row and per column, stored as two column arrays P and Q with
``P[r] != Q[r]``.  The device kernels use the reference's interleaved slot
layout (src/no_three_75/accelerated.py:18-24, src/no_three_75/tempering.py:38):

    slot s = 2*r + layer,  row(s) = s >> 1,  cols[2r] = P[r], cols[2r+1] = Q[r]

so a population is an ``int16[B, 2n]`` array of columns with rows implicit.
After a cross-layer column swap the two layers need not be permutations any
more; the point set is still a row/column 2-factor and
:func:`points_to_permutations` recovers a P/Q pair, as the reference does in
``TemperingChains.to_state`` (src/no_three_75/tempering.py:155-156).
"""
from __future__ import annotations

from dataclasses import dataclass
from random import Random

import numpy as np

Point = tuple[int, int]

#: Largest grid the device kernels accept (150 slots); the reference's
#: shared-memory kernels have the same bound (src/no_three_75/tempering.py:39,124).
MAX_N = 75


@dataclass(frozen=True)
class PairPermutations:
    """P/Q state; same fields and checks as src/no_three_75/state.py:10-44."""

    P: tuple[int, ...]
    Q: tuple[int, ...]

    @property
    def n(self) -> int:
        return len(self.P)

    def validate(self) -> None:
        n = self.n
        everything = set(range(n))
        if len(self.Q) != n:
            raise ValueError("P and Q have different lengths")
        if set(self.P) != everything:
            raise ValueError("P is not a permutation")
        if set(self.Q) != everything:
            raise ValueError("Q is not a permutation")
        clashes = [r for r in range(n) if self.P[r] == self.Q[r]]
        if clashes:
            raise ValueError(f"P/Q duplicate edges at rows {clashes}")

    def points(self) -> list[Point]:
        self.validate()
        return sorted([(r, self.P[r]) for r in range(self.n)] + [(r, self.Q[r]) for r in range(self.n)])

    def swapped(self, layer: int, row_a: int, row_b: int) -> "PairPermutations":
        """Same-layer transposition of rows a and b (state.py:35-44)."""
        if layer not in (0, 1):
            raise ValueError("layer must be 0 (P) or 1 (Q)")
        p, q = list(self.P), list(self.Q)
        target = p if layer == 0 else q
        target[row_a], target[row_b] = target[row_b], target[row_a]
        moved = PairPermutations(tuple(p), tuple(q))
        moved.validate()
        return moved

    def columns(self) -> np.ndarray:
        """Slot-layout columns, int16[2n]."""
        return pq_to_columns(np.asarray(self.P), np.asarray(self.Q))


def random_state(n: int, rng: Random) -> PairPermutations:
    """Seeded state exactly as src/no_three_75/state.py:88-95: shuffle P once,
    then reshuffle Q until it differs from P in every row.  The sequence of
    ``rng`` calls is the same, so ``random_state(n, Random(s))`` reproduces the
    reference's state for every seed ``s``."""
    p = list(range(n))
    q = list(range(n))
    rng.shuffle(p)
    while True:
        rng.shuffle(q)
        if all(a != b for a, b in zip(p, q)):
            return PairPermutations(tuple(p), tuple(q))


def seeded_population(n: int, count: int, base_seed: int = 91001) -> tuple[np.ndarray, np.ndarray]:
    """P, Q int32[count, n] with state i drawn by ``random_state(n, Random(base_seed + i))``
    (the population convention of the reference's gpu-benchmark, cli.py:203-204)."""
    p = np.empty((count, n), dtype=np.int32)
    q = np.empty((count, n), dtype=np.int32)
    for i in range(count):
        s = random_state(n, Random(base_seed + i))
        p[i] = s.P
        q[i] = s.Q
    return p, q


def pq_to_columns(p: np.ndarray, q: np.ndarray) -> np.ndarray:
    """Interleave P/Q ([..., n]) into slot columns ([..., 2n]) as int16."""
    p = np.asarray(p)
    q = np.asarray(q)
    if p.shape != q.shape or p.ndim < 1:
        raise ValueError("P and Q must have the same shape")
    out = np.empty(p.shape[:-1] + (2 * p.shape[-1],), dtype=np.int16)
    out[..., 0::2] = p
    out[..., 1::2] = q
    return out


def columns_to_pq(columns: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Inverse of :func:`pq_to_columns` (int32 layers)."""
    c = np.asarray(columns)
    if c.shape[-1] % 2:
        raise ValueError("slot columns must have an even last dimension")
    return c[..., 0::2].astype(np.int32), c[..., 1::2].astype(np.int32)


def columns_to_points(columns: np.ndarray) -> list[Point]:
    """Sorted (row, column) points of one slot-layout state."""
    c = np.asarray(columns).reshape(-1)
    return sorted((i // 2, int(v)) for i, v in enumerate(c))


def points_to_permutations(points: list[Point], n: int) -> PairPermutations:
    """Split a row/column 2-factor into P/Q (src/no_three_75/state.py:47-85).

    P is a perfect matching found by augmenting paths, visiting each row's two
    columns in ascending order; Q takes each row's other column.  The search
    order is the reference's, so the same points give the same P/Q."""
    if len(points) != 2 * n or len(set(points)) != len(points):
        raise ValueError("a 2-factor needs exactly 2n distinct points")
    adjacency: list[list[int]] = [[] for _ in range(n)]
    column_degree = [0] * n
    for r, c in points:
        if not (0 <= r < n and 0 <= c < n):
            raise ValueError(f"point {(r, c)} outside grid")
        adjacency[r].append(c)
        column_degree[c] += 1
    if any(len(a) != 2 for a in adjacency) or any(d != 2 for d in column_degree):
        raise ValueError("points are not a row/column 2-factor")
    for a in adjacency:
        a.sort()
    owner = [-1] * n  # column -> row matched through P

    def augment(row: int, seen: list[bool]) -> bool:
        for col in adjacency[row]:
            if seen[col]:
                continue
            seen[col] = True
            if owner[col] == -1 or augment(owner[col], seen):
                owner[col] = row
                return True
        return False

    for r in range(n):
        if not augment(r, [False] * n):
            raise ValueError("2-factor unexpectedly has no perfect matching")
    p = [-1] * n
    for col, r in enumerate(owner):
        p[r] = col
    q = [next(c for c in adjacency[r] if c != p[r]) for r in range(n)]
    state = PairPermutations(tuple(p), tuple(q))
    state.validate()
    return state


def legal_swap(columns: np.ndarray, u: int, v: int) -> bool:
    """Row-pair column swap legality of src/no_three_75/tempering.py:58: slots
    in different rows, different columns, and neither new point duplicates the
    other point of its row."""
    c = columns
    cu, cv = int(c[u]), int(c[v])
    return (u >> 1) != (v >> 1) and cu != cv and int(c[u ^ 1]) != cv and int(c[v ^ 1]) != cu


def check_two_factor(columns: np.ndarray) -> None:
    """Raise ValueError unless every row and column holds exactly two distinct
    points (the invariant of src/no_three_75/verifier_a.py:19-34)."""
    c = np.asarray(columns).reshape(-1)
    n = c.size // 2
    if c.size != 2 * n or n < 2:
        raise ValueError("slot columns must have length 2n, n >= 2")
    if c.min() < 0 or c.max() >= n:
        raise ValueError("column outside grid")
    if np.any(c[0::2] == c[1::2]):
        raise ValueError("duplicate point in a row")
    if np.any(np.bincount(c.astype(np.int64), minlength=n) != 2):
        raise ValueError("column degree is not exactly two")
