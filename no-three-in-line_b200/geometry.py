"""Integer geometry of grid points (drop-in for ``no_three_75.geometry``,
src/no_three_75/geometry.py:10-40).

Scalar host helpers with the reference's definitions: the population-scale
work (every pair of every state) runs on the device, in the determinant,
slope and line-analysis kernels; these serve single calls and the decoding
of the device's line records.
"""
from __future__ import annotations

from math import gcd

Point = tuple[int, int]
LineKey = tuple[int, int, int]


def determinant(a: Point, b: Point, c: Point) -> int:
    """(b - a) x (c - a): zero iff the three points are collinear (geometry.py:10-11)."""
    return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])


def canonical_line(a: Point, b: Point) -> LineKey:
    """The line through two distinct points as primitive integers (A, B, C)
    with A*row + B*col + C = 0, A > 0 or A = 0 < B (geometry.py:14-28)."""
    if a == b:
        raise ValueError("two distinct points are required")
    A, B = b[1] - a[1], a[0] - b[0]
    C = -(A * a[0] + B * a[1])
    g = gcd(gcd(abs(A), abs(B)), abs(C))
    A, B, C = A // g, B // g, C // g
    if A < 0 or (A == 0 and B < 0):
        A, B, C = -A, -B, -C
    return A, B, C


def primitive_slope(line: LineKey) -> tuple[int, int]:
    """Undirected direction (dx, dy) of a line, gcd 1, dx > 0 or dx = 0 < dy
    (geometry.py:31-40)."""
    dx, dy = line[1], -line[0]
    g = gcd(abs(dx), abs(dy))
    dx, dy = dx // g, dy // g
    if dx < 0 or (dx == 0 and dy < 0):
        dx, dy = -dx, -dy
    return dx, dy
