"""n3 for B200: the no-three-in-line population search hot path on sm_100a.

A drop-in for the scoring / delta / tempering path of the reference package
``no_three_75`` (MilliganCo/no-three-in-line).  Host code in this package
mirrors the reference's module and function names; all arithmetic runs in
hand-written CUDA kernels behind the C ABI of ``include/n3.h`` (``libn3.so``).

Modules:
    state        two-per-row/column state model and seeding (host)
    gpu          population scoring (determinant, slope, cross-checked)
"""
from __future__ import annotations

__version__ = "0.1.0"

from . import _lib, state  # noqa: F401


def build(force: bool = False):
    """Compile libn3.so for sm_100a (nvcc)."""
    return _lib.build(force=force)
