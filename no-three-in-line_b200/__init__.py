"""n3 for B200: the no-three-in-line population search hot path on sm_100a.

A drop-in for the scoring / delta / tempering path of the reference package
``no_three_75`` (MilliganCo/no-three-in-line).  Host code in this package
mirrors the reference's module and function names; all arithmetic runs in
hand-written CUDA kernels behind the C ABI of ``include/n3.h`` (``libn3.so``).

Modules (each mirrors the reference module of the same name where one exists):
    state            two-per-row/column state model and seeding (host)
    geometry         integer geometry helpers: determinant, canonical_line, primitive_slope
    gpu              population scoring: determinant, slope, cross-checked
    accelerated      the reference's CPU-API names (score_and_badness, evaluate_*) on the device
    gpu_delta        exact swap deltas and two-switch scores
    conflicts        line-by-line conflict analysis (analyze_points) on the device
    tempering        replica-exchange tempering chains, the epoch driver (main), checkpoints
    learned          learned move proposal: tcgen05 MLP inference, training, ring buffer
    autotune         launch-shape search for mixed-size tempering
    compare          time-to-target comparison of proposal methods
    gpu_device_search  device-resident beam search
    gpu_neighborhood   three-cycle, four-cycle and double-switch neighbourhood scans
    precompute       grid line tables built on the device and the two table scorers
    breakout         line-weighted energies
    io               candidate file formats (JSON, compact, text)
    shard            splitting populations and ladders over ranks
"""
from __future__ import annotations

__version__ = "0.1.0"

from . import _lib, state  # noqa: F401


def build(force: bool = False):
    """Compile libn3.so for sm_100a (nvcc)."""
    return _lib.build(force=force)
