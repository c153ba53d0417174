"""Population scoring on the B200 (drop-in for ``no_three_75.gpu``).

``score_population_gpu`` keeps the reference's signature and semantics
(src/no_three_75/gpu.py:61-77): P/Q int arrays [B, n] in, exact int32 triple
counts [B] out, ValueError on bad shapes, RuntimeError without a device.  Host
NumPy inputs are copied to the device and the result is returned as NumPy
(the reference's behaviour); CUDA tensors are used in place and a CUDA tensor
is returned without synchronising, so callers can keep populations resident.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import _lib


def _validate_batches(p_batch, q_batch):
    """Shape rules of src/no_three_75/gpu.py:61-66."""
    if _lib.is_tensor(p_batch):
        if p_batch.ndim != 2 or tuple(q_batch.shape) != tuple(p_batch.shape) or p_batch.shape[1] < 2:
            raise ValueError("P and Q must have the same two-dimensional shape")
        return p_batch, q_batch
    p = np.ascontiguousarray(p_batch, dtype=np.int32)
    q = np.ascontiguousarray(q_batch, dtype=np.int32)
    if p.ndim != 2 or q.shape != p.shape or p.shape[1] < 2:
        raise ValueError("P and Q must have the same two-dimensional shape")
    return p, q


def _check_n(n: int) -> None:
    if n > _lib.MAX_N:
        raise ValueError(f"n={n} exceeds the device limit {_lib.MAX_N}")


def score_population_gpu(p_batch, q_batch, *, badness: bool = False, stream=None):
    """Exact integer triple counts for a population of P/Q states.

    Replaces src/no_three_75/gpu.py:69-77 (kernel gpu.py:13-42).  With
    ``badness=True`` also returns the per-slot badness [B, 2n] of
    src/no_three_75/gpu_device_search.py:118-161."""
    p, q = _validate_batches(p_batch, q_batch)
    B, n = int(p.shape[0]), int(p.shape[1])
    _check_n(n)
    t = _lib.torch()
    device = _lib.require_device()
    host = not _lib.is_tensor(p_batch)
    dp = _lib.as_device(p, t.int32, device)
    dq = _lib.as_device(q, t.int32, device)
    scores = t.empty(B, dtype=t.int32, device=device)
    bad = t.empty((B, 2 * n), dtype=t.int32, device=device) if badness else None
    _lib.call("n3_score_population", _lib.ptr(dp), _lib.ptr(dq), B, n, _lib.ptr(scores), _lib.ptr(bad),
              _lib.stream_ptr(stream))
    if host:
        out = scores.cpu().numpy()
        return (out, bad.cpu().numpy()) if badness else out
    return (scores, bad) if badness else scores


def score_columns_gpu(columns, *, badness: bool = False, stream=None):
    """Determinant count over slot-layout columns ([B, 2n] int16 tensor or array)."""
    t = _lib.torch()
    device = _lib.require_device()
    host = not _lib.is_tensor(columns)
    c = _lib.as_device(columns, t.int16, device)
    if c.ndim != 2 or c.shape[1] % 2 or c.shape[1] < 4:
        raise ValueError("columns must have shape (B, 2n) with n >= 2")
    B, n = int(c.shape[0]), int(c.shape[1]) // 2
    _check_n(n)
    scores = t.empty(B, dtype=t.int32, device=device)
    bad = t.empty((B, 2 * n), dtype=t.int32, device=device) if badness else None
    _lib.call("n3_score_columns", _lib.ptr(c), B, n, _lib.ptr(scores), _lib.ptr(bad), _lib.stream_ptr(stream))
    if host:
        out = scores.cpu().numpy()
        return (out, bad.cpu().numpy()) if badness else out
    return (scores, bad) if badness else scores


def score_slope_gpu(columns, *, stream=None):
    """Normalised-slope line count: (E [B], badness [B, 2n])."""
    t = _lib.torch()
    device = _lib.require_device()
    host = not _lib.is_tensor(columns)
    c = _lib.as_device(columns, t.int16, device)
    B, n = int(c.shape[0]), int(c.shape[1]) // 2
    _check_n(n)
    scores = t.empty(B, dtype=t.int32, device=device)
    bad = t.empty((B, 2 * n), dtype=t.int32, device=device)
    _lib.call("n3_score_slope", _lib.ptr(c), B, n, _lib.ptr(scores), _lib.ptr(bad), _lib.stream_ptr(stream))
    if host:
        return scores.cpu().numpy(), bad.cpu().numpy()
    return scores, bad


@dataclass
class CheckedScores:
    scores: object      # determinant E per state
    badness: object     # slope badness per slot
    mismatches: int     # states whose determinant and slope counts differ
    error_word: int     # device error bits (1 column range, 2 duplicate point, 4 mismatch)


def score_checked_gpu(columns, *, stream=None, raise_on_mismatch: bool = True, badness: bool = True) -> CheckedScores:
    """Fused determinant + slope scoring with the on-device cross-check.
    Raises AssertionError on any disagreement (the reference's exact_match
    audit, src/no_three_75/gpu.py:131, made fatal) unless told not to.  With
    ``badness=False`` the slope side counts E alone (each triple once from its
    first slot) and ``badness`` of the result is None."""
    t = _lib.torch()
    device = _lib.require_device()
    host = not _lib.is_tensor(columns)
    c = _lib.as_device(columns, t.int16, device)
    B, n = int(c.shape[0]), int(c.shape[1]) // 2
    _check_n(n)
    scores = t.empty(B, dtype=t.int32, device=device)
    bad = t.empty((B, 2 * n), dtype=t.int32, device=device) if badness else None
    flags = t.zeros(2, dtype=t.int32, device=device)
    _lib.call("n3_score_checked", _lib.ptr(c), B, n, _lib.ptr(scores), _lib.ptr(bad), flags.data_ptr(),
              flags.data_ptr() + 4, _lib.stream_ptr(stream))
    f = flags.cpu().numpy()
    mism, err = int(f[0]), int(np.uint32(f[1]))
    if raise_on_mismatch and (mism or err):
        raise AssertionError(f"checked scoring: {mism} state(s) disagree, device error bits {err:#x}")
    if host:
        return CheckedScores(scores.cpu().numpy(), bad.cpu().numpy() if badness else None, mism, err)
    return CheckedScores(scores, bad, mism, err)


def gpu_device_name() -> str:
    t = _lib.torch()
    _lib.require_device()
    return t.cuda.get_device_name(t.cuda.current_device())


@dataclass(frozen=True)
class GpuBenchmark:
    """Fields of src/no_three_75/gpu.py:80-96."""

    device: str
    population: int
    n: int
    cpu_seconds: float
    gpu_end_to_end_seconds: float
    gpu_kernel_seconds: float
    exact_match: bool

    @property
    def end_to_end_speedup(self) -> float:
        return self.cpu_seconds / max(self.gpu_end_to_end_seconds, 1e-12)

    @property
    def kernel_speedup(self) -> float:
        return self.cpu_seconds / max(self.gpu_kernel_seconds, 1e-12)


def benchmark_gpu(p_batch, q_batch, *, repeats: int = 5, cpu_scores=None, cpu_seconds: float = float("nan")):
    """Timing harness of src/no_three_75/gpu.py:99-139.  The CPU side is the
    caller's (pass ``cpu_scores`` and ``cpu_seconds``); this package has no
    host scorer.  End-to-end includes the host<->device copies; the kernel
    time is CUDA-event timed on resident device buffers."""
    p, q = _validate_batches(p_batch, q_batch)
    t = _lib.torch()
    score_population_gpu(p[:1], q[:1])
    started = time.perf_counter()
    gpu_scores = None
    for _ in range(repeats):
        gpu_scores = score_population_gpu(p, q)
    e2e = (time.perf_counter() - started) / repeats
    device = _lib.require_device()
    dp = _lib.as_device(p, t.int32, device)
    dq = _lib.as_device(q, t.int32, device)
    out = t.empty(p.shape[0], dtype=t.int32, device=device)
    start, end = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(repeats):
        _lib.call("n3_score_population", _lib.ptr(dp), _lib.ptr(dq), p.shape[0], p.shape[1], _lib.ptr(out), None,
                  _lib.stream_ptr())
    end.record()
    end.synchronize()
    kernel = start.elapsed_time(end) / 1000.0 / repeats
    kernel_scores = out.cpu().numpy()
    exact = bool(np.array_equal(gpu_scores, kernel_scores) and
                 (cpu_scores is None or np.array_equal(np.asarray(cpu_scores), gpu_scores)))
    return GpuBenchmark(gpu_device_name(), int(p.shape[0]), int(p.shape[1]), cpu_seconds, e2e, kernel, exact)
