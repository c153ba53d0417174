"""ctypes binding of libn3.so (the C ABI declared in include/n3.h).

The library is the only compute path: if it is missing or no CUDA device is
present, every entry point raises instead of falling back to host code.
PyTorch provides device memory and the current stream; pointers and sizes
cross the boundary as plain integers.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libn3.so"
CSRC = PKG_DIR / "csrc"

N3_OK, N3_ERR_ARG, N3_ERR_RANGE, N3_ERR_CUDA, N3_ERR_MISMATCH, N3_ERR_TIMEOUT, N3_ERR_STATE = range(7)
MAX_N = 75
SENTINEL = 1 << 30

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_U64 = ctypes.c_uint64
_F = ctypes.c_float

# name -> argtypes (all return int status unless listed in _RESTYPE)
_SIGNATURES: dict[str, list] = {
    "n3_version": [],
    "n3_last_error": [],
    "n3_init_device": [],
    "n3_score_population": [_P, _P, _I, _I, _P, _P, _P],
    "n3_score_columns": [_P, _I, _I, _P, _P, _P],
    "n3_score_slope": [_P, _I, _I, _P, _P, _P],
    "n3_score_checked": [_P, _I, _I, _P, _P, _P, _P, _P],
    "n3_calibrate_det_ceiling": [_I, _I, _P, _P],
    "n3_calibrate_int_pipe": [_I, _I, _I, _P, _P],
    "n3_calibrate_l2_gather": [_P, _I64, _I, _I, _P, _P],
    "n3_swap_delta": [_P, _I, _I, _P, _I, _P, _P, _P],
    "n3_swap_delta_pairs": [_P, _I, _I, _P, _I, _P, _P, _P],
    "n3_two_switch_scores": [_P, _P, _P, _I, _I, _P, _I, _P, _P],
    "n3_transposition_scores": [_P, _P, _P, _I, _I, _P, _I, _P, _P],
    "n3_graph_begin": [_P],
    "n3_graph_end": [_P, ctypes.POINTER(ctypes.c_void_p)],
    "n3_graph_launch": [_P, _P],
    "n3_graph_destroy": [_P],
}
_RESTYPE = {"n3_last_error": ctypes.c_char_p}

_lib = None
_ready: set[int] = set()


def build(force: bool = False) -> Path:
    """Compile libn3.so for sm_100a with nvcc (csrc/Makefile)."""
    if force or not LIB_PATH.exists():
        subprocess.run(["make", "-s", "-C", str(CSRC)], check=True)
    return LIB_PATH


def lib():
    """The loaded library; raises RuntimeError when it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"the n3 CUDA library is not built ({LIB_PATH} missing); "
                               f"run `make -C {CSRC}` or __graft_entry__.build()")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, args in _SIGNATURES.items():
            try:
                f = getattr(L, name)
            except AttributeError:
                continue  # declared later in the build; symbol tests cover completeness
            f.argtypes = args
            f.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = L
    return _lib


def register(name: str, args: list, restype=ctypes.c_int) -> None:
    """Declare an entry point's argument types (used by the modules that wrap it)."""
    _SIGNATURES[name] = args
    if restype is not ctypes.c_int:
        _RESTYPE[name] = restype
    if _lib is not None:
        f = getattr(_lib, name)
        f.argtypes = args
        f.restype = restype


def last_error() -> str:
    raw = lib().n3_last_error()
    return raw.decode() if raw else ""


def check(rc: int, what: str) -> None:
    """Map a status code to the reference's exception conventions:
    ValueError for shapes/ranges (gpu.py:64-65, gpu_delta.py:96-97),
    AssertionError for incremental-vs-full mismatches (tempering.py:200-201),
    RuntimeError for device failures (gpu.py:50-51), TimeoutError for an
    expired bounded device wait."""
    if rc == N3_OK:
        return
    msg = f"{what}: {last_error()}"
    if rc in (N3_ERR_ARG, N3_ERR_RANGE, N3_ERR_STATE):
        raise ValueError(msg)
    if rc == N3_ERR_MISMATCH:
        raise AssertionError(msg)
    if rc == N3_ERR_TIMEOUT:
        raise TimeoutError(msg)
    raise RuntimeError(msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args), name)


# --------------------------------------------------------------------------
# Device helpers (torch is the allocator and stream provider only).
# --------------------------------------------------------------------------

def torch():
    import torch as _torch

    return _torch


def require_device():
    """Return the current CUDA device, or raise RuntimeError like gpu.py:50-51."""
    t = torch()
    if not t.cuda.is_available() or t.cuda.device_count() < 1:
        raise RuntimeError("no CUDA device is available")
    L = lib()
    dev = t.cuda.current_device()
    if dev not in _ready:
        check(L.n3_init_device(), "n3_init_device")
        _ready.add(dev)
    return t.device("cuda", dev)


def stream_ptr(stream=None) -> int:
    t = torch()
    s = stream if stream is not None else t.cuda.current_stream()
    return int(s.cuda_stream)


def ptr(x) -> int | None:
    return None if x is None else int(x.data_ptr())


def as_device(x, dtype, device=None):
    """A contiguous device tensor of `dtype` holding x (numpy, list or tensor).
    Tensors already on the device with the right dtype are used in place."""
    t = torch()
    device = device if device is not None else require_device()
    if isinstance(x, t.Tensor):
        if x.device.type == "cuda" and x.dtype == dtype and x.is_contiguous():
            return x
        return x.to(device=device, dtype=dtype).contiguous()
    arr = np.ascontiguousarray(np.asarray(x))
    return t.from_numpy(arr).to(device=device, dtype=dtype, non_blocking=False).contiguous()


def is_tensor(x) -> bool:
    try:
        return isinstance(x, torch().Tensor)
    except ImportError:  # pragma: no cover
        return False


def env_flag(name: str) -> bool:
    return os.environ.get(name, "") not in ("", "0", "false", "False")
