"""Shared test set-up.

Markers: ``gpu`` tests need a CUDA device and call the CUDA library through
its C ABI; everything else runs on CPU (oracle pins, host logic, symbol
exports, gloo multi-process tests).
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from __graft_entry__ import load_package  # noqa: E402

load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libn3.so")


@pytest.fixture(scope="session")
def golden():
    """Lazy loader of the fixtures in tests/golden (written by make_golden.py)."""
    cache = {}

    def get(name: str):
        if name not in cache:
            path = GOLDEN / name
            if path.suffix == ".json":
                cache[name] = json.loads(path.read_text())
            else:
                with np.load(path, allow_pickle=False) as z:
                    cache[name] = {k: z[k] for k in z.files}
        return cache[name]

    return get


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o

    o.lib()
    return o


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
