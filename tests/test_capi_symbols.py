"""The C-ABI library loads on a CPU-only host and exports every entry point
declared in include/n3.h (no compute calls here)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> list[str]:
    text = (ROOT / "include" / "n3.h").read_text()
    names = re.findall(r"^\s*(?:int|const char\s*\*|void)\s+(n3_\w+)\s*\(", text, flags=re.M)
    assert names, "no declarations found"
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from no_three_in_line_b200 import _lib

    L = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"libn3.so lacks {missing}"


def test_version_and_error_string_without_device():
    from no_three_in_line_b200 import _lib

    assert _lib.lib().n3_version() >= 100
    assert isinstance(_lib.last_error(), str)


def test_argument_errors_are_reported_without_touching_the_device():
    """Range and null-pointer checks run on the host before any launch."""
    from no_three_in_line_b200 import _lib

    L = _lib.lib()
    assert L.n3_score_columns(None, 4, 76, None, None, None) == _lib.N3_ERR_RANGE
    assert "76" in _lib.last_error()
    assert L.n3_score_columns(None, 4, 20, None, None, None) == _lib.N3_ERR_ARG
    assert L.n3_score_columns(None, -1, 20, None, None, None) == _lib.N3_ERR_ARG
    assert L.n3_score_columns(None, 0, 20, None, None, None) == _lib.N3_OK  # empty batch is a no-op
