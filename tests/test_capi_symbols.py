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


def test_line_table_entry_points_check_arguments_on_the_host():
    """n3_line_tables_* and n3_lines_score_*: ranges, counts and null buffers
    are refused before any launch; an empty batch is a no-op."""
    from no_three_in_line_b200 import _lib, precompute  # noqa: F401  (precompute declares the argument types)

    L = _lib.lib()
    assert L.n3_line_tables_count(0, None, None, None, None) == _lib.N3_ERR_RANGE
    assert L.n3_line_tables_count(76, None, None, None, None) == _lib.N3_ERR_RANGE
    assert L.n3_line_tables_count(5, None, None, None, None) == _lib.N3_ERR_ARG
    assert L.n3_line_tables_build(5, None, None, -1, None, None, None, None) == _lib.N3_ERR_ARG
    assert L.n3_line_tables_build(5, None, None, 22, None, None, None, None) == _lib.N3_ERR_ARG
    assert L.n3_lines_score_pairs(None, None, 3, 0, None, None, None, None) == _lib.N3_ERR_RANGE
    assert L.n3_lines_score_pairs(None, None, -1, 5, None, None, None, None) == _lib.N3_ERR_ARG
    assert L.n3_lines_score_pairs(None, None, 0, 5, None, None, None, None) == _lib.N3_OK
    assert L.n3_lines_score_pairs(None, None, 2, 5, None, None, None, None) == _lib.N3_ERR_ARG
    assert L.n3_lines_score_csr(None, None, 1, 76, 0, None, None, None, None, None, None) == _lib.N3_ERR_RANGE
    assert L.n3_lines_score_csr(None, None, 1, 5, -1, None, None, None, None, None, None) == _lib.N3_ERR_ARG
    assert L.n3_lines_score_csr(None, None, 0, 5, 22, None, None, None, None, None, None) == _lib.N3_OK
    assert L.n3_lines_score_csr(None, None, 4, 5, 22, None, None, None, None, None, None) == _lib.N3_ERR_ARG
    assert "CSR scores" in _lib.last_error()


def test_beam_entry_points_check_arguments_on_the_host():
    """n3_beam_*: descriptor sizes and buffers, and the mutation and shuffle
    arguments, are refused before any launch."""
    import ctypes

    from no_three_in_line_b200 import _lib
    from no_three_in_line_b200.gpu_device_search import BeamDesc

    L = _lib.lib()
    assert L.n3_beam_generation(None, 1, None) == _lib.N3_ERR_ARG
    desc = BeamDesc()
    desc.n, desc.population, desc.elite_size, desc.max_strength, desc.bad_bias, desc.energy_window = 75, 4096, 64, 12, 85, 12
    assert L.n3_beam_init(ctypes.byref(desc), 1, None) == _lib.N3_ERR_ARG  # null buffers
    for field, bad in (("n", 2), ("elite_size", 1), ("population", 65537), ("max_strength", 0), ("bad_bias", 101),
                       ("energy_window", -1)):
        d = BeamDesc()
        ctypes.pointer(d)[0] = desc
        setattr(d, field, bad)
        assert L.n3_beam_generation(ctypes.byref(d), 1, None) == _lib.N3_ERR_RANGE, field
    assert L.n3_beam_mutate(None, None, None, 4, 1, 75, 64, 2, 12, 85, 1, 1, None, None, None) == _lib.N3_ERR_ARG
    assert L.n3_py_random_shuffle(None, None, 3, None) == _lib.N3_ERR_ARG
    assert L.n3_py_shuffle_steps(None, 3, None, None) == _lib.N3_ERR_ARG
    assert L.n3_py_shuffle_steps(ctypes.c_void_p(16), 65537, ctypes.c_void_p(16), None) == _lib.N3_ERR_RANGE


def test_learned_step_checks_its_team_width_on_the_host():
    from no_three_in_line_b200 import _lib, learned
    from no_three_in_line_b200.tempering import N3Chains

    L = _lib.lib()
    ch, M, temps = N3Chains(), learned.N3Mlp(), ctypes.c_void_p(16)
    assert L.n3_mlp_step_team(ctypes.byref(ch), ctypes.byref(M), temps, 1, 1, 32, None) == _lib.N3_ERR_ARG
    assert "capacity" in _lib.last_error()  # an empty ring buffer
    M.rb_capacity = 1024
    assert L.n3_mlp_step_team(ctypes.byref(ch), ctypes.byref(M), temps, 1, 1, 48, None) == _lib.N3_ERR_RANGE
    assert "48" in _lib.last_error()
    assert L.n3_mlp_step_team(ctypes.byref(ch), ctypes.byref(M), temps, 1, 0, 32, None) == _lib.N3_ERR_RANGE
    assert L.n3_mlp_step_team(None, ctypes.byref(M), temps, 1, 1, 32, None) == _lib.N3_ERR_ARG
    # the Python wrapper refuses other widths before it allocates anything
    import pytest

    with pytest.raises(ValueError):
        learned.LearnedProposal.__init__(object.__new__(learned.LearnedProposal), None, threads_per_chain=48)
