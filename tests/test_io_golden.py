"""Candidate files (src/no_three_75/io.py) against the reference's own results
on the same inputs (tests/golden/io_golden.json, written by make_golden_io.py):
strict JSON rules, P/Q objects, compact codes, plain text, writer output."""
from __future__ import annotations

import json

import pytest

from no_three_in_line_b200 import io as n3io


@pytest.fixture(scope="module")
def g(golden):
    return golden("io_golden.json")


def outcome(fn):
    try:
        n, points, meta = fn()
        meta = {k: v for k, v in meta.items() if k != "source_path"}
        return {"ok": True, "n": n, "points": [list(p) for p in points], "meta": meta}
    except Exception as exc:  # noqa: BLE001 - compared with the reference's exception
        return {"ok": False, "error": type(exc).__name__, "message": str(exc)}


def test_json_candidates(g, tmp_path):
    for k, case in enumerate(g["json"]):
        path = tmp_path / f"c{k}.json"
        path.write_text(json.dumps(case["payload"]), encoding="utf-8")
        assert outcome(lambda: n3io.load_candidate(path, n=case["n"])) == case["result"], case


def test_text_and_compact_files(g, tmp_path):
    for k, case in enumerate(g["text"]):
        path = tmp_path / f"t{k}.txt"
        path.write_text(case["text"], encoding="utf-8")
        assert outcome(lambda: n3io.load_candidate(path, n=case["n"])) == case["result"], case


def test_decode_compact(g):
    for case in g["compact"]:
        try:
            n, sym, pts = n3io.decode_compact(case["code"], n=case["n"])
            got = {"ok": True, "n": n, "symmetry": sym, "points": [list(p) for p in pts]}
        except Exception as exc:  # noqa: BLE001
            got = {"ok": False, "error": type(exc).__name__, "message": str(exc)}
        assert got == case["result"], case


def test_encode_compact(g):
    for case in g["encode"]:
        try:
            got = {"ok": True, "code": n3io.encode_compact([tuple(p) for p in case["points"]], case["n"],
                                                           case["symmetry"])}
        except Exception as exc:  # noqa: BLE001
            got = {"ok": False, "error": type(exc).__name__, "message": str(exc)}
        assert got == case["result"], case


def test_writer_is_byte_identical(g, tmp_path):
    for k, case in enumerate(g["write"]):
        path = tmp_path / f"w{k}.json"
        n3io.write_candidate(path, case["n"], [tuple(p) for p in case["points"]], **case["meta"])
        assert path.read_text(encoding="utf-8") == case["text"]


def test_reference_fixture_round_trip(g, tmp_path):
    path = tmp_path / "best-near-solution-E10.json"
    path.write_text(g["e10_text"], encoding="utf-8")
    got = outcome(lambda: n3io.load_candidate(path))
    assert got == g["e10"]
    n, points, _ = n3io.load_candidate(path)
    code = n3io.encode_compact(points, n)
    assert n3io.decode_compact(code)[2] == sorted(points)
