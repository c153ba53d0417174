"""Candidate files (drop-in for ``no_three_75.io``, src/no_three_75/io.py:1-132).

Formats read by ``load_candidate``:

* JSON: an object with ``n`` (a positive int, never a bool, float or string) and
  ``points`` (a list of ``[row, column]`` pairs of plain ints, never coerced) or
  ``P`` / ``Q`` row lists; or a bare list of pairs.  Other keys are kept as
  metadata.  Coordinates stay as written (zero-based, no shifting).
* compact: one token, a symmetry prefix character followed by two column
  characters per row (``ALPHABET``), e.g. ``.0101`` for the 2x2 square.
* plain text: any whitespace/punctuation-separated integers, read as
  (row, column) pairs.

``write_candidate`` writes the JSON form with points sorted.  ``n`` resolves as:
the caller's ``n``, else the file's ``n``, else one more than the largest row.
The alphabet, symmetry prefixes and names are the reference's format tables.
"""
from __future__ import annotations

import json
import re
from pathlib import Path
from typing import Iterable

Point = tuple[int, int]

# format tables (io.py:10-21): column characters, symmetry prefix -> name
ALPHABET = "0123456789ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz#$%&@?!()[]<>{}=*+|-/~^_:;,."
SYMMETRY_NAMES = {".": "iden", ":": "rot2", "/": "dia1", "-": "ort1", "o": "rot4", "c": "rct4", "x": "dia2",
                  "+": "ort2", "*": "full"}
SYMMETRY_PREFIXES = "".join(SYMMETRY_NAMES)
_COLUMN_OF = {ch: i for i, ch in enumerate(ALPHABET)}


def _positive_int(value: object, label: str = "n") -> int:
    """An exact int >= 1 (bool is an int subclass and is refused)."""
    if type(value) is not int or value < 1:
        raise ValueError(f"{label} must be a positive integer")
    return value


def _pairs(value: object) -> list[Point]:
    if not isinstance(value, list):
        raise ValueError("JSON points must be a list")
    out: list[Point] = []
    for k, item in enumerate(value):
        if not (isinstance(item, list) and len(item) == 2 and type(item[0]) is int and type(item[1]) is int):
            raise ValueError(f"point {k} must be a list of exactly two integers")
        out.append((item[0], item[1]))
    return out


def decode_compact(code: str, n: int | None = None) -> tuple[int, str, list[Point]]:
    """(n, symmetry name, points) of a compact code (io.py:46-69)."""
    if n is not None:
        n = _positive_int(n)
    code = code.strip()
    if not code or code[0] not in SYMMETRY_NAMES:
        raise ValueError("compact code has no recognized symmetry prefix")
    body = code[1:]
    if n is None:
        if len(body) % 2:
            raise ValueError("compact payload length is not even")
        n = len(body) // 2
    n = _positive_int(n)
    if len(body) != 2 * n:
        raise ValueError(f"compact payload has {len(body)} columns, expected {2 * n}")
    points: list[Point] = []
    for k, ch in enumerate(body):
        column = _COLUMN_OF.get(ch)
        if column is None:
            raise ValueError(f"unknown compact character {ch!r}")
        if column >= n:
            raise ValueError(f"column {column} outside n={n}")
        points.append((k // 2, column))
    return n, SYMMETRY_NAMES[code[0]], points


def encode_compact(points: Iterable[Point], n: int, symmetry: str = "iden") -> str:
    """Compact code of a two-per-row point set (io.py:72-83); ``symmetry`` is a
    name (``iden`` ...) or a prefix character."""
    prefix = next((p for p, name in SYMMETRY_NAMES.items() if name == symmetry), None)
    if prefix is None and symmetry in SYMMETRY_PREFIXES:  # substring test, as the reference does
        prefix = symmetry
    if prefix is None:
        raise ValueError(f"unknown symmetry {symmetry!r}")
    per_row: list[list[int]] = [[] for _ in range(n)]
    for row, column in points:
        if not (0 <= row < n and 0 <= column < n):
            raise ValueError(f"point {(row, column)} outside n={n}")
        per_row[row].append(column)
    if any(len(cols) != 2 for cols in per_row):
        raise ValueError("compact format requires exactly two points in every row")
    return prefix + "".join(ALPHABET[c] for cols in per_row for c in sorted(cols))


def _from_json(payload, n: int | None, metadata: dict) -> tuple[int, list[Point], dict]:
    file_n = None
    if isinstance(payload, dict):
        if "n" in payload:
            file_n = _positive_int(payload["n"], "JSON n")
        data = payload.get("points")
        if data is None and "P" in payload and "Q" in payload:
            P, Q = payload["P"], payload["Q"]
            if not isinstance(P, list) or not isinstance(Q, list):
                raise ValueError("JSON P and Q must be lists")
            data = [[r, c] for r, c in enumerate(P)] + [[r, c] for r, c in enumerate(Q)]
        if data is None:
            raise ValueError("JSON candidate has neither points nor P/Q")
        metadata.update({k: v for k, v in payload.items() if k != "points"})
    elif isinstance(payload, list):
        data = payload
    else:
        raise ValueError("JSON candidate must be an object or a points list")
    points = _pairs(data)
    if n is not None:
        resolved = n
    elif file_n is not None:
        resolved = file_n
    else:
        resolved = max((r for r, _ in points), default=-1) + 1
    return _positive_int(resolved), points, metadata


def load_candidate(path: str | Path, n: int | None = None) -> tuple[int, list[Point], dict]:
    """(n, points, metadata) of a candidate file (io.py:86-126)."""
    if n is not None:
        n = _positive_int(n)
    p = Path(path)
    text = p.read_text(encoding="utf-8").strip()
    metadata: dict = {"source_path": str(p)}
    if p.suffix.lower() == ".json" or text[:1] in ("{", "["):
        return _from_json(json.loads(text), n, metadata)
    tokens = text.split()
    if len(tokens) == 1 and tokens[0][0] in SYMMETRY_NAMES:
        decoded_n, symmetry, points = decode_compact(tokens[0], n=n)
        metadata.update({"compact": tokens[0], "symmetry": symmetry})
        return decoded_n, points, metadata
    values = [int(v) for v in re.findall(r"-?\d+", text)]
    if len(values) % 2:
        raise ValueError("text candidate contains an odd number of integers")
    points = list(zip(values[0::2], values[1::2]))
    resolved = n if n is not None else max((r for r, _ in points), default=-1) + 1
    return _positive_int(resolved), points, metadata


def write_candidate(path: str | Path, n: int, points: Iterable[Point], **metadata: object) -> None:
    """JSON candidate with sorted points, then the metadata (io.py:129-132)."""
    ordered = sorted((int(r), int(c)) for r, c in points)
    payload = {"n": int(n), "points": [[r, c] for r, c in ordered], **metadata}
    Path(path).write_text(json.dumps(payload, indent=2, sort_keys=False) + "\n", encoding="utf-8")
