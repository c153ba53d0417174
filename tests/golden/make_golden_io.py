"""Generate the candidate-file fixture (io_golden.json) from the reference itself.

Run once, in a container that has the reference checked out:

    python tests/golden/make_golden_io.py [/path/to/reference]

Every case below is read by the reference's own ``io.load_candidate`` /
``io.decode_compact`` / ``io.encode_compact`` / ``io.write_candidate``
(src/no_three_75/io.py); the fixture records each input and either the result or
the exception type and message.  Inputs: the strictness cases of the reference's
tests/test_strict_candidate_input.py (written out here as data), compact codes
with every symmetry prefix, plain-text files, P/Q objects and the reference's
results/best-near-solution-E10.json.  The GPU box never runs this script.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
if len(sys.argv) > 1:
    REFERENCE = Path(sys.argv[1])
elif os.environ.get("N3_REFERENCE"):
    REFERENCE = Path(os.environ["N3_REFERENCE"])
else:
    raise SystemExit("usage: make_golden_io.py /path/to/reference  (or set N3_REFERENCE)")
sys.path.insert(0, str(REFERENCE / "src"))

from no_three_75 import io as ref_io  # noqa: E402

SQUARE = [[0, 0], [0, 1], [1, 0], [1, 1]]


def json_cases():
    cases = []
    for pts in ([[bool(r), bool(c)] for r, c in SQUARE], [[float(r), float(c)] for r, c in SQUARE],
                [[r + .25, c + .75] for r, c in SQUARE], [[str(r), str(c)] for r, c in SQUARE],
                ["00", "01", "10", "11"], [[0, 0, 99], [0, 1], [1, 0], [1, 1]], [[0], [0, 1], [1, 0], [1, 1]],
                [None, [0, 1], [1, 0], [1, 1]]):
        cases.append(("bad_points", {"n": 2, "points": pts}, None))
    for pts in (None, True, 3, "00", {"0": [0, 0]}):
        cases.append(("bad_container", {"n": 2, "points": pts}, None))
    for bad_n in (True, False, 2.0, 2.5, "2", None, 0, -1):
        for explicit in (None, 2):
            cases.append(("bad_file_n", {"n": bad_n, "points": SQUARE}, explicit))
    for bad_n in (True, False, 2.0, 2.5, "2", 0, -1):
        cases.append(("bad_api_n", {"n": 2, "points": SQUARE}, bad_n))
    for payload in (SQUARE, {"points": SQUARE}, {"n": 2, "points": SQUARE, "label": "synthetic"},
                    {"n": 2, "P": [0, 1], "Q": [1, 0]}, {"n": 2, "points": [[r + 1, c + 1] for r, c in SQUARE]},
                    {"n": 2, "points": SQUARE, "extra": [1, 2], "score": 3}, []):
        cases.append(("valid", payload, None))
    cases.append(("override", {"n": 2, "points": SQUARE}, 3))
    for bad in (True, 0.0, "0", None, [0, 1]):
        cases.append(("bad_pq", {"n": 2, "P": [bad, 1], "Q": [1, 0]}, None))
    for bad in ("01", {}, None, True):
        cases.append(("bad_pq_container", {"n": 2, "P": bad, "Q": [1, 0]}, None))
    cases.append(("no_points", {"n": 2}, None))
    cases.append(("scalar", 5, None))
    return cases


def outcome(fn):
    try:
        n, points, meta = fn()
        meta = {k: v for k, v in meta.items() if k != "source_path"}
        return {"ok": True, "n": n, "points": [list(p) for p in points], "meta": meta}
    except Exception as exc:  # noqa: BLE001 - the fixture records the reference's exception
        return {"ok": False, "error": type(exc).__name__, "message": str(exc)}


def main():
    out = {"json": [], "text": [], "compact": [], "encode": [], "write": []}
    with tempfile.TemporaryDirectory() as tmp:
        tmp = Path(tmp)
        for k, (label, payload, n) in enumerate(json_cases()):
            path = tmp / f"c{k}.json"
            path.write_text(json.dumps(payload), encoding="utf-8")
            out["json"].append({"label": label, "payload": payload, "n": n,
                                "result": outcome(lambda: ref_io.load_candidate(path, n=n))})
        for k, (text, n) in enumerate([("0 0\n0 1\n1 0\n1 1\n", None), ("(0,1) (2,3)\n(4,5)", None),
                                       ("0 0 1", None), ("3 4 -1 2", None), ("1 1 2 2", 5), ("", None),
                                       (".0101", None), (".0101", 2), (":10", None), ("*0101", 3)]):
            path = tmp / f"t{k}.txt"
            path.write_text(text, encoding="utf-8")
            out["text"].append({"text": text, "n": n, "result": outcome(lambda: ref_io.load_candidate(path, n=n))})
        for code, n in [(".0101", None), (".0101", 2), (":0110", None), ("/1212", 3), ("-0101", None),
                        ("o0101", None), ("c0101", None), ("x0101", None), ("+0101", None), ("*0101", None),
                        ("?0101", None), (".010", None), (".0102", None), (".01Z1", None), ("", None),
                        ("  .0101  ", None), (".0101", 3), (".0101", True)]:
            try:
                res = ref_io.decode_compact(code, n=n)
                r = {"ok": True, "n": res[0], "symmetry": res[1], "points": [list(p) for p in res[2]]}
            except Exception as exc:  # noqa: BLE001
                r = {"ok": False, "error": type(exc).__name__, "message": str(exc)}
            out["compact"].append({"code": code, "n": n, "result": r})
        for pts, n, sym in [(SQUARE, 2, "iden"), (SQUARE, 2, "."), (SQUARE, 2, "full"), (SQUARE, 2, "bogus"),
                            ([[0, 0], [0, 1], [1, 0]], 2, "iden"), ([[0, 0], [0, 5], [1, 0], [1, 1]], 2, "iden"),
                            (SQUARE, 2, ""), (SQUARE, 2, "ocx")]:
            try:
                r = {"ok": True, "code": ref_io.encode_compact([tuple(p) for p in pts], n, sym)}
            except Exception as exc:  # noqa: BLE001
                r = {"ok": False, "error": type(exc).__name__, "message": str(exc)}
            out["encode"].append({"points": pts, "n": n, "symmetry": sym, "result": r})
        for k, (n, pts, meta) in enumerate([(2, [[1, 1], [0, 0], [1, 0], [0, 1]], {}),
                                            (3, [[2, 0], [0, 2]], {"conflicts": 4, "P": [0, 1, 2], "label": "x"})]):
            path = tmp / f"w{k}.json"
            ref_io.write_candidate(path, n, [tuple(p) for p in pts], **meta)
            out["write"].append({"n": n, "points": pts, "meta": meta, "text": path.read_text(encoding="utf-8")})
        e10 = REFERENCE / "results" / "best-near-solution-E10.json"
        out["e10"] = outcome(lambda: ref_io.load_candidate(e10))
        out["e10_text"] = e10.read_text(encoding="utf-8")
    (HERE / "io_golden.json").write_text(json.dumps(out, indent=1) + "\n")
    print({k: len(v) for k, v in out.items() if isinstance(v, list)})


if __name__ == "__main__":
    main()
