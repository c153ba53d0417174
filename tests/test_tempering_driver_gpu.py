"""The tempering driver (tempering.py:228-319): output layout, records,
history audits, checkpoints, resume and the umbrella frontier."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path
from random import Random

import pytest

from no_three_in_line_b200 import gpu, io, state, tempering

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


def initial_file(tmp_path, n=20, seed=91001, name="init.json"):
    s = state.random_state(n, Random(seed))
    path = tmp_path / name
    io.write_candidate(path, n, s.points())
    return path


def test_driver_writes_the_reference_layout(cuda, tmp_path):
    init = initial_file(tmp_path)
    out = tmp_path / "run"
    rc = tempering.main(["--initial", str(init), "--output", str(out), "--seed", "3", "--replicas", "16",
                         "--ladder-size", "8", "--rounds", "60", "--steps", "40", "--bad-bias", "85"])
    assert rc == 0
    params = json.loads((out / "parameters.json").read_text())
    assert params["bad_bias"] == 85 and params["replicas"] == 16
    summary = json.loads((out / "summary.json").read_text())
    assert summary["proposals"] == 60 * 40 * 16 and summary["accepted"] > 0
    records = sorted(out.glob("best-E*.json"), key=lambda p: int(p.stem[6:]))
    assert records and int(records[0].stem[6:]) == summary["best"]
    for rec in records:
        n, pts, meta = io.load_candidate(rec)
        cols = tempering._state_columns(state.points_to_permutations(pts, n))[None]
        e = int(gpu.score_checked_gpu(cols).scores[0])
        assert e == meta["conflicts"] == int(rec.stem[6:])
        assert meta["method"] == "persistent CUDA replica exchange"
    hist = [json.loads(x) for x in (out / "history.jsonl").read_text().splitlines()]
    assert [h["epoch"] for h in hist] == [10, 20, 30, 40, 50, 60]
    assert all(len(h["scores"]) == 16 and len(h["distances"]) == 16 for h in hist)
    assert hist[-1]["best"] == summary["best"]
    # resume from the checkpoint and continue
    out2 = tmp_path / "run2"
    rc = tempering.main(["--initial", str(init), "--output", str(out2), "--seed", "3", "--replicas", "16",
                         "--ladder-size", "8", "--rounds", "20", "--steps", "40", "--resume",
                         str(out / "checkpoint.npz")])
    assert rc == 0
    assert json.loads((out2 / "summary.json").read_text())["best"] <= summary["best"]
    with pytest.raises(ValueError, match="dimensions"):
        tempering.main(["--initial", str(init), "--output", str(out2), "--seed", "3", "--replicas", "8",
                        "--ladder-size", "8", "--resume", str(out / "checkpoint.npz")])


def test_driver_umbrella_frontier(cuda, tmp_path):
    init = initial_file(tmp_path, seed=91007)
    out = tmp_path / "umb"
    rc = tempering.main(["--initial", str(init), "--output", str(out), "--seed", "5", "--replicas", "16",
                         "--ladder-size", "4", "--rounds", "30", "--steps", "60", "--umbrella-max", "24",
                         "--umbrella-strength", "0.5"])
    assert rc == 0
    frontier = sorted(out.glob("frontier-bin*.json"))
    assert frontier
    summary = json.loads((out / "summary.json").read_text())
    assert set(summary["distance_frontier"]) == {str(int(p.stem[len("frontier-bin"):])) for p in frontier}
    hist = [json.loads(x) for x in (out / "history.jsonl").read_text().splitlines()]
    assert all(h["exchanges"] == 0 for h in hist)  # exchanges are off under an umbrella


def test_driver_command_line(cuda, tmp_path):
    init = initial_file(tmp_path, n=12, seed=4)
    out = tmp_path / "cli"
    r = subprocess.run([sys.executable, str(ROOT / "no-three-in-line_b200"), "tempering", "--initial", str(init),
                        "--output", str(out), "--seed", "1", "--replicas", "8", "--ladder-size", "4", "--rounds",
                        "10", "--steps", "20"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert json.loads(r.stdout.strip().splitlines()[-1])["proposals"] == 10 * 20 * 8
    assert (out / "checkpoint.npz").exists()
