"""Benchmark of the n=75 population search hot path on B200.

One step = one cross-checked scoring pass over the n=75 population: 4096
seeded two-per-row/column states (150 int16 points each, 551,300 triple tests
per state), exact determinant count + independent gcd-normalised slope count
+ badness + on-device mismatch check, in one launch of n3_score_checked.
``value`` is states scored per second over all ranks with the population
resident in HBM; ``e2e`` is the same metric through the C ABI with host
buffers (pinned H2D of the step's columns, D2H of its scores and flags).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun each rank scores its own population (weak scaling, no
data-path collective); the step time is the max over ranks.
``--impl reference`` times the reference's CPU algorithm (the C restatement
in oracle/, all host threads) on the same workload and metric: determinant
count, slope line count with badness, and their comparison per state.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "n=75 states scored/s & swap deltas/s; time-to-E≤12, learned vs plain proposal"
UNIT = "states/s"
N = 75
STATES = 4096
TESTS_PER_STATE = math.comb(2 * N, 3)  # 551,300
# the determinant kernel tests every triple except those holding two points of
# one row (never collinear with a third point in another row): 75 rows x 148
KERNEL_TESTS_PER_STATE = TESTS_PER_STATE - N * (2 * N - 2)  # 540,200
# per test: one product on the FMA pipe (2 multiplies + 2 multiply-adds serve
# 4 tests) and one compare on the ALU pipe
OPS_PER_TEST = 2
L2_FLUSH_BYTES = 256 << 20             # > 126 MB L2
WORKLOAD = "n=75 population scoring, 4096 states, determinant + slope cross-check + badness"
# dram__bytes_read.sum + dram__bytes_write.sum of one det_kernel launch over the
# 4096-state population, from an ncu capture (1,253,632 B read, 0 B written; the
# algorithmic input is 1,228,800 B of int16 columns plus the 16 KB of counts).
DET_TRAFFIC_BYTES = 1253632


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--states", type=int, default=STATES)
    ap.add_argument("--mode", choices=["checked", "det", "slope", "tempering", "learned", "time-to-target", "beam",
                                       "scan", "lines", "exhaustive"],
                    default="checked",
                    help="kernel a step runs: fused checked scoring (default), determinant only, slope only; "
                         "tempering / learned chain rounds; one device beam-search generation (beam); one "
                         "four-cycle + double-switch neighbourhood scan (scan); the n = 75 line tables "
                         "and both table scorers (lines); one exhaustive 2-switch beam generation (exhaustive); "
                         "or the learned-vs-plain time-to-target comparison")
    ap.add_argument("--no-secondary", action="store_true", help="skip the delta/tempering/MLP measurements")
    ap.add_argument("--seeds", type=int, default=3, help="time-to-target: seeds per method")
    ap.add_argument("--budget", type=float, default=30.0, help="time-to-target: device seconds per run")
    ap.add_argument("--target", type=int, default=12, help="time-to-target: energy target")
    ap.add_argument("--methods", type=str, default="plain,plain:b85,learned:x16:b85",
                    help="time-to-target: comma-separated methods: plain, plain:b<bias>, learned, "
                         "learned:x<moves>, learned:x<moves>:b<bias> (b = the walk's badness-biased share)")
    ap.add_argument("--log", type=str, default=None, help="time-to-target: append each finished run to this JSONL file")
    ap.add_argument("--anneal-sweeps", type=int, default=0,
                    help="tempering / learned: untimed sweeps first, so the timed rounds run at low energies")
    ap.add_argument("--learned-moves", type=str, default="1",
                    help="time-to-target: comma-separated moves per learned step to compare (1 = one move per "
                         "step); learned: the first value is the moves per step")
    ap.add_argument("--learned-threads", type=int, default=0, choices=(0, 32, 64),
                    help="learned: threads per chain of the exact moves (0 = the library's default)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def population(n: int, count: int, rank: int):
    from no_three_in_line_b200 import state

    p, q = state.seeded_population(n, count, base_seed=91001 + rank * count)
    return p, q, state.pq_to_columns(p, q)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
            time.sleep(0.15)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.06)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = [r.split(",") for r in Path(self.path).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for name, flag in zip(names, r[5:9]):
                if flag.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def host_threads() -> int:
    """Host threads this process may run on (its CPU affinity)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # not Linux
        return os.cpu_count() or 1


def host_description() -> dict:
    model = "unknown"
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu": model, "nproc": os.cpu_count(), "affinity_threads": host_threads()}


def cpu_checked_pass(p, q, threads: int) -> int:
    """One CPU pass of the GPU step's work on the host: the reference's
    determinant count (accelerated.py:14-37) and its normalised-slope line
    count with badness (verifier_b.py:8-19 counted as conflicts.py:36-72 sums),
    both restated in C in oracle/, then the per-state comparison.  Returns the
    number of states whose counts differ."""
    from oracle import oracle

    det = oracle.score_population(p, q, threads=threads)
    slope, _ = oracle.slope_population(p, q, threads=threads)
    return int(np.count_nonzero(det != slope))


def cpu_reference_rate(p, q, *, threads: int, steps: int, warmup: int, step_seconds: float = 0.5) -> dict:
    """The CPU timing used by both the GPU arm's ``cpu_baseline`` and the
    ``--impl reference`` arm: the sample per step is sized to about
    ``step_seconds`` of work at this thread count, ``warmup`` untimed passes
    come first, then ``steps`` timed passes over consecutive samples."""
    cpu_checked_pass(p[:8], q[:8], 1)  # load the library
    t0 = time.perf_counter()
    cpu_checked_pass(p[:64], q[:64], threads)
    per_state = (time.perf_counter() - t0) / 64
    sample = int(max(threads, min(len(p), step_seconds / max(per_state, 1e-9))))
    for _ in range(warmup):
        cpu_checked_pass(p[:sample], q[:sample], threads)
    times = []
    for k in range(steps):
        lo = (k * sample) % max(1, len(p) - sample + 1)
        t0 = time.perf_counter()
        if cpu_checked_pass(p[lo:lo + sample], q[lo:lo + sample], threads):
            raise AssertionError("CPU determinant and slope counts differ")
        times.append(time.perf_counter() - t0)
    total = sum(times)
    return {"value": sample * steps / total, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{sample} n=75 states per pass, {steps} timed passes after {warmup} warm-up passes: "
                      f"determinant count (accelerated.py:14-37) + slope line count with badness "
                      f"(verifier_b.py:8-19, conflicts.py:36-72) + comparison, restated in C, {threads} threads",
            "host": host_description(), "seconds": total, "ms_per_step": 1e3 * total / steps}


def bench_config(states: int, world: int) -> dict:
    """The configuration both arms report for the default (checked) mode."""
    return {"workload": WORKLOAD, "n": N, "states_per_gpu": states, "slots": 2 * N,
            "triple_tests_per_state": TESTS_PER_STATE, "parallelism": f"shard{world}",
            "l2": "256 MiB buffer written between GPU steps, outside the per-step CUDA events"}


def lines_cpu_baseline(tables, p, q, sample: int = 24):
    """score_pair_table + score_csr (precompute.py:60-89, restated in NumPy in
    oracle/) on `sample` states after 2 warm-up states, one host thread (the
    restatement is single-threaded NumPy)."""
    from oracle import oracle

    t = {"n": tables.n, "pair_to_line": tables.pair_to_line, "offsets": tables.offsets, "indices": tables.indices,
         "line_count": tables.line_count}
    n = tables.n
    pts = [[(r, int(p[b, r])) for r in range(n)] + [(r, int(q[b, r])) for r in range(n)]
           for b in range(sample + 2)]
    for x in pts[:2]:
        oracle.score_pair_table(x, t)
        oracle.score_csr(x, t)
    t0 = time.perf_counter()
    for x in pts[2:]:
        oracle.score_pair_table(x, t)
        oracle.score_csr(x, t)
    dt = time.perf_counter() - t0
    return {"value": sample / dt, "unit": "states/s", "cores": 1, "kind": "port",
            "sample": f"{sample} n=75 states after 2 warm-up states, score_pair_table + score_csr (precompute.py:60-89 "
                      f"restated in NumPy), 1 thread, {dt:.2f} s", "host": host_description()}


def secondary_measurements(dev, p, q):
    """Swap deltas/s and tempering / learned-proposal throughput at the
    configurations of the metric, each timed with CUDA events after warm-up."""
    import torch

    from no_three_in_line_b200 import _lib, autotune, gpu_delta, learned, state, tempering

    out = {}
    launches = 0
    # batched exact swap deltas over the n=75 population
    cols = torch.from_numpy(state.pq_to_columns(p, q)).to(dev)
    rng = np.random.default_rng(5)
    M = 1 << 16
    moves = torch.from_numpy(np.stack([rng.integers(0, cols.shape[0], M), rng.integers(0, 150, M),
                                       rng.integers(0, 150, M)], 1).astype(np.int32)).to(dev)
    dE = torch.empty(M, dtype=torch.int32, device=dev)
    L = _lib.lib()
    sptr = _lib.stream_ptr()
    for _ in range(3):
        _lib.check(L.n3_swap_delta(cols.data_ptr(), cols.shape[0], N, moves.data_ptr(), M, dE.data_ptr(), None, sptr),
                   "n3_swap_delta")
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(10):
        _lib.check(L.n3_swap_delta(cols.data_ptr(), cols.shape[0], N, moves.data_ptr(), M, dE.data_ptr(), None, sptr),
                   "n3_swap_delta")
    b.record()
    b.synchronize()
    legal = int((dE != gpu_delta.SENTINEL).sum().item())
    out["swap_delta_batch"] = {"moves": M, "legal": legal, "deltas_per_s": 10 * M / (a.elapsed_time(b) / 1e3),
                               "kernel": "n3::swap_delta_kernel<false> (direction-class, no badness output)"}
    launches += 13
    # every 2-switch partner of every slot of 64 n=75 states (the reference plugin's
    # two_switch_scores, gpu_delta.py:19-75): 9600 anchors x 150 partners
    S = 64
    sc = torch.empty(S, dtype=torch.int32, device=dev)
    sb = torch.empty((S, 2 * N), dtype=torch.int32, device=dev)
    _lib.check(L.n3_score_columns(cols.data_ptr(), S, N, sc.data_ptr(), sb.data_ptr(), sptr), "n3_score_columns")
    anchors = torch.from_numpy(np.stack([np.repeat(np.arange(S), 2 * N), np.tile(np.arange(2 * N), S)], 1)
                               .astype(np.int32)).to(dev)
    A = anchors.shape[0]
    ts = torch.empty((A, 2 * N), dtype=torch.int32, device=dev)
    for _ in range(3):
        _lib.check(L.n3_two_switch_scores(cols.data_ptr(), sb.data_ptr(), sc.data_ptr(), S, N, anchors.data_ptr(), A,
                                          ts.data_ptr(), sptr), "n3_two_switch_scores")
    a.record()
    for _ in range(10):
        _lib.check(L.n3_two_switch_scores(cols.data_ptr(), sb.data_ptr(), sc.data_ptr(), S, N, anchors.data_ptr(), A,
                                          ts.data_ptr(), sptr), "n3_two_switch_scores")
    b.record()
    b.synchronize()
    legal_ts = int((ts != gpu_delta.SENTINEL).sum().item())
    out["two_switch_scores"] = {"anchors": A, "partners_scored": A * 2 * N, "legal": legal_ts,
                                "us_per_call": a.elapsed_time(b) / 10 * 1e3,
                                "scores_per_s": 10 * A * 2 * N / (a.elapsed_time(b) / 1e3),
                                "kernel": "n3::partner_scores_kernel<false>"}
    launches += 14
    # C3: 2048 chains at n=75, 32 ladders of 64 temperatures, exchange every 10 sweeps
    pc, qc = state.seeded_population(N, 2048)
    ch = tempering.TemperingChains(state.pq_to_columns(pc, qc), np.tile(tempering.geometric_ladder(0.05, 5.0, 64), 32),
                                   seed=1, ladder_size=64)
    ch.run(20, exchange_every=10, sweeps_per_launch=20)
    res = ch.run(100, exchange_every=10, sweeps_per_launch=100)
    ch.validate()
    out["tempering_n75_2048_chains"] = {"sweeps": res.sweeps, "seconds": res.seconds,
                                        "deltas_per_s": res.proposals / res.seconds,
                                        "triple_tests_per_s_equivalent": res.proposals / res.seconds * 43808,
                                        "best_E_after_120_sweeps": res.best}
    launches += 2
    # C4: mixed sizes in one launch, autotuned
    groups = []
    for k, (n, cnt) in enumerate([(40, 1024), (52, 768), (60, 512), (68, 384), (75, 256)]):
        pp, qq = state.seeded_population(n, cnt)
        groups.append((n, state.pq_to_columns(pp, qq)))
    mixed = tempering.TemperingChains.mixed(groups, tempering.geometric_ladder(0.05, 5.0, 32), seed=2)
    tune = autotune.autotune(mixed, probe_sweeps=20)
    mixed.run(max(tune.ladder_sweeps), exchange_every=10, chains_per_block=tune.chains_per_block,
              ladder_sweeps=tune.ladder_sweeps, threads_per_chain=tune.threads_per_chain)
    res = mixed.run(max(tune.ladder_sweeps), exchange_every=10, chains_per_block=tune.chains_per_block,
                    ladder_sweeps=tune.ladder_sweeps, threads_per_chain=tune.threads_per_chain)
    mixed.validate()
    per = {}
    for n in sorted(tune.size_sweeps):
        lad = int((mixed.ladder_n_host == n).sum())
        per[str(n)] = tune.size_sweeps[n] * 2 * n * 32 * lad / res.seconds
    out["mixed_sizes_one_launch"] = {"autotuned": {"threads_per_chain": tune.threads_per_chain,
                                                   "chains_per_block": tune.chains_per_block,
                                                   "sweeps_per_launch": {str(k): v for k, v in tune.size_sweeps.items()},
                                                   "shape_candidates_deltas_per_s": dict(tune.candidates)},
                                     "seconds": res.seconds, "deltas_per_s_per_size": per,
                                     "deltas_per_s_total": res.proposals / res.seconds}
    launches += 2
    # the reference CLI's default run shape (tempering.py:233-236): 128 replicas in
    # ladders of 16 temperatures 0.2..4, every (threads per chain, cpb) timed
    pr, qr = state.seeded_population(N, 128)
    small = tempering.TemperingChains(state.pq_to_columns(pr, qr),
                                      np.tile(tempering.geometric_ladder(0.2, 4.0, 16), 8), seed=3, ladder_size=16)
    tune_s = autotune.autotune(small, probe_sweeps=20)
    small.run(20, exchange_every=10, chains_per_block=tune_s.chains_per_block,
              threads_per_chain=tune_s.threads_per_chain)
    res = small.run(100, exchange_every=10, chains_per_block=tune_s.chains_per_block,
                    threads_per_chain=tune_s.threads_per_chain)
    small.validate()
    out["tempering_n75_128_chains"] = {"autotuned": {"threads_per_chain": tune_s.threads_per_chain,
                                                     "chains_per_block": tune_s.chains_per_block,
                                                     "shape_candidates_deltas_per_s": dict(tune_s.candidates)},
                                       "seconds": res.seconds, "deltas_per_s": res.proposals / res.seconds}
    launches += 2
    # C5: learned proposals, 2048 chains at n=75, 128 candidates per chain per step
    lp = learned.LearnedProposal(ch, seed=1, batch=4096)
    res = lp.run(300, exchange_every=300, train_every=10, block=50)
    st = lp.read_stats()
    tiles = ch.cols.shape[0]
    d = lp._descriptor()
    for _ in range(3):
        _lib.check(L.n3_mlp_infer(__import__("ctypes").byref(d), tiles, sptr), "n3_mlp_infer")
    a.record()
    for _ in range(10):
        _lib.check(L.n3_mlp_infer(__import__("ctypes").byref(d), tiles, sptr), "n3_mlp_infer")
    b.record()
    b.synchronize()
    infer_s = a.elapsed_time(b) / 1e3 / 10
    flop = 2.0 * tiles * 128 * (16 * 256 + 256 * 256)
    peaks, kind = measured_peaks()
    out["learned_n75_2048_chains"] = {"steps_per_s": 300 / res.seconds, "candidates_per_s": 300 * tiles * 128 /
                                      res.seconds, "mae_dE": st.mae, "accept_rate": st.accepted / max(1, st.proposals),
                                      "infer_kernel_us": infer_s * 1e6, "infer_tflops": flop / infer_s / 1e12,
                                      "infer_frac_of_bf16_peak": flop / infer_s / 1e12 / peaks["bf16_tflops"],
                                      "peak_kind": kind}
    launches += 13
    # learned vs plain: time to an energy level, seeds 1 and 2, 20 s of device time per
    # run (the full comparison over more seeds and budgets is --mode time-to-target)
    from no_three_in_line_b200 import compare

    budget, methods, seeds = 20.0, ("plain", "learned:x16:b85"), [1, 2]
    res = compare.compare(seeds, 12, budget, methods=methods)
    levels = {}
    for k, v in res["time_to_level"].items():
        if int(k) > 50:
            continue
        row = {m: (v[m]["median_s"] if v[m]["reached"] == len(seeds) else None) for m in methods}
        if row[methods[0]] is not None and row[methods[1]]:
            row["ratio"] = row[methods[0]] / row[methods[1]]
        levels[k] = row
    both = [k for k, r in levels.items() if "ratio" in r]
    out["time_to_level_short"] = {
        "workload": "n=75, 2048 chains, 32 ladders x 64 temperatures (0.05..5.0)",
        "methods": list(methods), "seeds": seeds, "budget_s_per_run": budget, "target": 12,
        "target_reached": {m: res[m]["reached"] for m in methods},
        "best_E_per_seed": {m: res[m]["best_per_seed"] for m in methods},
        "lowest_level_both_reach": min((int(k) for k in both), default=None),
        "median_ratio_plain_over_learned_at_that_level":
            levels[str(min(int(k) for k in both))]["ratio"] if both else None,
        "median_s_to_level": levels}
    return out, launches


def run_chain_mode(args):
    """One step = one exchange round (10 sweeps) of uniform-proposal tempering
    over 2048 n=75 chains in 64-temperature ladders (--mode tempering), or 50
    learned-proposal steps over the same chains (--mode learned)."""
    import torch

    from no_three_in_line_b200 import _lib, learned, state, tempering

    _lib.require_device()
    pc, qc = state.seeded_population(N, 2048)
    ch = tempering.TemperingChains(state.pq_to_columns(pc, qc), np.tile(tempering.geometric_ladder(0.05, 5.0, 64), 32),
                                   seed=1, ladder_size=64)
    if args.anneal_sweeps:
        ch.run(args.anneal_sweeps - args.anneal_sweeps % 10, exchange_every=10, sweeps_per_launch=100)
    e_start = ch.energy.float().mean().item()
    if args.mode == "tempering":
        step = lambda: ch.run(10, exchange_every=10, sweeps_per_launch=10)  # noqa: E731
        per_step, unit, what = 2048 * 150 * 10, "deltas/s", "exact swap deltas (proposals)"
    else:
        moves = int(args.learned_moves.split(",")[0])
        lp = learned.LearnedProposal(ch, seed=1, moves=moves, threads_per_chain=args.learned_threads)
        lp.run(50, exchange_every=50, train_every=10, block=50)
        step = lambda: lp.run(50, exchange_every=50, train_every=10, block=50, warm=False)  # noqa: E731
        per_step, unit, what = 2048 * 128 * 50, "candidates/s", "MLP-scored candidates"
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    secs = 0.0
    for _ in range(args.steps):
        secs += step().seconds
    ch.validate()
    line = {"metric": METRIC, "value": per_step * args.steps / secs, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32" if args.mode == "tempering" else "bf16",
            "data": "synthetic: random_state(75, Random(91001+c)) chain starts",
            "config": {"workload": f"n=75, 2048 chains, 32 ladders x 64 temperatures (0.05..5.0): {what}",
                       "mode": args.mode,
                       **({"moves_per_step": moves, "threads_per_chain": args.learned_threads}
                          if args.mode == "learned" else {}),
                       "anneal_sweeps": args.anneal_sweeps},
            "mean_E_at_start": e_start, "best_E": int(ch.best_energy.min().item())}
    print(json.dumps(line), flush=True)
    return 0


def run_search_mode(args):
    """--mode beam: one step = one generation of the device beam search at the
    reference CLI's defaults (gpu-search --engine device: population 32768,
    elite 64, max strength 12, energy window 12, bad bias 85; cli.py:1515-1527),
    n = 75, from random_state(75, Random(91001)).  --mode scan: one step = one
    n3_neighborhood_scan (every four-cycle and double switch, 4.67 M candidates)
    through the worst slot of that state."""
    from random import Random

    import torch

    from no_three_in_line_b200 import _lib, gpu_device_search, gpu_neighborhood, state

    _lib.require_device()
    init = state.random_state(N, Random(91001))
    stream = torch.cuda.current_stream()
    if args.mode == "beam":
        pop, elite = 32768, 64
        gens = args.warmup + args.steps
        beam = gpu_device_search.DeviceBeam(N, seed=1, population=pop, elite_size=elite, max_strength=12,
                                            energy_window=12, bad_bias=85, history_len=gens)
        beam.init(np.column_stack((init.P, init.Q)).astype(np.int32)[None])
        counter = iter(range(1, gens + 1))
        step = lambda: beam.generation(next(counter))  # noqa: E731
        per_step, unit, what = pop, "children/s", "device beam search generations (mutate, score, select, rank)"
        launches = 6
    else:
        anchor = gpu_neighborhood.bad_anchor_indices(init, 1)[0]
        dp = torch.tensor(init.P, dtype=torch.int32, device="cuda")
        dq = torch.tensor(init.Q, dtype=torch.int32, device="cuda")
        base = int(gpu_neighborhood.score_and_badness(np.asarray(init.P), np.asarray(init.Q))[0])
        out = torch.empty(4, dtype=torch.int64, device="cuda")
        L = _lib.lib()
        step = lambda: _lib.check(L.n3_neighborhood_scan(dp.data_ptr(), dq.data_ptr(), N, anchor, base,  # noqa: E731
                                                         out.data_ptr(), out.data_ptr() + 16,
                                                         int(stream.cuda_stream)), "n3_neighborhood_scan")
        per_step, unit, what = 64824 * 8 * 9, "candidates/s", "four-cycle + double-switch candidates scored exactly"
        launches = 1
    for _ in range(max(3, args.warmup) if args.mode == "scan" else args.warmup):
        step()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        end.synchronize()
    secs = start.elapsed_time(end) / 1e3
    line = {"metric": METRIC, "value": per_step * args.steps / secs, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic: random_state(75, Random(91001))",
            "config": {"workload": f"n=75: {what}", "mode": args.mode}, "gpu_launches": launches * args.steps,
            "clocks": clocks.summary()}
    if args.mode == "beam":
        line["best_E"] = int(beam.read_status()[1])
    print(json.dumps(line), flush=True)
    return 0


def run_lines_mode(args):
    """--mode lines: the line tables of the 75 x 75 grid (precompute.py:35-57)
    built once on the device (timed alone), then one step = score_pair_table and
    score_csr (:60-89) of 4096 seeded n = 75 states, inputs resident in HBM."""
    import torch

    from no_three_in_line_b200 import _lib, gpu, precompute, state

    _lib.require_device()
    stream = torch.cuda.current_stream()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    precompute.build_geometry_tables(N)  # warm-up: module load, allocator
    torch.cuda.synchronize()
    t0.record(stream)
    tables = precompute.build_geometry_tables(N)
    t1.record(stream)
    t1.synchronize()
    build_ms = t0.elapsed_time(t1)
    p, q = state.seeded_population(N, args.states)
    ids = np.concatenate(precompute._population_ids(p, q, N))
    dev = torch.device("cuda")
    d_ids = torch.from_numpy(ids).to(dev)
    d_starts = torch.arange(0, 2 * N * (args.states + 1), 2 * N, dtype=torch.int64, device=dev)
    d = tables.device
    pair_scores = torch.empty(args.states, dtype=torch.int64, device=dev)
    csr_scores = torch.empty_like(pair_scores)
    occ = torch.empty(((args.states + 31) // 32) * N * N, dtype=torch.int32, device=dev)
    err = torch.zeros(2, dtype=torch.int32, device=dev)
    L = _lib.lib()
    sp = int(stream.cuda_stream)

    def step():
        _lib.check(L.n3_lines_score_pairs(d_ids.data_ptr(), d_starts.data_ptr(), args.states, N,
                                          d.pair_to_line.data_ptr(), pair_scores.data_ptr(), err.data_ptr(), sp),
                   "n3_lines_score_pairs")
        _lib.check(L.n3_lines_score_csr(d_ids.data_ptr(), d_starts.data_ptr(), args.states, N, tables.line_count,
                                        d.offsets.data_ptr(), d.indices.data_ptr(), occ.data_ptr(),
                                        csr_scores.data_ptr(), err.data_ptr() + 4, sp), "n3_lines_score_csr")

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    want = np.asarray(gpu.score_population_gpu(p, q))
    if not (np.array_equal(pair_scores.cpu().numpy(), want) and np.array_equal(csr_scores.cpu().numpy(), want)
            and int(err.abs().sum()) == 0):
        raise AssertionError("line-table scores differ from the determinant scores")
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        end.synchronize()
    secs = start.elapsed_time(end) / 1e3
    # each scorer alone (events around each call), and the L2 random-gather rate
    # of the pair table itself as the pair scorer's ceiling
    pair_ev, csr_ev = [], []
    for _ in range(5):
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record(stream)
        _lib.check(L.n3_lines_score_pairs(d_ids.data_ptr(), d_starts.data_ptr(), args.states, N,
                                          d.pair_to_line.data_ptr(), pair_scores.data_ptr(), err.data_ptr(), sp),
                   "n3_lines_score_pairs")
        b.record(stream)
        _lib.check(L.n3_lines_score_csr(d_ids.data_ptr(), d_starts.data_ptr(), args.states, N, tables.line_count,
                                        d.offsets.data_ptr(), d.indices.data_ptr(), occ.data_ptr(),
                                        csr_scores.data_ptr(), err.data_ptr() + 4, sp), "n3_lines_score_csr")
        c.record(stream)
        pair_ev.append((a, b))
        csr_ev.append((b, c))
    torch.cuda.synchronize()
    pair_s = statistics.mean(x.elapsed_time(y) for x, y in pair_ev[1:]) / 1e3
    csr_s = statistics.mean(x.elapsed_time(y) for x, y in csr_ev[1:]) / 1e3
    gathers_per_state = math.comb(2 * N, 2)
    scratch = torch.zeros(2, dtype=torch.int64, device=dev)
    entries = int(d.pair_to_line.numel())
    blocks = torch.cuda.get_device_properties(dev).multi_processor_count * 8
    iters = 2048
    _lib.check(L.n3_calibrate_l2_gather(d.pair_to_line.data_ptr(), entries, blocks, iters, scratch.data_ptr(), sp),
               "l2 gather")
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(5):
        _lib.check(L.n3_calibrate_l2_gather(d.pair_to_line.data_ptr(), entries, blocks, iters, scratch.data_ptr(),
                                            sp), "l2 gather")
    g1.record(stream)
    torch.cuda.synchronize()
    gather_peak = blocks * 256 * iters * 5 / (g0.elapsed_time(g1) / 1e3)
    pair_gathers = args.states * gathers_per_state / pair_s
    lookups = (args.states + 31) // 32 * int(len(tables.indices))
    line = {"metric": METRIC, "value": args.states * args.steps / secs, "unit": "states/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic: random_state(75, Random(91001+i)) states",
            "config": {"workload": f"n=75 line tables: score_pair_table + score_csr of {args.states} states",
                       "mode": "lines", "line_count": tables.line_count, "line_incidences": int(len(tables.indices)),
                       "pair_table_bytes": int(tables.pair_to_line.nbytes)},
            "table_build_ms_with_host_copies": build_ms, "gpu_launches": 3 * args.steps,
            "gpu_launches_note": "3 kernels per step (pair scorer; occupancy + CSR scorer); each step also issues "
                                 "2 cudaMemsetAsync (the occupancy words and the scores)",
            "per_scorer": {"pair_table_us": pair_s * 1e6, "csr_us": csr_s * 1e6,
                           "pair_gathers_per_s": pair_gathers,
                           "csr_occupancy_lookups_per_s": lookups / csr_s},
            "roofline": {"bound": "L2 random 4-byte gathers (pair-table scorer)",
                         "kernel": "n3::lines::pair_score_kernel", "achieved": pair_gathers / 1e9,
                         "peak": gather_peak / 1e9, "unit": "G gathers/s", "frac": pair_gathers / gather_peak,
                         "peak_source": "measured on this GPU: n3_calibrate_l2_gather, xorshift-indexed 4-byte "
                                        f"loads from the {entries * 4 / 1e6:.0f} MB pair table itself (L2-resident)",
                         "algorithmic": f"C(150,2) = {gathers_per_state} pair-table gathers per n=75 state"},
            "clocks": clocks.summary(),
            "cpu_baseline": lines_cpu_baseline(tables, p, q)}
    print(json.dumps(line), flush=True)
    return 0


def run_exhaustive_mode(args):
    """--mode exhaustive: gpu_exhaustive_beam_search (gpu_exhaustive_beam.py:91-325)
    at the reference CLI defaults (elite 64, energy window 12, global anchors
    every 25 generations) from a seeded n = 75 state; one step = one
    generation: every legal 2-switch of every elite through a bad slot scored
    exactly on the device, pooled, shuffled, and the host's retention step.
    Timed by the host clock per generation (the retention step is host work)."""
    from random import Random

    from no_three_in_line_b200 import gpu_exhaustive_beam, state

    snaps = []
    total = max(3, args.warmup) + args.steps
    gpu_exhaustive_beam.gpu_exhaustive_beam_search(state.random_state(N, Random(91001)), seed=1, generations=total,
                                                   elite_size=64, energy_window=12, global_every=25,
                                                   report_every=1, callback=snaps.append)
    timed = snaps[-args.steps - 1:]
    secs = timed[-1].elapsed_seconds - timed[0].elapsed_seconds
    evals = timed[-1].evaluations - timed[0].evaluations
    steps = len(timed) - 1
    line = {"metric": METRIC, "value": evals / secs, "unit": "exact children scored/s", "n_gpus": 1,
            "steps": steps, "warmup": len(snaps) - steps, "ms_per_step": 1e3 * secs / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic: random_state(75, Random(91001)) initial state",
            "config": {"workload": "exhaustive 2-switch beam, n=75, elite 64, window 12, global every 25",
                       "mode": "exhaustive", "children_per_generation": evals / steps},
            "best_E": timed[-1].best_score,
            "timing": "host clock between generation reports (device work and the host retention step)"}
    print(json.dumps(line), flush=True)
    return 0


def run_time_to_target(args):
    from no_three_in_line_b200 import compare

    methods = tuple(m.strip() for m in args.methods.split(",") if m.strip())
    res = compare.compare(list(range(1, args.seeds + 1)), args.target, args.budget, methods=methods, log=args.log)
    line = {"metric": "time-to-E<=target, learned vs plain proposal (n=75, 2048 chains, 64-temperature ladders)",
            "unit": "s", "higher_is_better": False, "target": args.target, "budget_s": args.budget,
            **{k: v for k, v in res.items() if k.startswith("plain") or k.startswith("learned")},
            "common_level": res["common_level"], "time_to_level": res["time_to_level"],
            "data": "synthetic: random_state(75, Random(91001+c)) chain starts",
            "runs": [{k: r[k] for k in ("method", "seed", "reached", "seconds", "best", "mae")} for r in res["runs"]],
            "trajectories": {f'{r["method"]}-{r["seed"]}': r["trajectory"][::max(1, len(r["trajectory"]) // 40)]
                             for r in res["runs"]}}
    print(json.dumps(line), flush=True)
    return 0


def run_reference(args):
    """CPU arm: the reference algorithm (oracle port) on all host threads."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = host_threads()
    p, q, _ = population(N, args.states, 0)
    cpu = cpu_reference_rate(p, q, threads=threads, steps=args.steps, warmup=args.warmup)
    value = cpu["value"]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": cpu["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic: random_state(75, Random(91001+i)) states (the reference's seeding)",
            "config": bench_config(args.states, world),
            "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_b200(args):
    import torch
    import torch.distributed as dist

    from no_three_in_line_b200 import _lib

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", torch.cuda.current_device())
    L = _lib.lib()
    _lib.require_device()
    B = args.states
    p, q, cols_host = population(N, B, rank)
    cols = torch.from_numpy(cols_host).to(dev)
    scores = torch.empty(B, dtype=torch.int32, device=dev)
    badness = torch.empty((B, 2 * N), dtype=torch.int32, device=dev)
    flags = torch.zeros(2, dtype=torch.int32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    sptr = int(stream.cuda_stream)

    def step():
        if args.mode == "det":
            _lib.check(L.n3_score_columns(cols.data_ptr(), B, N, scores.data_ptr(), None, sptr), "n3_score_columns")
        elif args.mode == "slope":
            _lib.check(L.n3_score_slope(cols.data_ptr(), B, N, scores.data_ptr(), badness.data_ptr(), sptr),
                       "n3_score_slope")
        else:
            _lib.check(L.n3_score_checked(cols.data_ptr(), B, N, scores.data_ptr(), badness.data_ptr(),
                                          flags.data_ptr(), flags.data_ptr() + 4, sptr), "n3_score_checked")

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    # correctness gate before timing: bit-exact against the oracle on a sample
    from oracle import oracle

    ref = oracle.score_population(p[:64], q[:64], threads=0)
    got = scores[:64].cpu().numpy()
    if not np.array_equal(ref, got) or int(flags[0].item()) != 0:
        raise AssertionError("scores differ from the oracle; refusing to time")

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clocks:
        wall0 = time.perf_counter()
        for k in range(args.steps):
            flush.fill_(k)  # evict the population from L2 between steps
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    local_total = sum(step_ms)
    t_total = torch.tensor([local_total], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_total, op=dist.ReduceOp.MAX)
    total_ms = float(t_total.item())
    if int(flags[0].item()) != 0:
        raise AssertionError("device cross-check reported a mismatch during timing")
    value = world * B * args.steps / (total_ms / 1e3)

    # end to end through the C ABI with host buffers: every step copies its
    # population from pinned host memory and reads its scores and flags back.
    # The copies run on a second stream beside the compute: the population of
    # step k + 1 into the other of two device buffers while step k computes (a
    # copy waits until the compute that last used its buffer is done), and the
    # read-back of step k's scores and flags (two result buffers, so that step
    # k + 1 writes the other) while step k + 1 computes.
    h_cols = torch.from_numpy(cols_host).pin_memory()
    h_scores = torch.empty(B, dtype=torch.int32).pin_memory()
    h_flags = torch.empty(2, dtype=torch.int32).pin_memory()
    d_bufs = [torch.empty_like(cols), torch.empty_like(cols)]
    r_scores = [scores, torch.empty_like(scores)]
    r_flags = [flags, torch.zeros_like(flags)]
    copy_stream = torch.cuda.Stream(device=dev)
    e2e_steps = max(3, min(args.steps, 100))

    def e2e_run(steps):
        ready = [torch.cuda.Event(), torch.cuda.Event()]
        free = [torch.cuda.Event(), torch.cuda.Event()]    # step done with its input buffer and result buffers
        read = [torch.cuda.Event(), torch.cuda.Event()]    # result buffers copied to the host
        copy_stream.wait_stream(stream)
        with torch.cuda.stream(copy_stream):
            d_bufs[0].copy_(h_cols, non_blocking=True)
            ready[0].record(copy_stream)
        for k in range(steps):
            b = k & 1
            if k + 1 < steps:
                with torch.cuda.stream(copy_stream):
                    if k >= 1:
                        copy_stream.wait_event(free[1 - b])
                    d_bufs[1 - b].copy_(h_cols, non_blocking=True)
                    ready[1 - b].record(copy_stream)
            stream.wait_event(ready[b])
            if k >= 2:
                stream.wait_event(read[b])
            _lib.check(L.n3_score_checked(d_bufs[b].data_ptr(), B, N, r_scores[b].data_ptr(), badness.data_ptr(),
                                          r_flags[b].data_ptr(), r_flags[b].data_ptr() + 4, sptr),
                       "n3_score_checked")
            free[b].record(stream)
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(free[b])
                h_scores.copy_(r_scores[b], non_blocking=True)
                h_flags.copy_(r_flags[b], non_blocking=True)
                read[b].record(copy_stream)
        stream.wait_stream(copy_stream)  # the last read-back is inside the timed region

    e2e_run(2)
    torch.cuda.synchronize()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    e2e_run(e2e_steps)
    e_end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e_start.elapsed_time(e_end) / e2e_steps
    if not np.array_equal(h_scores[:64].numpy(), ref) or int(r_flags[0][0].item()) or int(r_flags[1][0].item()):
        raise AssertionError("end-to-end scores differ from the oracle")
    t_e2e = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_e2e, op=dist.ReduceOp.MAX)
    e2e_ms = float(t_e2e.item())

    # the dominant kernel alone (the determinant count), for the roofline
    det_ms = []
    for k in range(12):
        flush.fill_(k)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        _lib.check(L.n3_score_columns(cols.data_ptr(), B, N, scores.data_ptr(), None, sptr), "n3_score_columns")
        b.record(stream)
        det_ms.append((a, b))
    torch.cuda.synchronize()
    det_ms = [a.elapsed_time(b) for a, b in det_ms[2:]]
    det_launch_s = statistics.mean(det_ms) / 1e3

    # integer-pipe ceilings: each pipe alone (multiply-add chains, logic-op
    # chains), and the scorer's own expression on registers
    scratch = torch.zeros(2, dtype=torch.int64, device=dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count

    def timed_rate(launch, ops_per_launch, reps=5):
        launch()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(reps):
            launch()
        c1.record(stream)
        torch.cuda.synchronize()
        return ops_per_launch * reps / (c0.elapsed_time(c1) / 1e3)

    blocks, iters = sms * 8, 4096
    pipe_rate = {}
    for kind, name in ((0, "imad"), (1, "alu")):
        pipe_rate[name] = timed_rate(
            lambda k=kind: _lib.check(L.n3_calibrate_int_pipe(k, blocks, iters, scratch.data_ptr(), sptr), "pipe"),
            blocks * 256 * iters * 8)
    ceiling_tests = timed_rate(
        lambda: _lib.check(L.n3_calibrate_det_ceiling(blocks, iters, scratch.data_ptr(), sptr), "calibrate"),
        blocks * 256 * iters * 16)

    line = None
    if rank == 0:
        ms_per_step = total_ms / args.steps
        tests_per_s = value * TESTS_PER_STATE
        # the determinant kernel's own launches: 4096 states x 540,200 tested triples
        kernel_tests = B * KERNEL_TESTS_PER_STATE / det_launch_s
        pipe_tests = min(pipe_rate["imad"], pipe_rate["alu"])  # one op of each pipe per test
        achieved = kernel_tests * OPS_PER_TEST / 1e9
        peak = pipe_tests * OPS_PER_TEST / 1e9
        peaks, peak_kind = measured_peaks()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32",
            "data": "synthetic: random_state(75, Random(91001+i)) states (the reference's seeding), resident in HBM",
            "config": dict(bench_config(B, world), **({} if args.mode == "checked" else
                                                          {"workload": f"{WORKLOAD} ({args.mode} kernel only)"})),
            "triple_tests_per_s": tests_per_s,
            "e2e": {"value": world * B / (e2e_ms / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(cols_host.nbytes),
                    "d2h_bytes_per_step": int(h_scores.numel() * 4 + h_flags.numel() * 4),
                    "copies": "pinned host buffers; H2D of step k+1 and read-back of step k on a second stream beside the compute"},
            "gpu_launches": args.steps * (2 if args.mode == "checked" else 1),
            "roofline": {"bound": "int32 pipes (FMA pipe for products, ALU pipe for compares)",
                         "kernel": "n3::det_kernel<ColSource,false> (the larger of the checked step's two "
                                   "launches; the other is n3::slope4_kernel<2>), timed alone",
                         "kernel_launch_us": det_launch_s * 1e6,
                         "kernel_tests_per_s": kernel_tests,
                         "achieved": achieved, "peak": peak, "unit": "Gop/s", "frac": achieved / peak,
                         "peak_source": "measured on this GPU: n3_calibrate_int_pipe, multiply-add chains "
                                        f"{pipe_rate['imad'] / 1e12:.2f} Top/s and logic-op chains "
                                        f"{pipe_rate['alu'] / 1e12:.2f} Top/s; 2 ops per tested triple (one "
                                        "product share on the FMA pipe, one compare on the ALU pipe), "
                                        f"{KERNEL_TESTS_PER_STATE} tested triples per state",
                         "expression_ceiling": {"tests_per_s": ceiling_tests,
                                                "frac": kernel_tests / ceiling_tests,
                                                "source": "n3_calibrate_det_ceiling: the scorer's test "
                                                          "expression with per-test counting, on registers"},
                         "traffic": DET_TRAFFIC_BYTES,
                         "hbm_context": {"bytes_per_step": int(cols_host.nbytes + B * 4 + B * 2 * N * 4),
                                         "hbm_gbs_peak": peaks.get("hbm_gbs"), "peak_kind": peak_kind}},
            "wall_s_timed": wall,
            "clocks": clocks.summary(),
        }
        # the same CPU timing as the reference arm, on a bounded sample (3 passes)
        line["cpu_baseline"] = cpu_reference_rate(p, q, threads=host_threads(), steps=3, warmup=2)
        if world == 1 and not args.no_secondary and args.mode == "checked":
            line["secondary"], extra = secondary_measurements(dev, p, q)
            line["secondary"]["note"] = ("measured after the timed region; not part of value, e2e or gpu_launches")
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    from __graft_entry__ import load_package

    load_package()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "time-to-target":
        return run_time_to_target(args)
    if args.mode in ("tempering", "learned"):
        return run_chain_mode(args)
    if args.mode in ("beam", "scan"):
        return run_search_mode(args)
    if args.mode == "lines":
        return run_lines_mode(args)
    if args.mode == "exhaustive":
        return run_exhaustive_mode(args)
    return run_b200(args)


if __name__ == "__main__":
    raise SystemExit(main())
