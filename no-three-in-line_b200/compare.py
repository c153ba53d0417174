"""Time to a target energy: uniform-proposal tempering against learned-proposal
tempering on the same GPU, chains and seeds.

Both start from the same seeded states (random_state(n, Random(91001 + c))),
the same temperature ladders and the same exchange schedule (every 10 sweeps of
2n proposals).  The clock is the device's: CUDA events around the launches,
with the target checked at launch boundaries (plain: inside the kernel, at the
first exchange round after some chain reaches the target; learned: after each
block of steps).  A run that does not reach the target within its budget is
reported as censored at the budget.
"""
from __future__ import annotations

import json
import statistics
import time
from dataclasses import asdict, dataclass

import numpy as np

from . import state, tempering


@dataclass
class TargetRun:
    method: str
    seed: int
    target: int
    reached: bool
    seconds: float           # device time to the hit, or the time spent when censored
    best: int
    trajectory: list          # (device seconds, best E) after each launch or block


def seeded_chains(n: int, chains: int, ladder: int, seed: int, tmin: float = 0.05, tmax: float = 5.0):
    p, q = state.seeded_population(n, chains)
    temps = np.tile(tempering.geometric_ladder(tmin, tmax, ladder), chains // ladder)
    return tempering.TemperingChains(state.pq_to_columns(p, q), temps, seed, ladder_size=ladder)


def run_plain(seed: int, target: int, budget: float, *, n=75, chains=2048, ladder=64, block_sweeps=100,
              bad_bias=0, name=None):
    """Uniform-proposal tempering (config 3); with ``bad_bias`` that share of
    proposals draws slot u by badness, the reference walk's option."""
    name = name or ("plain" if not bad_bias else f"plain:b{bad_bias}")
    ch = seeded_chains(n, chains, ladder, seed)
    traj, spent = [], 0.0
    while spent < budget:
        res = ch.run(block_sweeps, exchange_every=10, target=target, sweeps_per_launch=block_sweeps,
                     bad_bias=bad_bias)
        if res.hit is not None:
            spent += res.hit[2]
            traj.append((spent, res.best))
            return TargetRun(name, seed, target, True, spent, res.best, traj)
        spent += res.seconds
        traj.append((spent, res.best))
    return TargetRun(name, seed, target, False, spent, int(ch.best_energy.min().item()), traj)


def run_learned(seed: int, target: int, budget: float, *, n=75, chains=2048, ladder=64, block=50,
                train_every=10, moves=1, exchange_steps=None, bad_bias=0, name=None):
    """Learned-proposal tempering; `moves` > 1 draws that many moves per step
    (without replacement) from each step's scored candidates; ``bad_bias``
    draws that share of the candidates' slot u by badness.  The run's
    proposal MAE (|predicted - exact dE| over every learned proposal) is kept."""
    from .learned import LearnedProposal

    ch = seeded_chains(n, chains, ladder, seed)
    lp = LearnedProposal(ch, seed=seed, moves=moves, bad_bias=bad_bias)
    if name is None:
        name = "learned" if moves == 1 else f"learned:x{moves}"
        name += f":b{bad_bias}" if bad_bias else ""
    # exchange every 10 sweeps, a sweep being 2n learned steps (scoring passes);
    # with moves > 1 each step makes up to `moves` proposals
    every = exchange_steps if exchange_steps else 10 * 2 * n
    traj, spent, first = [], 0.0, True
    abs_err = count = 0.0
    reached = False
    while spent < budget:
        res = lp.run(every, exchange_every=every, train_every=train_every, block=block, target=target, warm=first)
        first = False
        st = lp.read_stats()
        abs_err += st.mae * st.proposals
        count += st.proposals
        if res.hit is not None:
            spent += res.hit[2]
            traj.append((spent, res.best))
            reached = True
            break
        spent += res.seconds
        traj.append((spent, res.best))
    best = traj[-1][1] if reached else int(ch.best_energy.min().item())
    run = TargetRun(name, seed, target, reached, spent, best, traj)
    run.mae = abs_err / max(1.0, count)
    return run


def parse_method(spec: str) -> dict:
    """``plain``, ``plain:b85``, ``learned``, ``learned:x16``, ``learned:x16:b85``."""
    parts = spec.split(":")
    if parts[0] not in ("plain", "learned"):
        raise ValueError(f"unknown method {spec!r}")
    out = {"kind": parts[0], "moves": 1, "bad_bias": 0, "name": spec}
    for p in parts[1:]:
        if p.startswith("x") and parts[0] == "learned":
            out["moves"] = int(p[1:])
        elif p.startswith("b"):
            out["bad_bias"] = int(p[1:])
        else:
            raise ValueError(f"unknown method option {p!r} in {spec!r}")
    return out


def time_to_reach(traj, level: int):
    """Device seconds until the best energy first reached <= level (None if never)."""
    for t, e in traj:
        if e <= level:
            return t
    return None


def compare(seeds, target: int, budget: float, *, methods=("plain", "learned"), log=None, **kw) -> dict:
    """Every method on every seed; with ``log`` (a path) each finished run is
    appended to it as one JSON line, so an interrupted comparison keeps its runs."""
    specs = [parse_method(m) for m in methods]
    runs = []
    for s in seeds:
        for sp in specs:
            if sp["kind"] == "plain":
                runs.append(run_plain(s, target, budget, bad_bias=sp["bad_bias"], name=sp["name"], **kw))
            else:
                runs.append(run_learned(s, target, budget, moves=sp["moves"], bad_bias=sp["bad_bias"],
                                        name=sp["name"], **kw))
            if log is not None:
                with open(log, "a", encoding="utf-8") as f:
                    f.write(json.dumps(dict(asdict(runs[-1]), mae=getattr(runs[-1], "mae", None))) + "\n")
    out = {"target": target, "budget_s": budget, "runs": [dict(asdict(r), mae=getattr(r, "mae", None))
                                                          for r in runs]}
    names = [sp["name"] for sp in specs]
    for method in names:
        rs = [r for r in runs if r.method == method]
        out[method] = {"median_s": statistics.median(r.seconds for r in rs),
                       "reached": sum(r.reached for r in rs), "seeds": len(rs),
                       "median_best": statistics.median(r.best for r in rs),
                       "best_per_seed": sorted(r.best for r in rs)}
        maes = [r.mae for r in rs if getattr(r, "mae", None) is not None]
        if maes:
            out[method]["proposal_mae"] = statistics.mean(maes)
    # the lowest level every run reached, and the time each method took to it
    common = max(r.best for r in runs)
    out["common_level"] = common
    for method in names:
        times = [time_to_reach(r.trajectory, common) for r in runs if r.method == method]
        out[method]["median_s_to_common_level"] = statistics.median(times)
    # time to each level of a ladder of energies, censored at the budget
    levels = list(range(max(r.trajectory[0][1] for r in runs if r.trajectory), min(r.best for r in runs) - 1, -1))
    ladder = {}
    for level in levels:
        row = {}
        for method in names:
            ts = [time_to_reach(r.trajectory, level) for r in runs if r.method == method]
            row[method] = {"median_s": statistics.median(budget if t is None else t for t in ts),
                           "reached": sum(t is not None for t in ts)}
        ladder[str(level)] = row
    out["time_to_level"] = ladder
    return out


if __name__ == "__main__":  # pragma: no cover
    print(json.dumps(compare([1, 2, 3], 12, 30.0)))
