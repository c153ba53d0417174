"""Device beam search on the GPU (gpu_device_search.py:17-432) against the
golden trajectory written from the reference's own mutation kernel source,
rank_elites and random.Random (tests/golden/make_golden_beam.py), and against
the CPU oracle on further configurations.  Integer work: bit-exact."""
from __future__ import annotations

from random import Random

import numpy as np
import pytest

from no_three_in_line_b200 import gpu_device_search as gds
from no_three_in_line_b200 import state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def beam_golden(golden):
    return golden("beam_golden.npz")


@pytest.mark.parametrize("seed", [0, 1, 7, 91001, 2**32 + 5, 2**63 + 12345])
@pytest.mark.parametrize("count", [0, 1, 2, 3, 17, 1000, 40000])
def test_device_shuffle_is_cpython_shuffle(cuda, seed, count):
    values = list(range(count))
    Random(seed).shuffle(values)
    got = gds.py_random_shuffle_device(np.arange(count), seed)
    assert np.array_equal(got, np.asarray(values))


def test_device_mutation_matches_reference_kernel(cuda, beam_golden):
    g = beam_golden
    cp_, cq_ = gds.mutate_population_device(g["mut_parent_p"], g["mut_parent_q"], population=64, active_strength=3,
                                            max_strength=6, seed=5, generation=2)
    assert np.array_equal(cp_, g["mut_child_p"]) and np.array_equal(cq_, g["mut_child_q"])


@pytest.mark.parametrize("parents,population,badness", [
    (40, 1000, "states"),    # prefix sums staged per CTA; a ragged last CTA
    (200, 777, "states"),    # 200 n=75 parents exceed the staged prefix sums: linear scan
    (12, 300, "zeros"),      # zero badness in runs, some parents with none at all
    (12, 300, "negative"),   # a negative badness: the CTA falls back to the linear scan
])
def test_mutation_roulette_paths_match_oracle(cuda, oracle, parents, population, badness):
    """n3_beam_mutate through the C ABI against the oracle's restatement of the
    mutation kernel, with the parents' badness given explicitly."""
    import torch

    from no_three_in_line_b200 import _lib

    n, rng = 75, np.random.default_rng(parents + population)
    states = [state.random_state(n, Random(300 + k)) for k in range(parents)]
    pp = np.asarray([s.P for s in states], np.int32)
    pq = np.asarray([s.Q for s in states], np.int32)
    bad = rng.integers(0, 9, size=(parents, 2 * n)).astype(np.int32)
    if badness == "zeros":
        bad[:, 10:90] = 0
        bad[::3] = 0
    elif badness == "negative":
        bad[5, 17] = -3
    quality = max(1, parents // 4)
    args = dict(quality_count=quality, population=population, active_strength=4, max_strength=9, bad_bias=85,
                seed=2**40 + 77, generation=3)
    ref_p, ref_q = oracle.beam_mutate(pp, pq, bad, **args)
    dev = torch.device("cuda", 0)
    dp, dq, db = (torch.from_numpy(x).to(dev) for x in (pp, pq, bad))
    cp_ = torch.empty((population, n), dtype=torch.int32, device=dev)
    cq_ = torch.empty_like(cp_)
    _lib.call("n3_beam_mutate", _lib.ptr(dp), _lib.ptr(dq), _lib.ptr(db), parents, quality, n, population,
              args["active_strength"], args["max_strength"], args["bad_bias"], args["seed"], args["generation"],
              _lib.ptr(cp_), _lib.ptr(cq_), None)
    assert np.array_equal(cp_.cpu().numpy(), ref_p) and np.array_equal(cq_.cpu().numpy(), ref_q)


def run_device(initial_p, initial_q, extra, *, seed, generations, population, elite_size, max_strength,
               energy_window, bad_bias=85):
    """Generation by generation through DeviceBeam, reading the ranked elites back."""
    base = np.column_stack((initial_p, initial_q)).astype(np.int32)[None]
    if extra is not None:
        base = np.concatenate((base, np.asarray(extra, np.int32)), axis=0)
    base = base[:elite_size]
    beam = gds.DeviceBeam(len(initial_p), seed=seed, population=population, elite_size=elite_size,
                          max_strength=max_strength, energy_window=energy_window, bad_bias=bad_bias,
                          history_len=generations)
    beam.init(base)
    out = {"generation_best": [], "best_history": [], "elite_scores": [], "elite_p": [], "elite_q": []}
    for gen in range(1, generations + 1):
        beam.generation(gen)
        st = beam.read_status()
        if int(st[5]) != gen:
            break
        out["generation_best"].append(int(st[6]))
        out["best_history"].append(int(st[1]))
        out["elite_scores"].append(beam.elite_scores.cpu().numpy())
        out["elite_p"].append(beam.elite_p.cpu().numpy())
        out["elite_q"].append(beam.elite_q.cpu().numpy())
    st = beam.read_status()
    out.update(completed=int(st[5]), best_score=int(st[1]), best_p_raw=beam.best_p.cpu().numpy(),
               best_q_raw=beam.best_q.cpu().numpy(), history=beam.history.cpu().numpy())
    return out


@pytest.mark.parametrize("name", ["a", "b"])
def test_device_beam_trajectory_matches_reference(cuda, beam_golden, name):
    g = beam_golden
    n, seed, gens, pop, elite, max_s, window = map(int, g[f"{name}_config"])
    res = run_device(g[f"{name}_initial_p"], g[f"{name}_initial_q"], g.get(f"{name}_extra"), seed=seed,
                     generations=gens, population=pop, elite_size=elite, max_strength=max_s, energy_window=window)
    assert res["completed"] == int(g[f"{name}_completed"])
    assert res["best_score"] == int(g[f"{name}_best_score"])
    assert np.array_equal(res["generation_best"], g[f"{name}_generation_best"])
    assert np.array_equal(res["best_history"], g[f"{name}_best_history"])
    assert np.array_equal(np.stack(res["elite_scores"]), g[f"{name}_elite_scores"])
    assert np.array_equal(np.stack(res["elite_p"]), g[f"{name}_elite_p"])
    assert np.array_equal(np.stack(res["elite_q"]), g[f"{name}_elite_q"])
    assert np.array_equal(res["best_p_raw"], g[f"{name}_best_p_raw"])
    assert np.array_equal(res["history"][:gens, 0], g[f"{name}_generation_best"])


def test_public_search_result_matches_reference(cuda, beam_golden):
    g = beam_golden
    n, seed, gens, pop, elite, max_s, window = map(int, g["a_config"])
    init = state.PairPermutations(tuple(g["a_initial_p"].tolist()), tuple(g["a_initial_q"].tolist()))
    snaps = []
    res = gds.gpu_device_beam_search(init, seed=seed, generations=gens, population=pop, elite_size=elite,
                                     max_strength=max_s, energy_window=window, initial_elites=g["a_extra"],
                                     callback=snaps.append)
    assert res.score == int(g["a_best_score"]) and res.generations == int(g["a_completed"])
    assert res.evaluations == int(g["a_evaluations"])
    assert list(res.state.P) == g["a_best_p"].tolist() and list(res.state.Q) == g["a_best_q"].tolist()
    # snapshots on every report_every-th generation (and on improvements), as the reference reports
    assert {s.generation for s in snaps} >= set(range(5, gens + 1, 5))
    for s in snaps:
        assert s.best_score == int(g["a_best_history"][s.generation - 1])
        assert s.elite_scores == tuple(int(x) for x in g["a_elite_scores"][s.generation - 1])


@pytest.mark.parametrize("cfg", [
    dict(n=30, seed=123, generations=8, population=3000, elite_size=32, max_strength=8, energy_window=6),
    dict(n=12, seed=5, generations=12, population=64, elite_size=64, max_strength=4, energy_window=0, bad_bias=0),
    dict(n=50, seed=99, generations=5, population=4096, elite_size=200, max_strength=12, energy_window=40,
         bad_bias=100),
])
def test_device_beam_matches_oracle(cuda, oracle, cfg):
    cfg = dict(cfg)
    n = cfg.pop("n")
    init = state.random_state(n, Random(91001 + n))
    extra = np.asarray([np.column_stack((s.P, s.Q)) for s in
                        (state.random_state(n, Random(7 + k)) for k in range(2))], np.int32)
    ref = oracle.beam_search(np.asarray(init.P, np.int32), np.asarray(init.Q, np.int32), extra, **cfg)
    got = run_device(np.asarray(init.P, np.int32), np.asarray(init.Q, np.int32), extra, **cfg)
    assert got["completed"] == ref["completed"] and got["best_score"] == ref["best_score"]
    assert np.array_equal(got["generation_best"], ref["generation_best"])
    assert np.array_equal(np.stack(got["elite_scores"]), np.stack(ref["elite_scores"]))
    assert np.array_equal(np.stack(got["elite_p"]), np.stack(ref["elite_p"]))
    assert np.array_equal(np.stack(got["elite_q"]), np.stack(ref["elite_q"]))
    assert np.array_equal(got["best_p_raw"], ref["best_p_raw"])


def test_rejects_unsupported_sizes(cuda):
    init = state.random_state(10, Random(1))
    with pytest.raises(ValueError):
        gds.gpu_device_beam_search(init, seed=1, generations=1, population=8, elite_size=1, max_strength=2,
                                   energy_window=2)
    with pytest.raises(ValueError):
        gds.gpu_device_beam_search(init, seed=1, generations=1, population=70000, elite_size=8, max_strength=2,
                                   energy_window=2)


def cpython_steps(counts, seed):
    """The j of every step of random.Random(seed).shuffle, for each count in turn."""
    rng = Random(seed)
    out = []
    for count in counts:
        js = [0] * count
        for i in reversed(range(1, count)):
            js[i] = rng._randbelow(i + 1)
        out.append(np.asarray(js, np.int32))
    return out


@pytest.mark.parametrize("seed", [0, 7, 91001, 2**63 + 12345])
def test_shuffle_draws_resolved_by_the_cta_are_cpythons(cuda, seed):
    """The CTA-wide resolver (wide draw widths) and the warp (the last steps),
    over one generator: counts across block, batch and width boundaries, a
    fresh and a part-used state, the largest count."""
    counts = [0, 1, 2, 3, 257, 300, 1000, 4097, 5000, 12345, 40000, 65536, 511, 70]
    got = gds.py_shuffle_steps_device(counts, seed)
    want = cpython_steps(counts, seed)
    for c, g, w in zip(counts, got, want):
        assert np.array_equal(g, w), c
