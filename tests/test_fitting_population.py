"""The population drivers of cellbasedmodels.jl_b200/fitting.py on CPU:
swarmAlgorithm, geneticAlgorithm and beeColonyAlgorithm
(src/fitting/{swarm,genetic,beeColony}Algorithm.jl).

Julia's global RNG cannot be reproduced, so the checks are on the update
rules themselves.  A scripted generator feeds known draws, and the tests
check the velocity rule, the crossover and mutation rule, and the bee cycle
bookkeeping.  They also check seeded reproducibility, convergence on a
quadratic, the CSV columns, and the batched evaluator over the host stand-in
of the batch."""
import csv

import numpy as np
import pytest

import conftest
import _gloo_worker as W

cbm = conftest.cbm
F = cbm.fitting


class Scripted:
    """A generator whose uniform/random/choice/integers return scripted values
    (uniform(lo, hi) maps a scripted u in [0, 1) to lo + u (hi - lo))."""

    def __init__(self, us, choices=()):
        self.us = list(us)
        self.choices = list(choices)

    def _u(self):
        return self.us.pop(0)

    def uniform(self, lo, hi):
        return lo + self._u() * (hi - lo)

    def random(self):
        return self._u()

    def integers(self, n):
        return int(self._u() * n)

    def choice(self, n, size=None, p=None):
        if size is None:
            return self.choices.pop(0)
        return np.array([self.choices.pop(0) for _ in range(size)])


def quad(point):
    return (point["a"] - 3.0) ** 2 + (point["b"] + 1.0) ** 2


SEARCH = {"a": (0.0, 10.0), "b": (-5.0, 5.0)}


def test_swarm_velocity_rule_and_clamp():
    # population 2, one parameter on (0, 10): x0 = 2, 8; v0 = -10 + 20 u
    us = [0.2, 0.5, 0.8, 0.75,  # x, v of particle 0 then of particle 1
          0.5, 0.25,            # generation 2, particle 0: rand() for gbest, for pbest
          0.5, 0.5]             # particle 1
    rows = F.swarm_algorithm(lambda p: (p["a"] - 7.0) ** 2, {"a": (0.0, 10.0)}, population=2,
                             weight_inertia=0.5, weight_global_best=1.0,
                             weight_population_best=2.0, stop_max_generations=2,
                             rng=Scripted(us), return_all=True)
    g1, g2 = rows[:2], rows[2:]
    assert [r["a"] for r in g1] == [2.0, 8.0]
    assert [r["a_velocity_"] for r in g1] == [0.0, 5.0]
    # best of generation 1 is x = 8 (score 1): gbest = pbest = 8
    v0 = 0.5 * 0.0 + 1.0 * 0.5 * (8.0 - 2.0) + 2.0 * 0.25 * (8.0 - 2.0)
    v1 = 0.5 * 5.0 + 1.0 * 0.5 * 0.0 + 2.0 * 0.5 * 0.0
    assert g2[0]["a_velocity_"] == v0 and g2[0]["a"] == 2.0 + v0
    assert g2[1]["a_velocity_"] == v1 and g2[1]["a"] == 10.0  # 8 + 2.5 clamped to hi
    assert [r["_generation_"] for r in rows] == [1, 1, 2, 2]


def test_genetic_crossover_and_mutation_rule():
    # population 2, parameters a (continuous) and b (a list)
    search = {"a": (0.0, 10.0), "b": [1, 2, 3, 4]}
    us = [0.1, 0.0, 0.9, 0.99,  # a0 = 1, b0 = 1, a1 = 9, b1 = 4
          0.5, 0.05, 0.3, 0.95,  # gen 2, a: crossover test, mutation tests (child 0: draw 0.3)
          0.02, 0.5, 0.5]        # gen 2, b: crossover test, mutation tests
    # b: 0.1 < 0.02 is false, so child 0 takes the second parent's b and
    # child 1 the first's; neither mutates
    rows = F.genetic_algorithm(lambda p: p["a"], search, population=2, parent_selection_p=0.1,
                               mutation_rate=0.1, stop_max_generations=2,
                               rng=Scripted(us, choices=[1, 0]), return_all=True)
    g1, g2 = rows[:2], rows[2:]
    assert [(r["a"], r["b"]) for r in g1] == [(1.0, 1), (9.0, 4)]
    # parents (1, 0); a: 0.1 < 0.5 -> child0 = parent 1's (9), child1 = parent 0's (1);
    # child 0 mutated to 0.3 * 10 = 3; child 1 not (0.95)
    assert g2[0]["a"] == 3.0 and g2[1]["a"] == 1.0
    assert g2[0]["b"] == 1 and g2[1]["b"] == 4
    with pytest.raises(ValueError):
        F.genetic_algorithm(quad, SEARCH, population=3)


def test_bee_cycles_bookkeeping():
    """Every move scores worse, so every bee is reverted: its count grows by
    one per generation, it becomes a scout at limitCycles, and a scout keeps
    its count (the reference never resets it)."""
    calls = {"n": 0}

    def worse(points):
        calls["n"] += 1
        return [float(calls["n"])] * len(points)

    rows = F.bee_colony_algorithm(None, SEARCH, population=4, limit_cycles=2,
                                  stop_max_generations=6, rng=np.random.default_rng(3),
                                  evaluate_population=worse, return_all=True)
    cycles = [[r["_cycles_"] for r in rows[g * 4:(g + 1) * 4]] for g in range(6)]
    assert cycles == [[0] * 4, [1] * 4, [2] * 4, [3] * 4, [4] * 4, [5] * 4]
    first = rows[:4]
    for g in range(1, 6):  # reverted rows keep the first generation's positions and scores
        for i in range(4):
            r = rows[g * 4 + i]
            assert (r["a"], r["b"], r["_score_"]) == (first[i]["a"], first[i]["b"], 1.0)
            assert r["_generation_"] == g + 1
    # with improving scores every move is kept and the counts restart
    def better(points):
        calls["n"] += 1
        return [-float(calls["n"])] * len(points)

    rows = F.bee_colony_algorithm(None, SEARCH, population=4, limit_cycles=2,
                                  stop_max_generations=4, rng=np.random.default_rng(4),
                                  evaluate_population=better, return_all=True)
    assert all(r["_cycles_"] == 0 for r in rows)


@pytest.mark.parametrize("algo", ["swarm", "genetic", "bee"])
def test_seeded_runs_repeat_and_converge(algo, tmp_path):
    fn = {"swarm": F.swarm_algorithm, "genetic": F.genetic_algorithm,
          "bee": F.bee_colony_algorithm}[algo]
    kw = dict(population=40, stop_max_generations=25)
    a = fn(quad, SEARCH, rng=np.random.default_rng(11), return_all=True, **kw)
    b = fn(quad, SEARCH, rng=np.random.default_rng(11), return_all=True, **kw)
    assert a == b
    best = fn(quad, SEARCH, rng=np.random.default_rng(11), save_file_name=str(tmp_path / algo),
              **kw)
    first_gen = min(r["_score_"] for r in a[:40])
    assert best["_score_"] == min(r["_score_"] for r in a)
    assert best["_score_"] <= first_gen and best["_score_"] < 0.5
    for r in a:
        assert 0.0 <= r["a"] <= 10.0 and -5.0 <= r["b"] <= 5.0
    with open(tmp_path / f"{algo}.csv") as fh:
        lines = list(csv.reader(fh))
    assert len(lines) == 1 + 40 * 25
    extra = {"swarm": ["a_velocity_", "b_velocity_", "_score_", "_generation_"],
             "genetic": ["_score_", "_generation_"],
             "bee": ["_score_", "_generation_", "_cycles_"]}[algo]
    assert lines[0] == ["a", "b"] + extra


def test_continuous_only():
    with pytest.raises(ValueError):
        F.swarm_algorithm(quad, {"a": [1.0, 2.0]}, population=2)
    with pytest.raises(ValueError):
        F.bee_colony_algorithm(quad, {"a": [1.0, 2.0]}, population=2)


def test_initialisation_rows():
    init = {"a": [1.0, 2.0], "b": [0.0, 0.5]}
    rows = F.bee_colony_algorithm(quad, SEARCH, population=2, stop_max_generations=1,
                                  initialisation=init, return_all=True)
    assert [(r["a"], r["b"]) for r in rows] == [(1.0, 0.0), (2.0, 0.5)]


def test_batched_evaluator_host_batch():
    """A generation is one batch; successive generations take fresh community
    indices (the host batch moves community c by (c + 1) 1e-3 per step)."""
    search = {"k_rep": (5.0, 20.0), "sigma": (0.0, 0.1)}
    state = W.fit_state(0, None)
    ev = F.BatchedEvaluator(None, state, W.fit_loss, 5, (0.0,) * 3, (1.0,) * 3, W.FIT_DEFAULTS,
                            factory=W.FakeBatch)
    rows = F.swarm_algorithm(None, search, population=6, stop_max_generations=3,
                             rng=np.random.default_rng(2), evaluate_population=ev,
                             return_all=True)
    assert ev.calls == 3 and ev.next_community == 18
    x0 = np.asarray(state["x"], np.float32).astype(np.float64)
    for c, r in enumerate(rows):
        expect = float(np.mean(x0 + 5 * (c + 1) * 1e-3)) + r["sigma"]
        assert r["_score_"] == pytest.approx(expect, rel=1e-12)


def test_swarm_generations_sharded_over_two_gloo_ranks(tmp_path):
    """Each generation's batch is partitioned over two ranks and the scores
    gathered; both ranks then hold the single-rank run's rows exactly."""
    import socket

    import torch.multiprocessing as mp
    world = 2
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=W.run_swarm, args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    r0, r1 = (np.load(tmp_path / f"swarm{r}.npy") for r in range(world))
    np.testing.assert_array_equal(r0, r1)
    np.testing.assert_array_equal(r0, W.swarm_rows())
