"""Fitting drivers over the batched path.

CBMFitting.gridSearch (src/fitting/gridSearch.jl:19-65) evaluates a scoring
function at every point of a parameter grid, one whole simulation per point,
and returns the best point (argmin of `_score_`) or every point.
`grid_search` keeps that interface for any Python scoring function.

`batched_grid_search` is the B200 path for grids over the parameters a
community of the batched form carries (k_rep, r_rep, k_att, r_att, sigma):
every grid point becomes one community of a `Batch`, all of them advance in
one persistent launch, and the score of a point is `loss(point, final
state)`.  With `world > 1` the points are partitioned across ranks by agent
count (`sweep.ShardedBatch`), each rank scores its own share, and the scores
are gathered on every rank; no collective runs on the data path.

Grid order: the first parameter of `search_list` varies fastest, as the
reference's reshape builds its DataFrame.  Julia's Dict has no defined key
order; a Python dict keeps insertion order, which fixes it here.
"""
import csv
import math

import numpy as np

from . import _abi
from .sweep import ShardedBatch, max_over_ranks  # noqa: F401  (re-exported helper)

COMMUNITY_PARAMS = ("k_rep", "r_rep", "k_att", "r_att", "sigma")


def grid_points(search_list):
    """All points of the grid, as dicts, first parameter fastest."""
    names = list(search_list)
    sizes = [len(search_list[k]) for k in names]
    points = []
    for flat in range(math.prod(sizes) if sizes else 0):
        row, r = {}, flat
        for k, n in zip(names, sizes):
            row[k] = search_list[k][r % n]
            r //= n
        points.append(row)
    return points


def _finish(rows, names, return_all, save_file_name, extra=()):
    cols = list(names) + ["_score_"] + list(extra)
    if save_file_name is not None:
        with open(f"{save_file_name}.csv", "w", newline="") as fh:
            w = csv.writer(fh)
            w.writerow(cols)
            for r in rows:
                w.writerow([r[k] for k in cols])
    if return_all:
        return rows
    best = 0
    for i, r in enumerate(rows):  # argmin: the first of equal minima
        if r["_score_"] < rows[best]["_score_"]:
            best = i
    return rows[best]


def grid_search(eval_function, search_list, return_all=False, save_file_name=None, args=()):
    """gridSearch(evalFunction, searchList; returnAll, saveFileName, args):
    eval_function(point, *args) -> score for every grid point (point is a dict
    of the parameter values).  Returns the point of least score (a dict with
    `_score_`), or every point when return_all."""
    rows = grid_points(search_list)
    for r in rows:
        r["_score_"] = float(eval_function(dict(r), *args))
    return _finish(rows, list(search_list), return_all, save_file_name)


def community_descs(search_list, n, box_lo, box_hi, defaults, first_community=0):
    """One cbm_community_desc per grid point: `defaults` (all of
    COMMUNITY_PARAMS) overridden by the point's values; community index
    first_community + point index (it keys the noise of the point)."""
    unknown = [k for k in search_list if k not in COMMUNITY_PARAMS]
    if unknown:
        raise ValueError(f"not a per-community parameter of the batched form: {unknown}")
    missing = [k for k in COMMUNITY_PARAMS if k not in defaults and k not in search_list]
    if missing:
        raise ValueError(f"no value for {missing}")
    descs = []
    for i, point in enumerate(grid_points(search_list)):
        d = _abi.CbmCommunityDesc()
        d.n = int(n)
        for a in range(3):
            d.box_lo[a] = float(box_lo[a])
            d.box_hi[a] = float(box_hi[a])
        for k in COMMUNITY_PARAMS:
            setattr(d, k, float(point.get(k, defaults.get(k))))
        d.community = first_community + i
        descs.append(d)
    return descs


def batched_grid_search(base_cfg, search_list, initial_state, loss, steps, box_lo, box_hi,
                        defaults, return_all=False, save_file_name=None, first_community=0,
                        rank=0, world=1, dist=None, factory=None, tuning=None):
    """Every grid point simulated as one community of the batched form.

    base_cfg: the batched form's base cbm_config (3D, Float32, CLVD, EM);
    initial_state: {"x", "y", "z"} arrays shared by all points, or a callable
    (index, point) -> such a dict; loss(point, state) -> score, with state the
    downloaded {"x", "y", "z", "step", "N"} of the point after `steps` steps;
    defaults: values of COMMUNITY_PARAMS that the grid does not vary.
    rank/world/dist shard the points over ranks (dist: torch.distributed or
    None); factory builds the local batch (the GPU `Batch` by default)."""
    names = list(search_list)
    rows = grid_points(search_list)
    scores = batched_scores(base_cfg, rows, initial_state, loss, steps, box_lo, box_hi, defaults,
                            first_community=first_community, rank=rank, world=world, dist=dist,
                            factory=factory, tuning=tuning)
    for r, sc in zip(rows, scores):
        r["_score_"] = sc
    return _finish(rows, names, return_all, save_file_name)


def batched_scores(base_cfg, points, initial_state, loss, steps, box_lo, box_hi, defaults,
                   first_community=0, rank=0, world=1, dist=None, factory=None, tuning=None):
    """Scores of `points` (dicts of COMMUNITY_PARAMS values), every point one
    community of the batched form, all advanced together for `steps` steps;
    community index first_community + position keys each point's noise.
    The arguments are those of batched_grid_search."""
    rows = [dict(p) for p in points]

    def state_of(i):
        st = initial_state(i, dict(rows[i])) if callable(initial_state) else initial_state
        return {k: np.ascontiguousarray(st[k], dtype=np.float32) for k in "xyz"}

    descs = []
    for i, r in enumerate(rows):
        n = len(state_of(i)["x"])
        descs.append(community_descs({k: [v] for k, v in r.items()}, n, box_lo, box_hi,
                                     defaults, first_community + i)[0])
    sb = ShardedBatch(base_cfg, descs, rank=rank, world=world, factory=factory)
    if sb.batch is not None and tuning is not None:
        sb.batch.set_tuning(**tuning)
    for c in sb.mine:
        st = state_of(c)
        sb.upload(c, st["x"], st["y"], st["z"])
    sb.step(steps)
    mine = {c: float(loss(dict(rows[c]), st)) for c, st in sb.download_local().items()}
    if dist is not None and world > 1:
        box = [None] * world
        dist.all_gather_object(box, mine)
        scores = {}
        for part in box:
            scores.update(part)
    else:
        scores = mine
    return [scores[i] for i in range(len(rows))]


class BatchedEvaluator:
    """The `evaluate_population` of the population drivers on the batched
    form: each call simulates a whole generation as one batch (see
    batched_scores).  Successive calls take fresh community indices, so every
    evaluation draws its own noise, as every evalFunction call of the
    reference runs a fresh simulation."""

    def __init__(self, base_cfg, initial_state, loss, steps, box_lo, box_hi, defaults,
                 first_community=0, rank=0, world=1, dist=None, factory=None, tuning=None):
        self.kw = dict(base_cfg=base_cfg, initial_state=initial_state, loss=loss, steps=steps,
                       box_lo=box_lo, box_hi=box_hi, defaults=defaults, rank=rank, world=world,
                       dist=dist, factory=factory, tuning=tuning)
        self.next_community = first_community
        self.calls = 0

    def __call__(self, points):
        scores = batched_scores(points=points, first_community=self.next_community, **self.kw)
        self.next_community += len(points)
        self.calls += 1
        return scores


# ---------------------------------------------------------------------------
# Population drivers: swarmAlgorithm, geneticAlgorithm, beeColonyAlgorithm
# (src/fitting/{swarm,genetic,beeColony}Algorithm.jl).  Each keeps the
# reference's loops, update rules and bookkeeping columns (_score_,
# _generation_, _velocity_ / _cycles_), and the order of its random draws
# within a generation.  Draws come from `rng` (a numpy Generator, seeded by
# the caller) instead of Julia's global RNG.  A generation is evaluated by
# `evaluate_population(points) -> scores` when given (BatchedEvaluator: one
# batch per generation), else by eval_function(point, *args) point by point.
# ---------------------------------------------------------------------------


def _continuous(search_list, name):
    for k, v in search_list.items():
        if not (isinstance(v, tuple) and len(v) == 2):
            raise ValueError(f"{name} only works with continuous parameters (lo, hi): {k}")


def _draw(rng, spec):
    """rand(Uniform(lo, hi)) for a (lo, hi) tuple, rand(list) for a list."""
    if isinstance(spec, tuple):
        return float(rng.uniform(spec[0], spec[1]))
    return spec[int(rng.integers(len(spec)))]


def _initial_rows(search_list, population, initialisation, rng, draw):
    rows = []
    for i in range(population):
        r = {}
        for k in search_list:
            if initialisation is None:
                r[k] = draw(k)
            elif isinstance(initialisation, dict):
                r[k] = initialisation[k][i]
            else:
                r[k] = initialisation[i][k]
        rows.append(r)
    return rows


def _evaluate(rows, names, eval_function, evaluate_population, args):
    points = [{k: r[k] for k in names} for r in rows]
    if evaluate_population is not None:
        scores = evaluate_population(points)
    else:
        scores = [eval_function(dict(p), *args) for p in points]
    for r, sc in zip(rows, scores):
        r["_score_"] = float(sc)


def _argmin(rows):
    best = 0
    for i, r in enumerate(rows):
        if r["_score_"] < rows[best]["_score_"]:
            best = i
    return best


def _selection_weights(rows):
    """p = 1 - (score - min)/(max - min), normalised; uniform when all equal
    (geneticAlgorithm.jl / beeColonyAlgorithm.jl)."""
    sc = np.array([r["_score_"] for r in rows], dtype=np.float64)
    lo, hi = sc.min(), sc.max()
    if hi != lo:
        p = 1.0 - (sc - lo) / (hi - lo)
        return p / p.sum()
    return np.full(len(rows), 1.0 / len(rows))


def swarm_algorithm(eval_function, search_list, population=100, weight_inertia=0.1,
                    weight_global_best=0.1, weight_population_best=0.1, stop_max_generations=10,
                    initialisation=None, return_all=False, save_file_name=None, args=(), rng=None,
                    evaluate_population=None):
    """swarmAlgorithm (src/fitting/swarmAlgorithm.jl:38-155).  Velocities start
    uniform in ±(hi - lo); v = wI v + wG rand() (gbest - x) + wP rand() (pbest - x),
    x += v clamped to the range, with pbest the best of the current generation
    and gbest the best so far.  Returns the best row, or every row."""
    _continuous(search_list, "swarmAlgorithm")
    rng = np.random.default_rng() if rng is None else rng
    names = list(search_list)
    vel = {k: f"{k}_velocity_" for k in names}
    rows = []
    for i in range(population):
        r = {}
        for k in names:
            lo, hi = search_list[k]
            r[k] = (float(rng.uniform(lo, hi)) if initialisation is None else
                    (initialisation[k][i] if isinstance(initialisation, dict)
                     else initialisation[i][k]))
            r[vel[k]] = float(rng.uniform(-(hi - lo), hi - lo))
        r["_generation_"] = 1
        rows.append(r)
    _evaluate(rows, names, eval_function, evaluate_population, args)
    total = [dict(r) for r in rows]
    pbest = dict(rows[_argmin(rows)])
    gbest = dict(pbest)
    for gen in range(2, stop_max_generations + 1):
        new = []
        for i in range(population):
            r = {}
            for k in names:
                lo, hi = search_list[k]
                v = (weight_inertia * rows[i][vel[k]]
                     + weight_global_best * rng.random() * (gbest[k] - rows[i][k])
                     + weight_population_best * rng.random() * (pbest[k] - rows[i][k]))
                x = rows[i][k] + v
                r[vel[k]] = v
                r[k] = lo if x < lo else (hi if x > hi else x)
            r["_generation_"] = gen
            new.append(r)
        rows = new
        _evaluate(rows, names, eval_function, evaluate_population, args)
        total += [dict(r) for r in rows]
        pbest = dict(rows[_argmin(rows)])
        if pbest["_score_"] < gbest["_score_"]:
            gbest = dict(pbest)
    return _finish(total, names + [vel[k] for k in names], return_all, save_file_name,
                   extra=("_generation_",))


def genetic_algorithm(eval_function, search_list, population=100, parent_selection_alg="weighted",
                      parent_selection_p=0.1, mutation_rate=0.1, stop_max_generations=10,
                      initialisation=None, return_all=False, save_file_name=None, args=(),
                      rng=None, evaluate_population=None):
    """geneticAlgorithm (src/fitting/geneticAlgorithm.jl:36-156).  Pairs of
    parents are drawn with weights 1 - (score - min)/(max - min); each
    parameter is swapped between the two children when rand() <= P and
    mutated (redrawn from its range or list) with probability mutationRate.
    `parent_selection_alg` is accepted and, as in the reference, unused.
    The population must be even (children are made in pairs)."""
    if population % 2:
        raise ValueError("geneticAlgorithm makes children in pairs: population must be even")
    rng = np.random.default_rng() if rng is None else rng
    names = list(search_list)
    rows = _initial_rows(search_list, population, initialisation, rng,
                         lambda k: _draw(rng, search_list[k]))
    for r in rows:
        r["_generation_"] = 1
    _evaluate(rows, names, eval_function, evaluate_population, args)
    total = [dict(r) for r in rows]
    for gen in range(2, stop_max_generations + 1):
        p = _selection_weights(rows)
        new = [dict() for _ in range(population)]
        for i in range(0, population, 2):
            pa, pb = (int(c) for c in rng.choice(population, size=2, p=p))
            for k in names:
                if parent_selection_p < rng.random():
                    new[i][k], new[i + 1][k] = rows[pa][k], rows[pb][k]
                else:
                    new[i][k], new[i + 1][k] = rows[pb][k], rows[pa][k]
                if mutation_rate > rng.random():
                    new[i][k] = _draw(rng, search_list[k])
                if mutation_rate > rng.random():
                    new[i + 1][k] = _draw(rng, search_list[k])
        for r in new:
            r["_generation_"] = gen
        rows = new
        _evaluate(rows, names, eval_function, evaluate_population, args)
        total += [dict(r) for r in rows]
    return _finish(total, names, return_all, save_file_name, extra=("_generation_",))


def bee_colony_algorithm(eval_function, search_list, population=100, limit_cycles=10,
                         stop_max_generations=100, return_all=False, initialisation=None,
                         save_file_name=None, args=(), rng=None, evaluate_population=None):
    """beeColonyAlgorithm (src/fitting/beeColonyAlgorithm.jl:31-154).  Bee i
    moves to x + U(-1, 1) (x_c - x) toward a candidate c drawn with the
    selection weights, clamped to the range, and its cycle count restarts;
    a bee whose count has reached limitCycles is redrawn uniformly and keeps
    its count.  A move that scores worse is undone (old row, count + 1, the
    new generation number), as in the reference."""
    _continuous(search_list, "beeColonyAlgorithm")
    rng = np.random.default_rng() if rng is None else rng
    names = list(search_list)
    rows = _initial_rows(search_list, population, initialisation, rng,
                         lambda k: float(rng.uniform(*search_list[k])))
    for r in rows:
        r["_generation_"] = 1
        r["_cycles_"] = 0
    _evaluate(rows, names, eval_function, evaluate_population, args)
    total = [dict(r) for r in rows]
    for gen in range(2, stop_max_generations + 1):
        p = _selection_weights(rows)
        new = []
        for i in range(population):
            r = {"_generation_": gen, "_cycles_": rows[i]["_cycles_"]}
            cand = int(rng.choice(population, p=p))
            for k in names:
                lo, hi = search_list[k]
                if rows[i]["_cycles_"] < limit_cycles:
                    x = rows[i][k] + float(rng.uniform(-1.0, 1.0)) * (rows[cand][k] - rows[i][k])
                    r[k] = lo if x < lo else (hi if x > hi else x)
                else:
                    r[k] = float(rng.uniform(lo, hi))
            if rows[i]["_cycles_"] < limit_cycles:
                r["_cycles_"] = 0
            new.append(r)
        old = rows
        rows = new
        _evaluate(rows, names, eval_function, evaluate_population, args)
        for i in range(population):
            if rows[i]["_score_"] > old[i]["_score_"]:
                kept = dict(old[i])
                kept["_cycles_"] += 1
                kept["_generation_"] = gen
                rows[i] = kept
        total += [dict(r) for r in rows]
    return _finish(total, names, return_all, save_file_name, extra=("_generation_", "_cycles_"))
