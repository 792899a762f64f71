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


def _finish(rows, names, return_all, save_file_name):
    if save_file_name is not None:
        with open(f"{save_file_name}.csv", "w", newline="") as fh:
            w = csv.writer(fh)
            w.writerow(list(names) + ["_score_"])
            for r in rows:
                w.writerow([r[k] for k in names] + [r["_score_"]])
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

    def state_of(i):
        st = initial_state(i, dict(rows[i])) if callable(initial_state) else initial_state
        return {k: np.ascontiguousarray(st[k], dtype=np.float32) for k in "xyz"}

    sizes = [len(state_of(i)["x"]) for i in range(len(rows))]
    descs = []
    for i, n in enumerate(sizes):
        d = community_descs({k: [rows[i][k]] for k in names}, n, box_lo, box_hi, defaults,
                            first_community + i)[0]
        descs.append(d)
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
    for i, r in enumerate(rows):
        r["_score_"] = scores[i]
    return _finish(rows, names, return_all, save_file_name)
