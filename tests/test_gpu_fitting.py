"""The batched grid search on the device: every point's score equals the same
loss of a plain-path run with that point's parameters (the batched form
reproduces the plain trajectory bit for bit)."""
import numpy as np
import pytest

import conftest
from scenarios import batched_sweep, plain_config_for

cbm = conftest.cbm
pytestmark = pytest.mark.gpu

TUNING = dict(threads=256, ctas_per_sm=2, skin=0.3, rebuild_threshold=0.0, tile_agents=0)


def test_batched_grid_search_matches_plain_runs(gpu_lib, abi):
    base, descs, states = batched_sweep(abi, n_comm=1, n_lo=400, n_hi=400, seed=21)
    st = states[0]
    L = descs[0]["box_hi"][0]
    x0 = np.asarray(st["x"], np.float32)
    search = {"k_rep": [5.0, 15.0, 30.0], "sigma": [0.02, 0.08]}
    defaults = dict(r_rep=2.0, k_att=1.0, r_att=3.0)

    def loss(point, s):
        return float(np.mean((s["x"] - x0) ** 2))

    rows = cbm.fitting.batched_grid_search(abi.make_config(**base), search, st, loss, 40,
                                           (0.0,) * 3, (L,) * 3, defaults, return_all=True,
                                           tuning=TUNING)
    assert len(rows) == 6
    for i, r in enumerate(rows):
        desc = dict(n=len(x0), box_lo=(0.0,) * 3, box_hi=(L,) * 3, k_rep=r["k_rep"],
                    sigma=r["sigma"], community=i, **defaults)
        g = cbm.Context(abi.make_config(**plain_config_for(abi, base, desc, TUNING)))
        g.upload(st)
        g.step(40)
        assert r["_score_"] == loss(r, g.download()), f"point {i}"
        g.close()
    best = cbm.fitting.batched_grid_search(abi.make_config(**base), search, st, loss, 40,
                                           (0.0,) * 3, (L,) * 3, defaults, tuning=TUNING)
    i = int(np.argmin([r["_score_"] for r in rows]))
    assert (best["k_rep"], best["sigma"], best["_score_"]) == \
        (rows[i]["k_rep"], rows[i]["sigma"], rows[i]["_score_"])


def test_swarm_on_batched_evaluator_matches_plain_runs(gpu_lib, abi):
    """Two generations of swarmAlgorithm, each one batch: every score equals
    the loss of a plain-path run of that point with the community index the
    evaluator gave it (generation g, individual i -> g * population + i)."""
    base, descs, states = batched_sweep(abi, n_comm=1, n_lo=300, n_hi=300, seed=22)
    st = states[0]
    L = descs[0]["box_hi"][0]
    x0 = np.asarray(st["x"], np.float32)
    defaults = dict(r_rep=2.0, k_att=1.0, r_att=3.0)

    def loss(point, s):
        return float(np.mean((s["x"] - x0) ** 2))

    ev = cbm.fitting.BatchedEvaluator(abi.make_config(**base), st, loss, 30, (0.0,) * 3,
                                      (L,) * 3, defaults, tuning=TUNING)
    rows = cbm.fitting.swarm_algorithm(None, {"k_rep": (5.0, 30.0), "sigma": (0.0, 0.08)},
                                       population=4, stop_max_generations=2,
                                       rng=np.random.default_rng(5), evaluate_population=ev,
                                       return_all=True)
    assert len(rows) == 8 and ev.calls == 2
    for c, r in enumerate(rows):
        desc = dict(n=len(x0), box_lo=(0.0,) * 3, box_hi=(L,) * 3, k_rep=r["k_rep"],
                    sigma=r["sigma"], community=c, **defaults)
        g = cbm.Context(abi.make_config(**plain_config_for(abi, base, desc, TUNING)))
        g.upload(st)
        g.step(30)
        assert r["_score_"] == loss(r, g.download()), f"row {c}"
        g.close()
