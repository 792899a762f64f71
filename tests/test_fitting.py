"""Fitting drivers (cellbasedmodels.jl_b200/fitting.py) on CPU: the grid of
CBMFitting.gridSearch (src/fitting/gridSearch.jl:19-65; first parameter
fastest, argmin of `_score_`, optional CSV), and the batched driver with the
host stand-in of the batch, on one rank and sharded over two gloo ranks."""
import csv
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import conftest
import _gloo_worker as W

cbm = conftest.cbm


def test_grid_points_first_parameter_fastest():
    pts = cbm.fitting.grid_points({"a": [1, 2, 3], "b": [10, 20]})
    assert [(p["a"], p["b"]) for p in pts] == [(1, 10), (2, 10), (3, 10), (1, 20), (2, 20), (3, 20)]
    assert cbm.fitting.grid_points({}) == []


def test_grid_search_best_all_and_csv(tmp_path):
    search = {"a": [1.0, 2.0, 3.0], "b": [10.0, 20.0]}
    f = lambda p, w: (p["a"] - 2.0) ** 2 + w * p["b"]  # noqa: E731
    best = cbm.fitting.grid_search(f, search, args=(0.01,))
    assert (best["a"], best["b"]) == (2.0, 10.0) and best["_score_"] == pytest.approx(0.1)
    rows = cbm.fitting.grid_search(f, search, return_all=True, args=(0.01,),
                                   save_file_name=str(tmp_path / "grid"))
    assert len(rows) == 6 and rows[3]["_score_"] == pytest.approx(1.2)
    with open(tmp_path / "grid.csv") as fh:
        lines = list(csv.reader(fh))
    assert lines[0] == ["a", "b", "_score_"] and len(lines) == 7
    # ties: the first point of least score, as argmin
    tie = cbm.fitting.grid_search(lambda p: 0.0, search)
    assert (tie["a"], tie["b"]) == (1.0, 10.0)


def test_community_descs_checks():
    with pytest.raises(ValueError):
        cbm.fitting.community_descs({"dt": [0.1]}, 10, (0,) * 3, (1,) * 3, W.FIT_DEFAULTS)
    with pytest.raises(ValueError):  # sigma neither searched nor given
        cbm.fitting.community_descs({"k_rep": [1.0]}, 10, (0,) * 3, (1,) * 3, W.FIT_DEFAULTS)
    d = cbm.fitting.community_descs(W.FIT_SEARCH, 10, (0,) * 3, (2,) * 3, W.FIT_DEFAULTS, 7)
    assert [x.community for x in d] == list(range(7, 13))
    assert [(x.k_rep, x.sigma) for x in d][:4] == [(5.0, 0.0), (10.0, 0.0), (20.0, 0.0), (5.0, 0.1)]
    assert d[0].box_hi[2] == 2.0 and d[0].r_att == 3.0


def _expected_rows():
    pts = cbm.fitting.grid_points(W.FIT_SEARCH)
    out = []
    for i, p in enumerate(pts):
        x0 = W.fit_state(i, p)["x"].astype(np.float32).astype(np.float64)
        out.append(float(np.mean(x0 + 5 * (i + 1) * 1e-3)) + p["sigma"])
    return out


def test_batched_grid_search_host_batch():
    rows = cbm.fitting.batched_grid_search(None, W.FIT_SEARCH, W.fit_state, W.fit_loss, 5,
                                           (0.0,) * 3, (1.0,) * 3, W.FIT_DEFAULTS,
                                           return_all=True, factory=W.FakeBatch)
    np.testing.assert_allclose([r["_score_"] for r in rows], _expected_rows(), rtol=1e-12)
    best = cbm.fitting.batched_grid_search(None, W.FIT_SEARCH, W.fit_state, W.fit_loss, 5,
                                           (0.0,) * 3, (1.0,) * 3, W.FIT_DEFAULTS,
                                           factory=W.FakeBatch)
    assert best["_score_"] == min(r["_score_"] for r in rows)


def test_batched_grid_search_world2(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=W.run_fit, args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    r0, r1 = (np.load(tmp_path / f"fit{r}.npy") for r in range(world))
    np.testing.assert_array_equal(r0, r1)  # every rank holds every score
    np.testing.assert_allclose(r0[:, 2], _expected_rows(), rtol=1e-12)
