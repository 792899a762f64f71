"""Parity of the B200 path with the CPU checker on the measured configurations
at their configured sizes.

- the 3D colony grown on the device from 10^4 agents (the timed workload's
  state): 100 steps from 10^5 agents in Float32 and Float64, and 3 steps from
  10^6 agents in Float32;
- the 2D aggregation as configured: 4096 agents, Float64, 1000 steps;
- the 2D chemotaxis as configured: 2x10^5 agents on a 1024^2 medium, 100 steps;
- the 3D medium line as benched: 2x10^5 agents on a 256^3 medium with
  secretion, uptake and chemotaxis, 20 steps (TMA-fed stencils, gather by
  patches);
- communities of the batched sweep, compared with the checker directly;
- trajectory gradients of the 65536-agent adjoint problem (200 steps,
  checkpoint every 20) against the checker's forward-mode dual numbers.

Everything but the gradients is bit-exact: cell ids, cell order, N, ids,
parent ids, positions, volumes and medium fields.  Gradients: 1e-6 relative,
the loss 1e-10 relative (Float64).
"""
import os

import numpy as np
import pytest

import conftest
from _oracle import OracleContext, oracle_adjoint_dual
from scenarios import (adjoint_problem, aggregation_2d, batched_sweep, chemotaxis_2d,
                       growing_colony_3d, make_descs, medium_colony, plain_config_for)
from test_gpu_parity import assert_same_grid, assert_same_lists, assert_same_state

cbm = conftest.cbm
pytestmark = pytest.mark.gpu

THREADS = os.cpu_count()
COLONY_KEYS = ["x", "y", "z", "v", "g", "id", "parent"]


def grown_colony(abi, n_target, precision, headroom=1.2):
    """The configured colony (10^4 agents uniform in a radius-20 ball centred
    in [0,400]^3, seed 2) grown on the device until N >= n_target.  Returns
    the configuration and the state with its counters."""
    kw, st = growing_colony_3d(abi, n_target, precision=precision, headroom=headroom)
    g = cbm.Context(abi.make_config(**kw))
    g.upload(st)
    steps = 0
    while g.counters()["N"] < n_target:
        g.step(10)
        steps += 10
        assert steps < 5000
    snap = g.download()
    g.close()
    assert snap["step"] == steps
    return kw, snap


def from_snapshot(abi, kw, snap):
    """A device context and the checker, both loaded with the same state
    (loadToPlatform! on each side, so both rebuild their grids and lists)."""
    cfg = abi.make_config(**kw)
    state = {k: snap[k] for k in COLONY_KEYS}
    up = dict(t=snap["t"], step=snap["step"], id_max=snap["id_max"])
    g = cbm.Context(cfg)
    o = OracleContext(abi, cfg, threads=THREADS)
    g.upload(state, **up)
    o.upload(state, **up)
    return g, o


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_grown_colony_1e5_100_steps_bitexact(gpu_lib, abi, prec):
    """The grown colony at 10^5 agents (core density about 2 per unit
    volume): 100 steps with division, death and noise, bit-exact."""
    # 100 more steps grow the colony by about 2^(100/200): room for 1.6x
    kw, snap = grown_colony(abi, 100_000, abi.F32 if prec == "f32" else abi.F64, headroom=1.6)
    assert snap["N"] >= 100_000
    g, o = from_snapshot(abi, kw, snap)
    for _ in range(4):
        g.step(25)
        assert o.step(25) == 0  # no Verlet row of the checker overflowed
        a, b = g.download(), o.download()
        assert_same_state(a, b, COLONY_KEYS)
        assert (a["id_max"], a["step"]) == (b["id_max"], b["step"])
    assert a["N"] > snap["N"]
    assert_same_lists(g, o)
    g.close()
    o.close()


def test_grown_colony_1e6_three_steps_bitexact(gpu_lib, abi):
    """The benched state itself: the colony grown to 10^6 agents (about 4
    agents per unit volume in the core, some 350 partners per agent), three
    steps, bit-exact."""
    kw, snap = grown_colony(abi, 1_000_000, abi.F32)
    assert snap["N"] >= 1_000_000
    g, o = from_snapshot(abi, kw, snap)
    g.step(3)
    assert o.step(3) == 0  # no Verlet row of the checker overflowed
    a, b = g.download(), o.download()
    assert_same_state(a, b, COLONY_KEYS)
    assert a["id_max"] == b["id_max"]
    assert a["N"] != snap["N"]
    assert len(np.unique(a["id"])) == a["N"]
    g.close()
    o.close()


def test_aggregation_2d_as_configured(gpu_lib, abi):
    """4096 agents in [0,100]^2, Float64, Euler dt 0.01, reflecting walls,
    CellLinked edge 3: all 1000 steps, bit-exact, with the grid."""
    kw, st = aggregation_2d(abi)
    cfg = abi.make_config(**kw)
    g = cbm.Context(cfg)
    o = OracleContext(abi, cfg, threads=THREADS)
    g.upload(st)
    o.upload(st)
    for _ in range(4):
        g.step(250)
        o.step(250)
        assert_same_state(g.download(), o.download(), ["x", "y"])
    assert g.counters()["step"] == 1000
    assert_same_grid(g, o)


def test_chemotaxis_2d_as_configured(gpu_lib, abi):
    """2x10^5 agents on the 1024^2 Float32 medium (bilinear secretion, FTCS,
    chemotactic drift, EM noise): 100 steps, bit-exact, medium included."""
    kw, st = chemotaxis_2d(abi)
    cfg = abi.make_config(**kw)
    g = cbm.Context(cfg)
    o = OracleContext(abi, cfg, threads=THREADS)
    g.upload(st)
    o.upload(st)
    for _ in range(2):
        g.step(50)
        o.step(50)
        assert_same_state(g.download(), o.download(), ["x", "y", "c", "gx", "gy"])
    assert_same_grid(g, o)


def test_medium_3d_as_benched(gpu_lib, abi):
    """The 3D medium line: 2x10^5 agents on a 256^3 Float32 field (unit
    spacing, secretion, first-order uptake, chemotaxis, EM noise), the field
    drawn from U(0, 1) with seed 9: 20 steps, bit-exact, field and gradient
    included."""
    n = 256
    kw, st = medium_colony(abi, 3, N=200_000, L=float(n), n_medium=n)
    st["c"] = np.random.default_rng(9).uniform(0.0, 1.0, n ** 3).astype(np.float32)
    cfg = abi.make_config(**kw)
    g = cbm.Context(cfg)
    o = OracleContext(abi, cfg, threads=THREADS)
    g.upload(st)
    o.upload(st)
    for _ in range(2):
        g.step(10)
        o.step(10)
        assert_same_state(g.download(), o.download(), ["x", "y", "z", "c", "gx", "gy", "gz"])
    assert_same_grid(g, o)


def test_batched_communities_match_the_checker(gpu_lib, abi):
    """The first six communities of the configured sweep (N_i from U[500,
    20000], log-uniform k, a, sigma): one persistent launch of 500 EM steps
    under the autotuned tuning, each community compared with the checker
    run on its own parameters."""
    base, descs, states = batched_sweep(abi, n_comm=6)
    b = cbm.Batch(abi.make_config(**base), make_descs(abi, descs))
    for c, st in enumerate(states):
        b.upload(c, st["x"], st["y"], st["z"])
    tuning = b.autotune(trial_steps=5).as_dict()
    for c, st in enumerate(states):
        b.upload(c, st["x"], st["y"], st["z"])
    b.step(500)
    for c in range(len(descs)):
        got = b.download(c)
        o = OracleContext(abi, abi.make_config(**plain_config_for(abi, base, descs[c], tuning)),
                          threads=THREADS)
        o.upload(states[c])
        o.step(500)
        ref = o.download()
        o.close()
        assert got["step"] == 500
        for k in "xyz":
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"community {c} {k}")


def test_adjoint_65536_gradients_match_dual_numbers(gpu_lib, abi):
    """The configured adjoint problem (65536 agents in [0,80]^3, 200 Euler
    steps, Float64, checkpoint every 20): dL/dtheta and dL/dx0 at a handful
    of coordinates against forward-mode dual numbers of the checker."""
    steps = 200
    kw, x0, star = adjoint_problem(abi, N=65536, steps=steps)
    k, a, rho = star
    tgt = cbm.Adjoint(abi.make_config(**dict(kw, k_rep=k, k_att=a, r_rep=rho, r_att=1.5 * rho,
                                             cell_edge=max(kw["cell_edge"], 1.5 * rho)))
                      ).forward(x0, steps)
    res = cbm.Adjoint(abi.make_config(**kw)).run(x0, tgt, steps, checkpoint_every=20)
    seeds = [(7, 0), (20000, 1), (40001, 2), (65535, 0)]
    loss, grad, dx = oracle_adjoint_dual(abi, abi.make_config(**kw), x0, tgt, steps, seeds=seeds)
    assert abs(res["loss"] - loss) <= 1e-10 * abs(loss)
    np.testing.assert_allclose(res["dtheta"], grad, rtol=1e-6)
    scale = max(np.max(np.abs(d)) for d in res["dx0"])
    for s, (i, ax) in enumerate(seeds):
        assert abs(res["dx0"][ax][i] - dx[s]) <= 1e-6 * scale, (i, ax, res["dx0"][ax][i], dx[s])
