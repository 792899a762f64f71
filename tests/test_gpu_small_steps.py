"""Small fate-free CellLinked communities: all the steps of a cbm_step call run
in one cooperative launch (csrc/cbm_small.cuh).  The state after the launch
(positions, grid, counters, parity) is the one the step graphs leave: every
result is bit-identical to the CPU checker and to the kernel-by-kernel path,
and the stage calls continue from it."""
import numpy as np
import pytest

import conftest
from _oracle import OracleContext
from scenarios import aggregation_2d
from test_gpu_parity import assert_same_grid, assert_same_state

cbm = conftest.cbm
pytestmark = pytest.mark.gpu


def community(abi, dims, prec, walls, integ, N=1500, L=60.0, seed=41):
    rng = np.random.default_rng(seed)
    kw = dict(dims=dims, precision=abi.F32 if prec == "f32" else abi.F64, n_max=N,
              box_lo=(0.0,) * dims, box_hi=(L,) * dims, dt=0.01, seed=seed,
              neighbors=abi.NEIGH_CELL_LINKED, cell_edge=3.0,
              integrator=abi.INT_EM if integ == "em" else abi.INT_EULER, sigma=0.3,
              k_rep=10.0, r_rep=2.0, k_att=1.0, r_att=3.0,
              walls={"none": abi.WALLS_NONE, "reflect": abi.WALLS_REFLECT,
                     "push": abi.WALLS_PUSH}[walls], wall_force=1.0, wall_range=0.5)
    # a few agents start beyond the box, so reflection and the ghost cells act
    st = {k: rng.uniform(-1.0, L + 1.0, N) for k in "xyz"[:dims]}
    return kw, st


@pytest.mark.parametrize("integ", ["euler", "em"])
@pytest.mark.parametrize("walls", ["none", "reflect", "push"])
@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("dims", [1, 2, 3])
def test_one_launch_matches_checker_and_graph_free_path(gpu_lib, abi, dims, prec, walls, integ):
    N = {1: 400, 2: 1500, 3: 2500}[dims]
    L = {1: 300.0, 2: 60.0, 3: 22.0}[dims]
    kw, st = community(abi, dims, prec, walls, integ, N=N, L=L)
    cfg = abi.make_config(**kw)
    a = cbm.Context(cfg)  # one launch per call
    b = cbm.Context(cfg)  # kernel by kernel
    o = OracleContext(abi, cfg, threads=4)
    for ctx in (a, b, o):
        ctx.upload(st)
    keys = list("xyz"[:dims])
    for n in (1, 7, 24):  # odd and even step counts: the parity carries over
        a.step(n)
        b.step(n, abi.SYNC | abi.NO_GRAPH)
        o.step(n)
        sa, sb, so = a.download(), b.download(), o.download()
        assert_same_state(sa, so, keys)
        assert_same_state(sa, sb, keys)
        assert sa["step"] == so["step"] and sa["t"] == so["t"]
    assert_same_grid(a, o)


def test_stages_continue_after_one_launch(gpu_lib, abi):
    """After a one-launch call the stage entry points (agentStepRule! ...
    computeNeighbors!) take the state as the step graphs leave it."""
    kw, st = aggregation_2d(abi, N=1200, L=50.0)
    cfg = abi.make_config(**kw)
    g, o = cbm.Context(cfg), OracleContext(abi, cfg, threads=4)
    g.upload(st)
    o.upload(st)
    g.step(11)
    o.step(11)
    for _ in range(3):
        for name in ("agent_rule", "agent_de", "medium_rule", "medium_de", "update", "neighbors"):
            g.stage(name)
            o.stage(name)
    g.step(5)
    o.step(5)
    assert_same_state(g.download(), o.download(), ["x", "y"])
    assert_same_grid(g, o)
    assert g.counters()["step"] == 19


def test_aggregation_as_configured_in_one_launch(gpu_lib, abi):
    """The 2D aggregation (4096 agents, Float64): 1000 steps in a single call."""
    kw, st = aggregation_2d(abi)
    cfg = abi.make_config(**kw)
    g, o = cbm.Context(cfg), OracleContext(abi, cfg, threads=8)
    g.upload(st)
    o.upload(st)
    g.step(1000)
    o.step(1000)
    assert_same_state(g.download(), o.download(), ["x", "y"])
    assert_same_grid(g, o)
