"""Heun, RungeKutta4 and EulerHeun agent integrators (src/integrators.jl:
516-668,744-814) on the device against the checker, bit for bit: every stage
evaluates f over the cell grid of the last rebuild at the stage's positions
(own cell from the position, no face pruning), with the reference's
combination expressions; EulerHeun with noise (sigma > 0)."""
import numpy as np
import pytest

import conftest
from scenarios import aggregation_2d, chemotaxis_2d, colony_3d, packed_colony_3d
from test_gpu_parity import assert_same_grid, assert_same_lists, assert_same_state, both

cbm = conftest.cbm
pytestmark = pytest.mark.gpu

INTEGRATORS = {"heun": "INT_HEUN", "rk4": "INT_RK4", "euler_heun": "INT_EULER_HEUN"}
SIGMA = {"heun": 0.0, "rk4": 0.0, "euler_heun": 0.05}
ALL = ["heun", "rk4", "euler_heun"]


@pytest.mark.parametrize("integ", ALL)
def test_multistage_aggregation_2d(gpu_lib, abi, integ):
    """2D soft spheres, reflecting walls, Float64, CellLinked."""
    kw, st = aggregation_2d(abi, N=1500, L=60.0)
    kw = dict(kw, integrator=getattr(abi, INTEGRATORS[integ]), sigma=SIGMA[integ])
    g, o = both(abi, kw, st)
    for _ in range(3):
        g.step(20)
        o.step(20)
        assert_same_state(g.download(), o.download(), ["x", "y"])
    assert_same_grid(g, o)


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("integ", ALL)
def test_multistage_colony_3d(gpu_lib, abi, integ, prec):
    """3D colony with growth, division and death, CellLinked."""
    kw, st = colony_3d(abi, N=3000, L=60.0, n_max=12000, p_death=2e-3, sigma=SIGMA[integ],
                       precision=abi.F32 if prec == "f32" else abi.F64,
                       neighbors=abi.NEIGH_CELL_LINKED)
    kw = dict(kw, integrator=getattr(abi, INTEGRATORS[integ]))
    g, o = both(abi, kw, st)
    for _ in range(3):
        g.step(20)
        o.step(20)
        a, b = g.download(), o.download()
        assert_same_state(a, b, ["x", "y", "z", "v", "g", "id", "parent"])
    assert a["id_max"] > 3000


@pytest.mark.parametrize("integ", ALL)
def test_multistage_verlet_displacement(gpu_lib, abi, integ):
    """VerletDisplacement lists: every stage reads the list of the last
    rebuild; the final combination checks the displacement for the rebuild."""
    kw, st = colony_3d(abi, N=1500, L=60.0, n_max=6000, p_death=0.0, sigma=SIGMA[integ],
                       neighbors=abi.NEIGH_VERLET_DISPLACEMENT)
    kw = dict(kw, integrator=getattr(abi, INTEGRATORS[integ]), fate=abi.FATE_NONE, growth=0)
    g, o = both(abi, kw, st)
    for _ in range(3):
        g.step(20)
        o.step(20)
        assert_same_state(g.download(), o.download(), ["x", "y", "z"])
    assert_same_lists(g, o)


@pytest.mark.parametrize("integ", ALL)
def test_multistage_dense_colony(gpu_lib, abi, integ):
    """4 agents per unit volume: the stages' walks fill their partner lists."""
    kw, st = packed_colony_3d(abi, N=4000, density=4.0, L=60.0, n_max=8000)
    kw = dict(kw, neighbors=abi.NEIGH_CELL_LINKED, sigma=SIGMA[integ],
              integrator=getattr(abi, INTEGRATORS[integ]))
    g, o = both(abi, kw, st)
    for _ in range(2):
        g.step(5)
        o.step(5)
        assert_same_state(g.download(), o.download(), ["x", "y", "z", "v", "id"])


@pytest.mark.parametrize("integ", ["heun", "rk4"])
def test_multistage_chemotaxis_and_full(gpu_lib, abi, integ):
    """The chemotactic drift sampled at stage positions (2D, medium), and the
    Full neighbor algorithm (3D)."""
    kw, st = chemotaxis_2d(abi, N=2000, L=128.0, n_medium=128)
    kw = dict(kw, sigma=0.0, integrator=getattr(abi, INTEGRATORS[integ]))
    g, o = both(abi, kw, st)
    for _ in range(2):
        g.step(15)
        o.step(15)
        assert_same_state(g.download(), o.download(), ["x", "y", "c", "gx", "gy"])
    rng = np.random.default_rng(9)
    n = 300
    p = rng.uniform(0, 12, size=(3, n))
    kw = dict(dims=3, precision=abi.F32, n_max=n, box_lo=(0.0,) * 3, box_hi=(12.0,) * 3,
              dt=0.01, neighbors=abi.NEIGH_FULL, integrator=getattr(abi, INTEGRATORS[integ]),
              k_rep=10.0, r_rep=2.0, k_att=1.0, r_att=3.0)
    g, o = both(abi, kw, dict(x=p[0], y=p[1], z=p[2]))
    g.step(10)
    o.step(10)
    assert_same_state(g.download(), o.download(), ["x", "y", "z"])


def test_multistage_rejects_sde_and_lists(gpu_lib, abi):
    base = dict(dims=2, precision=abi.F32, n_max=10, box_lo=(0.0, 0.0), box_hi=(10.0, 10.0),
                dt=0.01, neighbors=abi.NEIGH_CELL_LINKED, cell_edge=3.0,
                integrator=abi.INT_RK4, k_rep=10.0, r_rep=2.0, k_att=1.0, r_att=3.0)
    for bad in (dict(sigma=0.1), dict(neighbors=abi.NEIGH_CLVD, skin=3.0, n_max_neighbors=16),
                dict(force_mode=abi.FORCE_LAGGED)):
        with pytest.raises(cbm.CbmError):
            cbm.Context(abi.make_config(**dict(base, **bad)))
