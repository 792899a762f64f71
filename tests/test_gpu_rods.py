"""The device rods2D and rods2dGrowth models (cbm_rods_*, src/models/rods.jl)
against the checker, bit for bit: Float32 and Float64, CellLinked and
all-pairs neighbors, dense colonies where most rods touch several others, rods
outside the simBox (clamped into the border cells), several steps per call,
graph and one-by-one launches, the empty and single-rod cases, and growing
colonies whose rods divide (rows filled from the tail as update! does)."""
import math

import numpy as np
import pytest

from _oracle import OracleRods

pytestmark = pytest.mark.gpu

PARAMS = dict(dt=1e-4, kn=2.0e6, gamma_n=100.0, gamma_t=20.0, mu_cc=0.1, beta=0.8, beta_w=0.8)


def _colony(abi, n, seed, half, spread_out=0.0):
    rng = np.random.default_rng(seed)
    st = {k: np.zeros(n) for k in abi.ROD_FIELDS}
    st["x"] = rng.uniform(-half - spread_out, half + spread_out, n)
    st["y"] = rng.uniform(-half - spread_out, half + spread_out, n)
    st["vx"] = rng.normal(0, 0.1, n)
    st["vy"] = rng.normal(0, 0.1, n)
    st["theta"] = rng.uniform(-math.pi, math.pi, n)
    st["omega"] = rng.normal(0, 0.1, n)
    st["d"] = np.full(n, 1.0)
    st["l"] = rng.uniform(1.0, 3.0, n)
    st["m"] = rng.uniform(0.8, 1.2, n)
    return st


def _compare(abi, cbm, cfg, st, steps, flags=None):
    g = cbm._abi.Rods2D(cfg)
    o = OracleRods(abi, cfg)
    g.upload(st)
    o.upload(st)
    contacts = 0
    for s in steps:
        g.step(s, abi.SYNC if flags is None else flags)
        o.step(s)
        a = g.download()
        b = o.download()
        for k in abi.ROD_FIELDS:
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"{k} after {s} steps")
        contacts = max(contacts, int(np.count_nonzero(b["pressure"])))
    g.close()
    o.close()
    return contacts


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("neighbors", ["cell_linked", "full"])
def test_rods_bitexact(gpu_lib, abi, prec, neighbors):
    from conftest import cbm
    n = 1500 if neighbors == "cell_linked" else 400
    half = math.sqrt(n) * 0.9  # about 0.3 rods per unit area: most rods touch
    st = _colony(abi, n, 11, half)
    cfg = abi.make_rods_config(
        n, (-half - 2, -half - 2), (half + 2, half + 2), cell_edge=4.0,
        neighbors=abi.NEIGH_CELL_LINKED if neighbors == "cell_linked" else abi.NEIGH_FULL,
        precision=abi.F32 if prec == "f32" else abi.F64, **PARAMS)
    contacts = _compare(abi, cbm, cfg, st, [1, 1, 5, 13])
    assert contacts > n // 3


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_rods_outside_box(gpu_lib, abi, prec, graph):
    """Rods beyond the simBox fall in the border cells (cellPos clamps); the
    steps replayed from the two-step graphs and launched one by one agree."""
    from conftest import cbm
    n = 600
    st = _colony(abi, n, 12, 10.0, spread_out=6.0)
    cfg = abi.make_rods_config(n, (-10.0, -10.0), (10.0, 10.0), cell_edge=3.5,
                               precision=abi.F32 if prec == "f32" else abi.F64, **PARAMS)
    _compare(abi, cbm, cfg, st, [3, 4], flags=abi.SYNC | (0 if graph else abi.NO_GRAPH))


def test_rods_large_grid_f32(gpu_lib, abi):
    """A 40k-rod colony for 6 steps: many blocks, a multi-tile cell scan."""
    from conftest import cbm
    n = 40000
    half = math.sqrt(n) * 0.9
    st = _colony(abi, n, 13, half)
    cfg = abi.make_rods_config(n, (-half - 2, -half - 2), (half + 2, half + 2), cell_edge=4.0,
                               precision=abi.F32, **PARAMS)
    _compare(abi, cbm, cfg, st, [2, 4])


@pytest.mark.parametrize("n", [0, 1])
def test_rods_empty_and_single(gpu_lib, abi, n):
    from conftest import cbm
    st = _colony(abi, n, 14, 3.0)
    cfg = abi.make_rods_config(8, (-5.0, -5.0), (5.0, 5.0), cell_edge=3.0, **PARAMS)
    _compare(abi, cbm, cfg, st, [1, 2])


def test_rods_step_before_upload(gpu_lib, abi):
    from conftest import cbm
    cfg = abi.make_rods_config(8, (-5.0, -5.0), (5.0, 5.0), cell_edge=3.0, **PARAMS)
    g = cbm._abi.Rods2D(cfg)
    with pytest.raises(cbm._abi.CbmError):
        g.step(1)
    with pytest.raises(cbm._abi.CbmError):
        g.upload({k: np.zeros(9) for k in abi.ROD_FIELDS})  # n > n_max
    g.close()


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_rods_bacteries_constants(gpu_lib, abi, prec):
    """The constants and step of examples/Bacteries.ipynb (dt 0.1, soft contacts,
    cellEdge 4) on a packed 3000-rod disc, 40 steps."""
    from conftest import cbm
    import bench
    st = bench.rod_disc(abi, 3000, seed=5)
    cfg = abi.make_rods_config(3000, (-300.0, -300.0), (300.0, 300.0), cell_edge=4.0,
                               precision=abi.F32 if prec == "f32" else abi.F64,
                               **bench.ROD_PARAMS)
    contacts = _compare(abi, cbm, cfg, st, [1, 9, 30])
    assert contacts > 1000


GROW = dict(growth=0.5, alpha=50.0, sigma_l_target=0.2, l_max=3.0, seed=91)


def _growth_colony(abi, n, seed, half):
    st = _colony(abi, n, seed, half)
    rng = np.random.default_rng(seed + 1)
    st["l"] = rng.uniform(2.0, 3.0, n)
    st["l_target"] = st["l"] + rng.uniform(-0.05, 0.3, n)
    return st


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("neighbors", ["cell_linked", "full"])
def test_rods_growth_bitexact(gpu_lib, abi, prec, neighbors, graph):
    """rods2dGrowth: rods grow at dt(l) = growth/(1+α pressure), divide past
    lTarget into two daughters with drawn torque and targets, and update!
    fills the parents' rows from the tail; the device matches the checker
    row by row while the colony grows."""
    from conftest import cbm
    n0 = 400 if neighbors == "cell_linked" else 150
    half = math.sqrt(n0) * 0.9
    st = _growth_colony(abi, n0, 31, half)
    cfg = abi.make_rods_config(
        4 * n0, (-half - 30, -half - 30), (half + 30, half + 30), cell_edge=4.0,
        neighbors=abi.NEIGH_CELL_LINKED if neighbors == "cell_linked" else abi.NEIGH_FULL,
        precision=abi.F32 if prec == "f32" else abi.F64, **bench_rod_params(), **GROW)
    g = cbm._abi.Rods2D(cfg)
    o = OracleRods(abi, cfg)
    g.upload(st)
    o.upload(st)
    sizes = []
    for s in [1, 2, 5, 8]:
        g.step(s, abi.SYNC | (0 if graph else abi.NO_GRAPH))
        o.step(s)
        a, b = g.download(), o.download()
        assert len(a["x"]) == len(b["x"]) == o.count()[0]
        for k in abi.ROD_FIELDS:
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"{k} after {s} steps")
        sizes.append(len(a["x"]))
    g.close()
    o.close()
    assert sizes[0] > n0 and sizes[-1] > sizes[0]


@pytest.mark.parametrize("n_max", [100, 101, 130, 160, 199, 300])
def test_rods_growth_overflow(gpu_lib, abi, n_max):
    """Births beyond n_max are dropped in order and every parent is still
    removed (functionRule.jl:58-70), old rows moving into the holes when
    fewer daughters than parents were born; the status reports the
    overflow.  Rows match the checker bit for bit, from no room to room for
    every birth."""
    from conftest import cbm
    st = _growth_colony(abi, 100, 32, 9.0)
    st["l_target"] = st["l"] + np.where(np.arange(100) % 4 == 1, 1.0, -1.0)  # 75 divide
    cfg = abi.make_rods_config(n_max, (-20.0, -20.0), (20.0, 20.0), cell_edge=4.0,
                               **bench_rod_params(), **GROW)
    g = cbm._abi.Rods2D(cfg)
    o = OracleRods(abi, cfg)
    g.upload(st)
    o.upload(st)
    if n_max < 250:
        with pytest.raises(cbm._abi.CbmError) as e:
            g.step(1)
        assert e.value.code == abi.CBM_ERR_AGENT_OVERFLOW
    else:
        g.step(1)
    o.step(1)
    a, b = g.download(), o.download()
    assert len(a["x"]) == len(b["x"]) == 100 + min(150, n_max - 100) - 75
    for k in abi.ROD_FIELDS:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    g.close()
    o.close()


@pytest.mark.parametrize("first,stride,n_max", [(60, 1, 110), (60, 1, 100), (60, 1, 125),
                                                (51, 2, 112), (90, 1, 104)])
def test_rods_growth_overflow_top_rows(gpu_lib, abi, first, stride, n_max):
    """Dividers in the top rows with little room: rows first, first+stride,
    ... up to 99 divide, and only n_max - 100 daughters fit.  Fewer daughters
    than parents are born, so the fill moves surviving old rows, and some of
    them have holes above them and stay where they are (update.jl:15-119)."""
    from conftest import cbm
    st = _growth_colony(abi, 100, 33, 9.0)
    divide = np.zeros(100, bool)
    divide[first::stride] = True
    st["l_target"] = st["l"] + np.where(divide, -1.0, 1.0)
    cfg = abi.make_rods_config(n_max, (-20.0, -20.0), (20.0, 20.0), cell_edge=4.0,
                               **bench_rod_params(), **GROW)
    g = cbm._abi.Rods2D(cfg)
    o = OracleRods(abi, cfg)
    g.upload(st)
    o.upload(st)
    n_div = int(divide.sum())
    if 2 * n_div > n_max - 100:
        with pytest.raises(cbm._abi.CbmError) as e:
            g.step(1)
        assert e.value.code == abi.CBM_ERR_AGENT_OVERFLOW
    else:
        g.step(1)
    o.step(1)
    a, b = g.download(), o.download()
    assert len(a["x"]) == len(b["x"]) == 100 + min(2 * n_div, n_max - 100) - n_div
    for k in abi.ROD_FIELDS:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    g.close()
    o.close()


def bench_rod_params():
    import bench
    return dict(bench.ROD_PARAMS)
