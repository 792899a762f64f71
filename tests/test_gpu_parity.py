"""Parity of the B200 path (through the C ABI) with the CPU checker.

Bit-exact: cell ids, cell membership and order, Verlet lists, N, NAdd/NRemove,
ids, parent ids, and — because both sides evaluate the same IEEE operations in
the same order without FMA contraction and share the counter-based noise —
positions, volumes and medium fields too.  The one exception is bilinear
secretion under a Verlet algorithm, whose atomic sums may be added in any
order: there the tolerance is 1e-5 relative (Float32), stated in the test.
"""
import numpy as np
import pytest

import conftest
from _oracle import OracleContext
from scenarios import aggregation_2d, chemotaxis_2d, colony_3d
from test_oracle_golden import LATTICE_EXPECTED, aggregation_cfg, lattice_algs, lattice_positions

cbm = conftest.cbm
pytestmark = pytest.mark.gpu


def both(abi, kw, state, **up):
    cfg = abi.make_config(**kw)
    g = cbm.Context(cfg)
    o = OracleContext(abi, cfg, threads=4)
    g.upload(state, **up)
    o.upload(state, **up)
    return g, o


def assert_same_state(a, b, keys, exact=True, rtol=0.0):
    assert a["N"] == b["N"]
    for k in keys:
        if exact:
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
        else:
            np.testing.assert_allclose(a[k], b[k], rtol=rtol, atol=rtol, err_msg=k)


def assert_same_grid(g, o):
    a, b = g.grid(), o.grid()
    assert a["shape"] == b["shape"]
    for k in ("agent_cell", "cell_start", "cell_count", "cell_agents"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def assert_same_lists(g, o):
    ca, la = g.neighbors()
    cb, lb = o.neighbors()
    np.testing.assert_array_equal(ca, cb)
    for i in range(len(ca)):
        np.testing.assert_array_equal(la[i, : ca[i]], lb[i, : cb[i]])


@pytest.mark.parametrize("d", [1, 2, 3])
@pytest.mark.parametrize("alg", ["Full", "VerletDisplacement", "CellLinked", "CLVD"])
def test_lattice_neighbor_counts_gpu(gpu_lib, abi, d, alg):
    cfg = abi.make_config(dims=d, n_max=3 ** d, box_lo=(0.5,) * d, box_hi=(1.5,) * d, dt=1.0,
                          **lattice_algs(abi)[alg])
    g = cbm.Context(cfg)
    g.upload(lattice_positions(d))
    g.stage("neighbors")
    assert list(g.count_neighbors(1.1)) == LATTICE_EXPECTED[d]


def test_aggregation_traces_gpu(gpu_lib, abi):
    g = cbm.Context(aggregation_cfg(abi, 2, (-5, -2), (5, 2)))
    g.upload(dict(x=np.array([-0.1, 0.1]), y=np.zeros(2)))
    xs, fx = [], []
    for _ in range(5):
        g.step(1)
        s = g.download()
        xs.append(s["x"][0])
        fx.append(s["fx"][0])
    np.testing.assert_allclose(xs, [-0.1, -0.16, -0.22, -0.268, -0.304], atol=1e-12)
    np.testing.assert_allclose(fx, [-0.6, -0.6, -0.48, -0.36, -0.264], atol=1e-12)
    g = cbm.Context(aggregation_cfg(abi, 1, (-2, -2), (2, 2)))
    g.upload(dict(x=np.array([0.0]), y=np.array([-2.5])))
    ys = []
    for _ in range(9):
        g.step(1)
        ys.append(g.download()["y"][0])
    np.testing.assert_allclose(ys, [-2.5, -2.4, -2.3, -2.2, -2.1, -2.0, -1.9, -1.8, -1.7], atol=1e-12)


def test_add_remove_bookkeeping_gpu(gpu_lib, abi):
    N = 100
    kw = dict(dims=1, n_max=N + N // 2, box_lo=(0,), box_hi=(1,), dt=1.0, fate=abi.FATE_ID_PARITY)
    g, o = both(abi, kw, dict(x=np.linspace(0, 1, N)))
    for ctx in (g, o):
        ctx.stage("agent_rule")
    cg, co = g.counters(), o.counters()
    assert (cg["N"], cg["n_add"], cg["n_remove"], cg["id_max"], cg["flag"]) == (N, 50, 50, 150, 1)
    assert cg["n_add"] == co["n_add"] and cg["n_remove"] == co["n_remove"]
    for ctx in (g, o):
        ctx.stage("agent_de")
        ctx.stage("update")
    cg = g.counters()
    assert (cg["N"], cg["n_add"], cg["n_remove"], cg["id_max"]) == (N, 0, 0, 150)
    a, b = g.download(), o.download()
    assert_same_state(a, b, ["x", "id", "parent"])
    assert set(range(2, N + 1, 2)) <= set(a["parent"].tolist())


def test_removal_only_and_empty_community_gpu(gpu_lib, abi):
    kw = dict(dims=3, n_max=12, dt=0.1, fate=abi.FATE_VOLUME, p_death=1.0,
              neighbors=abi.NEIGH_CELL_LINKED, cell_edge=0.5)
    g, o = both(abi, kw, dict(x=np.zeros(2), y=np.zeros(2), z=np.zeros(2)))
    g.step(10)
    o.step(10)
    assert g.counters()["N"] == 0 == o.counters()["N"]
    # an empty community steps without error
    g2 = cbm.Context(abi.make_config(**{**kw, "p_death": 0.0}))
    g2.upload(dict(x=np.zeros(0), y=np.zeros(0), z=np.zeros(0)))
    g2.step(3)
    assert g2.counters()["N"] == 0


@pytest.mark.parametrize("graph", [True, False])
def test_aggregation_2d_bitexact(gpu_lib, abi, graph):
    kw, st = aggregation_2d(abi, N=1500, L=60.0)
    g, o = both(abi, kw, st)
    assert_same_grid(g, o)
    flags = abi.SYNC | (0 if graph else abi.NO_GRAPH)
    for _ in range(4):
        g.step(25, flags)
        o.step(25)
        assert_same_state(g.download(), o.download(), ["x", "y"])
    assert_same_grid(g, o)


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("alg", ["CLVD", "VerletDisplacement", "CellLinked"])
def test_colony_3d_bitexact(gpu_lib, abi, prec, alg):
    neigh = dict(CLVD=abi.NEIGH_CLVD, VerletDisplacement=abi.NEIGH_VERLET_DISPLACEMENT,
                 CellLinked=abi.NEIGH_CELL_LINKED)[alg]
    N = 1500 if alg == "VerletDisplacement" else 3000
    kw, st = colony_3d(abi, N=N, L=60.0, n_max=4 * N, p_death=2e-3,
                       precision=abi.F32 if prec == "f32" else abi.F64, neighbors=neigh)
    g, o = both(abi, kw, st)
    births = 0
    for _ in range(4):
        g.step(25)
        o.step(25)
        a, b = g.download(), o.download()
        assert_same_state(a, b, ["x", "y", "z", "v", "g", "id", "parent"])
        assert a["id_max"] == b["id_max"]
        births = a["id_max"] - N
    assert births > 100  # divisions happened
    assert a["N"] != N
    if alg == "CellLinked":
        assert_same_grid(g, o)
    else:
        assert_same_lists(g, o)


def test_packed_colony_1m_bitexact(gpu_lib, abi):
    """The bench workload at its full size (10^6 agents, Float32, CLVD,
    divisions every step): three steps, bit-exact against the checker."""
    from scenarios import packed_colony_3d
    kw, st = packed_colony_3d(abi, N=1_000_000)
    cfg = abi.make_config(**kw)
    g = cbm.Context(cfg)
    o = OracleContext(abi, cfg, threads=16)
    g.upload(st)
    o.upload(st)
    g.step(3)
    o.step(3)
    a, b = g.download(), o.download()
    assert a["N"] > 1_000_000
    assert_same_state(a, b, ["x", "y", "z", "v", "g", "id", "parent"])
    assert a["id_max"] == b["id_max"]
    # size-independent invariants of the state
    assert len(np.unique(a["id"])) == a["N"]
    born = a["id"] > 1_000_000
    assert born.sum() > 0
    assert np.all(a["parent"][born] >= 1) and np.all(a["parent"][born] < a["id"][born])
    assert a["id"].max() <= a["id_max"]


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("alg", ["CellLinked", "CLVD"])
def test_dense_colony_bitexact(gpu_lib, abi, prec, alg):
    """A compressed colony (4 agents per unit volume, the core density a colony
    grown from 10^4 reaches): the force walk stores some 450 partners per
    agent in its partner lists; still bit-exact, through divisions, with the
    grid."""
    from scenarios import packed_colony_3d
    neigh = abi.NEIGH_CELL_LINKED if alg == "CellLinked" else abi.NEIGH_CLVD
    kw, st = packed_colony_3d(abi, N=6000, density=4.0, L=60.0, n_max=12000,
                              precision=abi.F32 if prec == "f32" else abi.F64)
    kw = dict(kw, neighbors=neigh, n_max_neighbors=1024)
    g, o = both(abi, kw, st)
    for _ in range(3):
        g.step(8)
        o.step(8)
        assert_same_state(g.download(), o.download(), ["x", "y", "z", "v", "id", "parent"])
    assert g.counters()["N"] > 6000
    if alg == "CellLinked":
        assert_same_grid(g, o)


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_overcrowded_colony_bitexact(gpu_lib, abi, prec):
    """24 agents per unit volume: agents have over 1024 partners, more than a
    partner list holds, so lists fill in the middle of the walk and their
    terms are added there; the sums keep the reference's order."""
    from scenarios import packed_colony_3d
    kw, st = packed_colony_3d(abi, N=3000, density=24.0, L=60.0, n_max=6000,
                              precision=abi.F32 if prec == "f32" else abi.F64)
    kw = dict(kw, neighbors=abi.NEIGH_CELL_LINKED)
    g, o = both(abi, kw, st)
    for _ in range(2):
        g.step(4)
        o.step(4)
        assert_same_state(g.download(), o.download(), ["x", "y", "z", "v", "id", "parent"])
    assert_same_grid(g, o)


@pytest.mark.parametrize("alg", ["CellLinked", "CLVD"])
def test_agents_beyond_the_box_gpu(gpu_lib, abi, alg):
    """Agents outside simBox fall in the ghost cells (cellPos clamps,
    neighbors.jl:636-638); the grid, the lists and the trajectories follow the
    reference, including the pairs its ghost layer does not see."""
    rng = np.random.default_rng(21)
    n = 1200
    L = 24.0
    p = rng.uniform(-4.0, L + 4.0, size=(3, n))  # a shell of agents beyond every face
    neigh = abi.NEIGH_CELL_LINKED if alg == "CellLinked" else abi.NEIGH_CLVD
    kw = dict(dims=3, precision=abi.F64, n_max=n, box_lo=(0.0,) * 3, box_hi=(L,) * 3, dt=0.01,
              seed=21, neighbors=neigh, cell_edge=3.3, skin=3.3, rebuild_threshold=0.15,
              n_max_neighbors=64, integrator=abi.INT_EM, sigma=0.05, k_rep=10.0, r_rep=2.0,
              k_att=1.0, r_att=3.0)
    g, o = both(abi, kw, dict(x=p[0], y=p[1], z=p[2]))
    for _ in range(3):
        g.step(10)
        o.step(10)
        assert_same_state(g.download(), o.download(), ["x", "y", "z", "id"])
    if alg == "CellLinked":
        assert_same_grid(g, o)
    else:
        assert_same_lists(g, o)


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_external_noise_bitexact(gpu_lib, abi, prec):
    """Noise generated once on the host and fed to both sides (cbm_step_noise):
    a growing colony stays bit-identical while N changes every step."""
    kw, st = colony_3d(abi, N=2000, L=50.0, n_max=8000, p_death=2e-3,
                       precision=abi.F32 if prec == "f32" else abi.F64)
    g, o = both(abi, kw, st)
    rng = np.random.default_rng(77)
    for _ in range(30):
        n = g.counters()["N"]
        assert n == o.counters()["N"]
        xi = rng.standard_normal((n, 3))
        g.step_noise(xi)
        o.step_noise(xi)
    a, b = g.download(), o.download()
    assert a["N"] > 2000
    assert_same_state(a, b, ["x", "y", "z", "v", "id", "parent"])
    # and the given noise is what moved the agents: the drawn stream differs
    g2, _ = both(abi, kw, st)
    g2.step(30)
    assert not np.array_equal(g2.download()["x"][:100], a["x"][:100])


@pytest.mark.parametrize("bilinear", [False, True])
def test_chemotaxis_2d(gpu_lib, abi, bilinear):
    kw, st = chemotaxis_2d(abi, N=3000, L=128.0, n_medium=128, bilinear=bilinear)
    g, o = both(abi, kw, st)
    keys = ["x", "y", "c", "gx", "gy"]
    for _ in range(4):
        g.step(25)
        o.step(25)
        a, b = g.download(), o.download()
        assert_same_state(a, b, keys)
    assert np.max(a["c"]) > 0


def test_bilinear_secretion_atomic_path(gpu_lib, abi):
    """Bilinear secretion with a Verlet algorithm adds through atomics in any
    order; with a stable model (k dt = 0.2) the results agree with the checker
    to Float32 rounding: tolerance 1e-5 relative."""
    kw, st = chemotaxis_2d(abi, N=2000, L=128.0, n_medium=128, bilinear=True)
    kw.update(neighbors=abi.NEIGH_CLVD, skin=2.4, n_max_neighbors=32, cell_edge=2.4, dt=0.02)
    g, o = both(abi, kw, st)
    g.step(50)
    o.step(50)
    a, b = g.download(), o.download()
    for k in ("x", "y"):
        np.testing.assert_allclose(a[k], b[k], rtol=1e-5, atol=1e-4, err_msg=k)
    np.testing.assert_allclose(a["c"], b["c"], rtol=1e-5, atol=1e-6)


def test_exp_decay_and_em_variance_gpu(gpu_lib, abi):
    g = cbm.Context(abi.make_config(dims=3, n_max=3, dt=0.1, drift_linear=0.5))
    g.upload(dict(x=np.ones(3), y=np.zeros(3), z=np.zeros(3)))
    for _ in range(100):
        g.step(1)
        s = g.download()
        assert np.all(np.abs(s["x"] - np.exp(-0.5 * s["t"])) < 0.05)
    N = 10000
    kw = dict(dims=3, n_max=N, dt=0.1, integrator=abi.INT_EM, sigma=1.0, seed=11)
    g, o = both(abi, kw, dict(x=np.zeros(N), y=np.zeros(N), z=np.zeros(N)))
    for _ in range(100):
        g.step(1)
        s = g.download()
        assert abs(s["t"] - np.var(s["x"])) < 0.5
    o.step(100)
    assert_same_state(g.download(), o.download(), ["x", "y", "z"])


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_rng_stream_matches_checker(gpu_lib, abi, prec):
    cfg = abi.make_config(dims=1, n_max=1, seed=5, precision=abi.F64 if prec == "f64" else abi.F32)
    g, o = cbm.Context(cfg), OracleContext(abi, cfg)
    for kind, a, b in ((0, 1.0, 2.0), (1, 1.0, 2.0), (2, 3.0, 0.0)):
        np.testing.assert_array_equal(g.rng_fill(kind, a, b, 100000, step=7),
                                      o.rng_fill(kind, a, b, 100000, step=7))
    nrm = g.rng_fill(0, 1.0, 2.0, 100000).astype(np.float64)
    assert abs(nrm.mean() - 1) < 0.05 and abs(nrm.var() - 4) < 0.05


def test_stage_double_buffer(gpu_lib, abi):
    """x vs x__ before and after update! (test/testCommunity.jl:33-236)."""
    kw, st = aggregation_2d(abi, N=300, L=30.0)
    g, o = both(abi, kw, st)
    x0 = g.download()["x"]
    for ctx in (g, o):
        ctx.stage("agent_rule")
        ctx.stage("agent_de")
    a, b = g.download(), o.download()
    np.testing.assert_array_equal(a["x"], x0)  # committed x unchanged
    an, bn = g.download(abi.VIEW_NEW), o.download(abi.VIEW_NEW)
    np.testing.assert_array_equal(an["x"], bn["x"])
    assert not np.array_equal(an["x"], x0)
    for ctx in (g, o):
        ctx.stage("medium_rule")
        ctx.stage("medium_de")
        ctx.stage("update")
        ctx.stage("neighbors")
    np.testing.assert_array_equal(g.download()["x"], an["x"])
    assert g.counters()["step"] == 1
    assert_same_grid(g, o)


def test_agent_overflow_reported(gpu_lib, abi):
    kw, st = colony_3d(abi, N=500, L=40.0, n_max=520, p_death=0.0, precision=abi.F64)
    st["v"] = np.full(500, 1.99)
    g, o = both(abi, kw, st)
    with pytest.raises(cbm.CbmError) as e:
        g.step(5)
    assert e.value.code == abi.CBM_ERR_AGENT_OVERFLOW
    o.step(5)
    a, b = g.download(), o.download()
    assert a["N"] <= 520
    assert_same_state(a, b, ["x", "y", "z", "v", "id", "parent"])


def test_neighbor_overflow_reported(gpu_lib, abi):
    kw, st = colony_3d(abi, N=400, R=3.0, L=20.0, p_death=0.0, precision=abi.F64,
                       neighbors=abi.NEIGH_VERLET_DISPLACEMENT)
    kw["n_max_neighbors"] = 4
    # VerletDisplacement builds its list at load
    with pytest.raises(cbm.CbmError) as e:
        g = cbm.Context(abi.make_config(**kw))
        g.upload(st)
    assert e.value.code == abi.CBM_ERR_NEIGHBOR_OVERFLOW
    # CLVD builds its list when it is first needed
    kw["neighbors"] = abi.NEIGH_CLVD
    g = cbm.Context(abi.make_config(**kw))
    g.upload(st)
    with pytest.raises(cbm.CbmError) as e:
        g.neighbors()
    assert e.value.code == abi.CBM_ERR_NEIGHBOR_OVERFLOW


def test_host_api_evolve(gpu_lib, abi):
    """evolve! through the Python mirror of the reference's interface."""
    kw, st = colony_3d(abi, N=800, L=40.0, p_death=1e-3, precision=abi.F32)
    model = cbm.ABM(3, force=cbm.SoftSpheres(k=10, a=1, r=1),
                    neighborsAlg=cbm.CBMNeighbors.CLVD(skin=3.3, nMaxNeighbors=64, cellEdge=3.3,
                                                       rebuildThreshold=0.15),
                    agentAlg=cbm.CBMIntegrators.EM(), sigma=0.05,
                    growth=cbm.Growth(vDiv=2.0, sep=0.5), pDeath=1e-3, platform=cbm.B200("f32"),
                    seed=kw["seed"])
    com = cbm.Community(model, N=800, dt=0.005, simBox=[[0, 40]] * 3, **st)
    cbm.evolve(com, steps=60, saveEach=20, preallocateAgents=3200)
    assert len(com.pastTimes) == 3 and not com.loaded
    o = OracleContext(abi, abi.make_config(**{**kw, "n_max": 4000}))
    o.upload(st)
    o.step(60)
    b = o.download()
    assert com.N == b["N"]
    np.testing.assert_array_equal(com.x, b["x"])
    np.testing.assert_array_equal(com.id, b["id"])


@pytest.mark.parametrize("offset", [1.0e5, -3.0e4])
@pytest.mark.parametrize("alg", ["CLVD", "CellLinked"])
def test_colony_3d_f64_far_from_origin(gpu_lib, abi, alg, offset):
    """A dividing Float64 colony whose box lies far from the origin: at
    |x| ~ 1e5 rounding a coordinate to Float32 moves it by up to ~0.004, so
    the Float32 filter of the Float64 walk works with a bound widened well
    past the cutoff, and the exact Float64 test decides every pair.
    Bit-exact with the checker, grid and lists included."""
    neigh = dict(CLVD=abi.NEIGH_CLVD, CellLinked=abi.NEIGH_CELL_LINKED)[alg]
    N = 3000
    kw, st = colony_3d(abi, N=N, L=60.0, n_max=4 * N, p_death=2e-3, precision=abi.F64,
                       neighbors=neigh)
    kw.update(box_lo=(offset,) * 3, box_hi=(offset + 60.0,) * 3)
    for k in "xyz":
        st[k] = st[k] + offset
    g, o = both(abi, kw, st)
    for _ in range(3):
        g.step(20)
        o.step(20)
        a, b = g.download(), o.download()
        assert_same_state(a, b, ["x", "y", "z", "v", "g", "id", "parent"])
        assert a["id_max"] == b["id_max"]
    assert a["id_max"] > N  # divisions happened
    if alg == "CellLinked":
        assert_same_grid(g, o)
    else:
        assert_same_lists(g, o)
