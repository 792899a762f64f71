"""The CPU checker against the reference's own known answers (runs without a GPU).

Golden vectors and known-answer cases, each from the reference's tests or docs:
  - neighbor counts on a 3^d lattice, test/testCommunity.jl:359-415
  - @addAgent/@removeAgent bookkeeping, test/testCommunity.jl:239-316
  - Euler decay dx/dt = -0.5x, test/testCommunity.jl:418-464
  - EM variance dx = dW, test/testCommunity.jl:467-512
  - normal/uniform/exponential moments, test/testCommunity.jl:319-356
  - two-particle repulsion trace and wall trace, docs/src/Aggregation.md:191-195, :275-279
plus the Philox-4x32-10 known-answer vectors of Salmon et al. (SC'11).
"""
import ctypes as C
import math

import numpy as np
import pytest

from _oracle import OracleContext, load_oracle

LATTICE_EXPECTED = {
    1: [1, 2, 1],
    2: [2, 3, 2, 3, 4, 3, 2, 3, 2],
    3: [3, 4, 3, 4, 5, 4, 3, 4, 3, 4, 5, 4, 5, 6, 5, 4, 5, 4, 3, 4, 3, 4, 5, 4, 3, 4, 3],
}


def lattice_positions(d):
    v = np.zeros((3, 27))
    v[0] = np.tile([0, 1, 2], 9)
    v[1] = np.tile(np.repeat([0, 1, 2], 3), 3)
    v[2] = np.repeat([0, 1, 2], 9)
    return {k: v[i, : 3 ** d].copy() for i, k in enumerate("xyz"[:d])}


def lattice_algs(abi):
    return {
        "Full": dict(neighbors=abi.NEIGH_FULL),
        "VerletDisplacement": dict(neighbors=abi.NEIGH_VERLET_DISPLACEMENT, skin=1.1,
                                   n_max_neighbors=10),
        "CellLinked": dict(neighbors=abi.NEIGH_CELL_LINKED, cell_edge=1.0),
        "CLVD": dict(neighbors=abi.NEIGH_CLVD, skin=1.1, n_max_neighbors=10, cell_edge=10.0),
    }


def aggregation_cfg(abi, N, lo, hi):
    """The Aggregation.md model: lagged forces, rRep=.8, fRep=1, rAtr=1, fAtr=1, D=0, EM."""
    return abi.make_config(dims=2, n_max=N, box_lo=lo, box_hi=hi, dt=0.1,
                           neighbors=abi.NEIGH_FULL, integrator=abi.INT_EM, sigma=0.0,
                           force_mode=abi.FORCE_LAGGED, att_form=abi.ATT_TO_ATT, k_rep=1.0,
                           r_rep=0.8, k_att=1.0, r_att=1.0, walls=abi.WALLS_PUSH,
                           wall_force=1.0, wall_range=0.4)


def test_philox_known_answers(abi):
    lib = load_oracle(abi)
    out = (C.c_uint32 * 4)()
    kat = [((0, 0, 0, 0), (0, 0), "6627e8d5 e169c58d bc57ac4c 9b00dbd8"),
           ((0xffffffff,) * 4, (0xffffffff,) * 2, "408f276d 41c83b0e a20bc7c6 6d5451fd"),
           ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
            "d16cfe09 94fdcceb 5001e420 24126ea1")]
    for ctr, key, expect in kat:
        lib.oracle_philox(*ctr, *key, out)
        assert " ".join("%08x" % v for v in out) == expect


def test_own_log_and_cossin_accuracy(abi):
    lib = load_oracle(abi)
    rng = np.random.default_rng(0)
    for x in np.concatenate([rng.uniform(1e-16, 1.0, 2000), [1.0, 0.5, 2.0 ** -52]]):
        assert abs(lib.oracle_log_f64(x) - math.log(x)) <= 4e-16 * max(1.0, abs(math.log(x)))
        assert abs(lib.oracle_log_f32(x) - math.log(np.float32(x))) <= 4e-7 * max(1.0, abs(math.log(x)))
    c, s = C.c_double(), C.c_double()
    cf, sf = C.c_float(), C.c_float()
    for w in np.concatenate([rng.uniform(0, 1, 2000), [0.0, 0.125, 0.25, 0.5, 0.75]]):
        lib.oracle_cossin_f64(w, C.byref(c), C.byref(s))
        assert abs(c.value - math.cos(2 * math.pi * w)) < 1e-15
        assert abs(s.value - math.sin(2 * math.pi * w)) < 1e-15
        lib.oracle_cossin_f32(w, C.byref(cf), C.byref(sf))
        assert abs(cf.value - math.cos(2 * math.pi * w)) < 1e-6
        assert abs(sf.value - math.sin(2 * math.pi * w)) < 1e-6


@pytest.mark.parametrize("d", [1, 2, 3])
@pytest.mark.parametrize("alg", ["Full", "VerletDisplacement", "CellLinked", "CLVD"])
def test_lattice_neighbor_counts(abi, d, alg):
    cfg = abi.make_config(dims=d, n_max=3 ** d, box_lo=(0.5,) * d, box_hi=(1.5,) * d, dt=1.0,
                          **lattice_algs(abi)[alg])
    o = OracleContext(abi, cfg)
    o.upload(lattice_positions(d))
    o.stage("neighbors")
    assert list(o.count_neighbors(1.1)) == LATTICE_EXPECTED[d]


def test_two_particle_trace(abi):
    o = OracleContext(abi, aggregation_cfg(abi, 2, (-5, -2), (5, 2)))
    o.upload(dict(x=np.array([-0.1, 0.1]), y=np.zeros(2)))
    xs, fx = [], []
    for _ in range(5):
        o.step(1)
        s = o.download()
        xs.append(s["x"].copy())
        fx.append(s["fx"].copy())
    np.testing.assert_allclose([x[0] for x in xs], [-0.1, -0.16, -0.22, -0.268, -0.304], atol=1e-12)
    np.testing.assert_allclose([x[1] for x in xs], [0.1, 0.16, 0.22, 0.268, 0.304], atol=1e-12)
    np.testing.assert_allclose([f[0] for f in fx], [-0.6, -0.6, -0.48, -0.36, -0.264], atol=1e-12)


def test_wall_trace(abi):
    o = OracleContext(abi, aggregation_cfg(abi, 1, (-2, -2), (2, 2)))
    o.upload(dict(x=np.array([0.0]), y=np.array([-2.5])))
    ys = []
    for _ in range(9):
        o.step(1)
        s = o.download()
        ys.append(s["y"][0])
        assert s["x"][0] == 0.0 and s["fx"][0] == 0.0 and s["fy"][0] == 1.0
    np.testing.assert_allclose(ys, [-2.5, -2.4, -2.3, -2.2, -2.1, -2.0, -1.9, -1.8, -1.7], atol=1e-12)


def test_add_remove_bookkeeping(abi):
    N = 100
    cfg = abi.make_config(dims=1, n_max=N + N // 2, box_lo=(0,), box_hi=(1,), dt=1.0,
                          fate=abi.FATE_ID_PARITY)
    o = OracleContext(abi, cfg)
    o.upload(dict(x=np.zeros(N)))
    o.stage("agent_rule")
    c = o.counters()
    assert (c["N"], c["n_add"], c["n_remove"], c["id_max"], c["flag"]) == (N, N // 2, N // 2, 150, 1)
    new = o.download(which=abi.VIEW_NEW, capacity=N + N // 2)
    o.stage("agent_de")
    o.stage("update")
    c = o.counters()
    assert (c["N"], c["n_add"], c["n_remove"], c["id_max"], c["flag"]) == (N, 0, 0, 150, 1)
    s = o.download()
    assert set(range(2, N + 1, 2)) <= set(s["parent"].tolist())
    assert sorted(s["id"].tolist()) == list(range(2, N + 1, 2)) + list(range(N + 1, 151))
    del new


def test_removal_only_evolve_empties(abi):
    cfg = abi.make_config(dims=3, n_max=12, dt=0.1, fate=abi.FATE_VOLUME, p_death=1.0)
    o = OracleContext(abi, cfg)
    o.upload(dict(x=np.zeros(2), y=np.zeros(2), z=np.zeros(2)))
    for _ in range(10):
        o.step(1)
    assert o.counters()["N"] == 0


def test_euler_exponential_decay(abi):
    cfg = abi.make_config(dims=3, n_max=3, dt=0.1, drift_linear=0.5)
    o = OracleContext(abi, cfg)
    o.upload(dict(x=np.ones(3), y=np.zeros(3), z=np.zeros(3)))
    for _ in range(100):
        o.step(1)
        s = o.download()
        assert np.all(np.abs(s["x"] - np.exp(-0.5 * s["t"])) < 0.05)


def test_em_variance(abi):
    N = 10000
    cfg = abi.make_config(dims=3, n_max=N, dt=0.1, integrator=abi.INT_EM, sigma=1.0, seed=11)
    o = OracleContext(abi, cfg)
    o.upload(dict(x=np.zeros(N), y=np.zeros(N), z=np.zeros(N)))
    for _ in range(100):
        o.step(1)
        s = o.download()
        assert abs(s["t"] - np.var(s["x"])) < 0.5


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_distribution_moments(abi, prec):
    N = 100000
    cfg = abi.make_config(dims=1, n_max=1, seed=5, precision=abi.F64 if prec == "f64" else abi.F32)
    o = OracleContext(abi, cfg)
    nrm = o.rng_fill(0, 1.0, 2.0, N).astype(np.float64)
    uni = o.rng_fill(1, 1.0, 2.0, N).astype(np.float64)
    exp = o.rng_fill(2, 3.0, 0.0, N).astype(np.float64)
    assert abs(nrm.mean() - 1) < 0.05 and abs(nrm.var() - 4) < 0.05
    assert abs(uni.min() - 1) < 0.05 and abs(uni.max() - 2) < 0.05 and uni.min() >= 1 and uni.max() < 2
    assert abs(exp.mean() - 3) < 0.05


def test_ftcs_heat_kernel(abi):
    """2D FTCS of a Gaussian against the exact heat kernel (the reference's
    PDE test checks a diffusing Gaussian, test/testCommunity.jl:515-566)."""
    n, L, D, dt, steps = 101, 20.0, 1.0, 0.005, 400  # D dt / dx^2 = 0.13 (stable)
    cfg = abi.make_config(dims=2, n_max=1, box_lo=(-L / 2, -L / 2), box_hi=(L / 2, L / 2), dt=dt,
                          medium=1, n_medium=(n, n), diff_D=D)
    dx = L / n
    xs = -L / 2 + dx * (np.arange(n) + 0.5)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    s0 = 1.0
    c0 = np.exp(-(X ** 2 + Y ** 2) / (2 * s0 ** 2)) / (2 * np.pi * s0 ** 2)
    o = OracleContext(abi, cfg)
    o.upload(dict(x=np.zeros(1), y=np.zeros(1), c=c0.T.reshape(-1)))  # x fastest
    o.step(steps)
    c = o.download()["c"].reshape(n, n).T
    s2 = s0 ** 2 + 2 * D * dt * steps
    exact = np.exp(-(X ** 2 + Y ** 2) / (2 * s2)) / (2 * np.pi * s2)
    assert np.max(np.abs(c - exact)) < 2e-3


def test_compaction_matches_serial_tail_fill(abi):
    """Division + death bookkeeping against a pure-Python restatement of
    kernelListSurvived + kernelFillHolesParameters (update.jl:15-84)."""
    N = 60
    rng = np.random.default_rng(3)
    v = np.where(rng.uniform(size=N) < 0.3, 2.5, 1.0)
    cfg = abi.make_config(dims=2, n_max=200, box_lo=(0, 0), box_hi=(10, 10), dt=0.01, growth=1,
                          fate=abi.FATE_VOLUME, v_div=2.0, div_sep=0.5, p_death=0.2, seed=9)
    o = OracleContext(abi, cfg)
    ids = np.arange(1, N + 1)
    o.upload(dict(x=rng.uniform(0, 10, N), y=rng.uniform(0, 10, N), v=v, g=np.ones(N), id=ids))
    o.stage("agent_rule")
    before = o.download(which=abi.VIEW_NEW, capacity=200)
    c = o.counters()
    n_add, n_rem = c["n_add"], c["n_remove"]
    ids_tail = None
    o.stage("agent_de")
    o.stage("update")
    after = o.download()
    # serial reference: holes ascending, survivors from the tail
    dividing = v >= 2.0
    # dead agents: dividers plus those whose death draw fired; recover them from the ids left
    alive_ids = set(after["id"].tolist())
    dead = [i for i in range(N) if (i + 1) not in alive_ids]
    flag = np.ones(N + n_add, bool)
    flag[dead] = False
    assert len(dead) == n_rem and all(dividing[i] for i in dead if v[i] >= 2.0)
    total = N + n_add
    repos, last = [], total - 1
    while len(repos) < n_rem and last >= 0:
        if flag[last]:
            repos.append(last)
        last -= 1
    order = list(range(total))
    for h, s in zip(sorted(dead), repos):
        if h < s:
            order[h] = s
    expect_ids = np.concatenate([np.arange(1, N + 1), 60 + np.arange(1, n_add + 1)])
    np.testing.assert_array_equal(after["id"], expect_ids[order[: total - n_rem]])
    del before, ids_tail


def test_dual_gradient_matches_central_differences(abi):
    """The forward-mode checker of the adjoint against central differences
    of its own loss (no pair near the cutoff in this small, dilute case)."""
    from _oracle import oracle_adjoint_dual
    rng = np.random.default_rng(21)
    n, L, steps = 30, 9.0, 15
    x0 = [rng.uniform(0, L, n) for _ in range(3)]
    tgt = [x + rng.normal(scale=0.05, size=n) for x in x0]
    theta = dict(k_rep=10.0, k_att=1.0, r_rep=2.0)

    def cfg(**over):
        t = dict(theta, **over)
        return abi.make_config(dims=3, n_max=n, dt=0.01, box_hi=(L,) * 3, k_rep=t["k_rep"],
                               k_att=t["k_att"], r_rep=t["r_rep"], r_att=3.0,
                               neighbors=abi.NEIGH_CELL_LINKED, cell_edge=3.3)

    loss, g, dx = oracle_adjoint_dual(abi, cfg(), x0, tgt, steps, seeds=[(3, 0), (7, 2)])
    for q, name in enumerate(("k_rep", "k_att", "r_rep")):
        h = 1e-6 * theta[name]
        lp = oracle_adjoint_dual(abi, cfg(**{name: theta[name] + h}), x0, tgt, steps)[0]
        lm = oracle_adjoint_dual(abi, cfg(**{name: theta[name] - h}), x0, tgt, steps)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[q]) <= 1e-5 * max(abs(g[q]), 1e-12), (name, fd, g[q])
    for s, (i, ax) in enumerate([(3, 0), (7, 2)]):
        h = 1e-6
        xp = [a.copy() for a in x0]
        xm = [a.copy() for a in x0]
        xp[ax][i] += h
        xm[ax][i] -= h
        fd = (oracle_adjoint_dual(abi, cfg(), xp, tgt, steps)[0] -
              oracle_adjoint_dual(abi, cfg(), xm, tgt, steps)[0]) / (2 * h)
        assert abs(fd - dx[s]) <= 1e-5 * max(abs(dx[s]), 1e-9)


def test_external_noise_zero_equals_sigma_zero(abi):
    """A step fed zero EM increments equals a step with sigma = 0: the given
    noise replaces the drawn one and nothing else."""
    from scenarios import colony_3d
    kw, st = colony_3d(abi, N=300, L=40.0, precision=abi.F64, p_death=0.0)
    kw = dict(kw, growth=0, fate=abi.FATE_NONE)
    a = OracleContext(abi, abi.make_config(**kw))
    b = OracleContext(abi, abi.make_config(**dict(kw, sigma=0.0)))
    a.upload(st)
    b.upload(st)
    for _ in range(5):
        a.step_noise(np.zeros((300, 3)))
        b.step(1)
    da, db = a.download(), b.download()
    for k in "xyz":
        np.testing.assert_array_equal(da[k], db[k])
