"""Seeded synthetic scenarios shared by the parity tests and bench.py.

Each builder returns (config keyword arguments, initial state dict).  Shapes
and value distributions follow the workloads the reference's hot path is
measured on (soft-sphere aggregation, a growing 3D colony, chemotaxis on a
medium, many small communities, a differentiable ODE trajectory); sizes are
parameters so that tests run small cases and the bench the full ones.
"""
import json
import os

import numpy as np


def aggregation_2d(abi, N=4096, L=100.0, seed=1, precision=None, steps_hint=1000):
    """2D soft spheres in [0,L]^2, r=1, k=10, a=1, reflecting walls, Euler,
    dt=0.01, cell grid edge 3 (CellLinked)."""
    rng = np.random.default_rng(seed)
    kw = dict(dims=2, precision=abi.F64 if precision is None else precision, n_max=N,
              box_lo=(0.0, 0.0), box_hi=(L, L), dt=0.01, seed=seed,
              neighbors=abi.NEIGH_CELL_LINKED, cell_edge=3.0, integrator=abi.INT_EULER,
              k_rep=10.0, r_rep=2.0, k_att=1.0, r_att=3.0, att_form=abi.ATT_FROM_REP,
              walls=abi.WALLS_REFLECT)
    state = dict(x=rng.uniform(0, L, N), y=rng.uniform(0, L, N))
    return kw, state


def ball_radius(N, density=0.15):
    """Radius of a ball holding N agents at `density` agents per unit volume
    (0.15 is the packing density of spheres of radius 1)."""
    return (3 * N / (4 * np.pi * density)) ** (1 / 3)


def colony_3d(abi, N=10000, R=None, L=400.0, n_max=None, seed=2, precision=None,
              neighbors=None, p_death=1e-4, sigma=0.05, n_max_neighbors=64):
    """3D colony: N agents uniform in a radius-R ball centred in [0,L]^3 (R from
    the packing density 0.15 when not given),
    v ~ U(1,2), g ~ U(0.8,1.2), EM sigma, divide at v >= 2 into daughters at
    +-0.5 r, death probability p_death, CLVD with R_list 3.3 and rebuild at 0.15,
    dt = 0.005, Verlet rows of n_max_neighbors."""
    rng = np.random.default_rng(seed)
    R = ball_radius(N) if R is None else R
    u = rng.normal(size=(N, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    rad = R * rng.uniform(size=N) ** (1 / 3)
    p = L / 2 + u * rad[:, None]
    alg = abi.NEIGH_CLVD if neighbors is None else neighbors
    kw = dict(dims=3, precision=abi.F32 if precision is None else precision,
              n_max=n_max or int(1.2 * N), box_lo=(0.0,) * 3, box_hi=(L,) * 3, dt=0.005,
              seed=seed, neighbors=alg, cell_edge=3.3, skin=3.3, rebuild_threshold=0.15,
              n_max_neighbors=n_max_neighbors, integrator=abi.INT_EM, sigma=sigma, k_rep=10.0, r_rep=2.0,
              k_att=1.0, r_att=3.0, att_form=abi.ATT_FROM_REP, growth=1, fate=abi.FATE_VOLUME,
              v_div=2.0, div_sep=0.5, p_death=p_death)
    state = dict(x=p[:, 0], y=p[:, 1], z=p[:, 2], v=rng.uniform(1, 2, N), g=rng.uniform(0.8, 1.2, N))
    return kw, state


# Verlet row capacity of the growing colony: rows must hold every agent within
# the list radius 3.3, for the reference's CLVD to be defined (a fuller row
# writes past neighborList_).  The colony grown to 10^6 has up to about 820
# such agents (about 4 agents per unit volume in its core).
GROWN_COLONY_ROW = 1024


def growing_colony_3d(abi, n_target, precision=None, seed=2, headroom=1.2):
    """The configured 3D growing colony: 10^4 agents uniform in a radius-20
    ball centred in [0,400]^3 (colony_3d's model), with capacity
    headroom * n_target and Verlet rows that hold the grown state's partners."""
    return colony_3d(abi, N=10_000, R=20.0, L=400.0, n_max=int(headroom * n_target), seed=seed,
                     precision=precision, n_max_neighbors=GROWN_COLONY_ROW)


def packed_colony_3d(abi, N=1_000_000, density=0.15, L=400.0, seed=2, n_max=None, precision=None,
                     p_death=1e-4):
    """A grown colony snapshot: N agents at the packed density (agents per unit
    volume) in a ball centred in [0,L]^3, ages spread so that divisions occur
    every step (v ~ U(1,2))."""
    R = ball_radius(N, density)
    kw, state = colony_3d(abi, N=N, R=R, L=L, n_max=n_max or int(1.2 * N), seed=seed,
                          precision=precision, p_death=p_death)
    return kw, state


def chemotaxis_2d(abi, N=200000, L=1024.0, n_medium=1024, seed=3, bilinear=True, precision=None):
    """2D chemotaxis: agents in [0,L]^2 on an n_medium^2 FTCS grid (D=1, dt=0.2,
    decay 0.01, secretion 0.1), drift 0.5 grad c / (1 + |grad c|), sigma 0.1,
    repulsion k=10, r=1 (cutoff 2r), CellLinked edge 2."""
    rng = np.random.default_rng(seed)
    kw = dict(dims=2, precision=abi.F32 if precision is None else precision, n_max=N,
              box_lo=(0.0, 0.0), box_hi=(L, L), dt=0.2, seed=seed,
              neighbors=abi.NEIGH_CELL_LINKED, cell_edge=2.0, integrator=abi.INT_EM, sigma=0.1,
              k_rep=10.0, r_rep=2.0, k_att=0.0, r_att=2.0, medium=1,
              n_medium=(n_medium, n_medium), diff_D=1.0, decay=0.01, secretion=0.1,
              chemotaxis=0.5,
              medium_sampling=abi.MEDIUM_BILINEAR if bilinear else abi.MEDIUM_NEAREST)
    state = dict(x=rng.uniform(0, L, N), y=rng.uniform(0, L, N))
    return kw, state


def batched_sweep(abi, n_comm=512, n_lo=500, n_hi=20000, seed=4, dt=0.01, skin=0.3):
    """Parameter sweep: n_comm 3D soft-sphere communities, N_i ~ U[n_lo, n_hi],
    k, a, sigma each log-uniform in [0.3, 3] x (10, 1, 0.05), r = 1, cube side
    2.5 N_i^(1/3), positions uniform in the cube, EM, Float32.
    Returns (base config kwargs, community descriptor kwargs, initial states)."""
    rng = np.random.default_rng(seed)
    base = dict(dims=3, precision=abi.F32, n_max=1, dt=dt, seed=seed, neighbors=abi.NEIGH_CLVD,
                integrator=abi.INT_EM, n_max_neighbors=256, skin=3.0 + skin, cell_edge=3.0 + skin,
                rebuild_threshold=skin / 2, k_rep=10.0, r_rep=2.0, k_att=1.0, r_att=3.0)
    descs, states = [], []
    for c in range(n_comm):
        n = int(rng.integers(n_lo, n_hi + 1))
        L = 2.5 * n ** (1 / 3)
        f = np.exp(rng.uniform(np.log(0.3), np.log(3.0), 3))
        descs.append(dict(n=n, box_lo=(0.0, 0.0, 0.0), box_hi=(L, L, L), k_rep=10.0 * f[0],
                          r_rep=2.0, k_att=1.0 * f[1], r_att=3.0, sigma=0.05 * f[2], community=c))
        p = rng.uniform(0, L, size=(3, n))
        states.append(dict(x=p[0], y=p[1], z=p[2]))
    return base, descs, states


def plain_config_for(abi, base, desc, tuning):
    """The plain-path configuration whose trajectory a batched community reproduces."""
    R = max(desc["r_rep"], desc["r_att"]) + tuning["skin"]
    thr = tuning["rebuild_threshold"] if tuning["rebuild_threshold"] > 0 else tuning["skin"] / 2
    return dict(dims=3, precision=abi.F32, n_max=desc["n"], box_lo=desc["box_lo"],
                box_hi=desc["box_hi"], dt=base["dt"], seed=base["seed"],
                community=desc["community"], neighbors=abi.NEIGH_CLVD, skin=R, cell_edge=R,
                rebuild_threshold=thr, n_max_neighbors=base["n_max_neighbors"],
                integrator=abi.INT_EM, sigma=desc["sigma"], k_rep=desc["k_rep"],
                r_rep=desc["r_rep"], k_att=desc["k_att"], r_att=desc["r_att"])


def make_descs(abi, descs):
    out = []
    for d in descs:
        x = abi.CbmCommunityDesc()
        x.n = d["n"]
        x.box_lo = (C_double3 := type(x.box_lo))(*d["box_lo"])
        x.box_hi = C_double3(*d["box_hi"])
        for k in ("k_rep", "r_rep", "k_att", "r_att", "sigma", "community"):
            setattr(x, k, d[k])
        out.append(x)
    return out


def adjoint_problem(abi, N=65536, L=80.0, seed=5, steps=200, precision=None, theta=(10.0, 1.0, 2.0)):
    """Differentiable 3D ODE trajectory: N agents uniform in [0,L]^3, soft
    spheres with theta = (k, a, 2r), forward Euler dt=0.01, CellLinked edge
    3.3; the target comes from the same simulation at theta* = theta (1 +
    0.1 N(0,1)).  Returns (config kwargs, x0, theta*)."""
    rng = np.random.default_rng(seed)
    k, a, rho = theta
    kw = dict(dims=3, precision=abi.F64 if precision is None else precision, n_max=N,
              box_lo=(0.0,) * 3, box_hi=(L,) * 3, dt=0.01, seed=seed,
              neighbors=abi.NEIGH_CELL_LINKED, cell_edge=3.3, integrator=abi.INT_EULER,
              k_rep=k, r_rep=rho, k_att=a, r_att=1.5 * rho, att_form=abi.ATT_FROM_REP)
    x0 = [rng.uniform(0, L, N) for _ in range(3)]
    star = tuple(t * (1 + 0.1 * z) for t, z in zip(theta, rng.normal(size=3)))
    return kw, x0, star


def profile_colony_3d(abi, r_edges, r_counts, v_edges, v_counts, g_edges, g_counts, N=None,
                      L=400.0, seed=12, precision=None, n_max=None):
    """A colony drawn from measured distributions instead of grown: agents at
    the radial density of the histogram (r_edges, r_counts) around the centre
    of [0,L]^3 (uniform in volume inside each shell), with volumes and growth
    rates drawn from their histograms (uniform inside each bin).  N defaults
    to the histogram's total.  The configuration is colony_3d's."""
    rng = np.random.default_rng(seed)
    r_counts = np.asarray(r_counts, np.float64)
    N = int(r_counts.sum()) if N is None else int(N)

    def draw(edges, counts, n):
        edges = np.asarray(edges, np.float64)
        p = np.asarray(counts, np.float64)
        k = rng.choice(len(p), size=n, p=p / p.sum())
        return k, edges[k] + (edges[k + 1] - edges[k]) * rng.uniform(size=n)

    k, _ = draw(r_edges, r_counts, N)
    r_edges = np.asarray(r_edges, np.float64)
    lo3, hi3 = r_edges[k] ** 3, r_edges[k + 1] ** 3
    rad = np.cbrt(lo3 + (hi3 - lo3) * rng.uniform(size=N))
    u = rng.normal(size=(N, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    p = L / 2 + u * rad[:, None]
    _, v = draw(v_edges, v_counts, N)
    _, g = draw(g_edges, g_counts, N)
    kw, _ = colony_3d(abi, N=1, R=1.0, L=L, n_max=n_max or int(1.2 * N), seed=seed,
                      precision=precision)
    state = dict(x=p[:, 0], y=p[:, 1], z=p[:, 2], v=v, g=g)
    return kw, state


def medium_colony(abi, dims, N=3000, L=40.0, n_medium=40, seed=6, bilinear=True, precision=None,
                  neighbors=None, uptake=0.05, secretion=0.1, chemotaxis=0.5, dt=0.05):
    """Agents on a 1D/2D/3D FTCS medium (unit spacing by default): soft-sphere
    repulsion (k=10, r=1), EM noise sigma 0.1, secretion, first-order uptake
    and chemotactic drift, D=1, decay 0.01, CellLinked edge 2 unless another
    neighbor algorithm is given."""
    rng = np.random.default_rng(seed)
    alg = abi.NEIGH_CELL_LINKED if neighbors is None else neighbors
    kw = dict(dims=dims, precision=abi.F32 if precision is None else precision, n_max=N,
              box_lo=(0.0,) * dims, box_hi=(L,) * dims, dt=dt, seed=seed, neighbors=alg,
              cell_edge=2.4, skin=2.4, n_max_neighbors=64, integrator=abi.INT_EM, sigma=0.1,
              k_rep=10.0, r_rep=2.0, k_att=0.0, r_att=2.0, medium=1,
              n_medium=(n_medium,) * dims, diff_D=1.0, decay=0.01, secretion=secretion,
              uptake=uptake, chemotaxis=chemotaxis,
              medium_sampling=abi.MEDIUM_BILINEAR if bilinear else abi.MEDIUM_NEAREST)
    p = rng.uniform(0, L, size=(dims, N))
    state = {k: p[d] for d, k in enumerate("xyz"[:dims])}
    return kw, state


def grown_colony_stand_in(abi, precision=None, seed=12):
    """A stand-in for the colony grown to 10^6 that is built without growing
    it: agents drawn from the grown colony's measured radial density, volume
    and growth-rate histograms (tests/golden/grown_colony_1e6_profile.json),
    numbered in the order of the cell grid (edge 3.3, x fastest).  Its agents
    have the grown state's partner counts (about 354 within the cutoff), and
    the CPU restatement steps it at least as fast as the grown state: the
    grown colony's own numbering keeps some locality (sisters sit next to each
    other), which a random numbering loses and the cell numbering exceeds."""
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "grown_colony_1e6_profile.json")) as f:
        prof = json.load(f)
    kw, st = profile_colony_3d(abi, prof["r_edges"], prof["r_counts"], prof["v_edges"],
                               prof["v_counts"], prof["g_edges"], prof["g_counts"], seed=seed,
                               precision=precision)
    c = np.floor(np.stack([st["x"], st["y"], st["z"]]) / 3.3).astype(np.int64)
    order = np.lexsort((c[0], c[1], c[2]))
    st = {k: np.asarray(v)[order] for k, v in st.items()}
    kw = dict(kw, n_max_neighbors=GROWN_COLONY_ROW)
    return kw, st
