"""The explicit medium in 1D, 2D and 3D on the device against the CPU checker:
FTCS diffusion with decay (macros.jl:203-258), secretion and first-order
uptake by the agents, and chemotactic drift along the gradient.

Bit-exact wherever each node's additions have one order: the gather path
(bilinear sampling with CellLinked neighbors, agents added in index order)
and nearest-node sampling (every agent of a node adds the same term, so the
atomic sum does not depend on the order).  Bilinear sampling with a Verlet
algorithm adds unequal terms through atomics in any order: 1e-5 relative
(Float32), stated in that test.
"""
import numpy as np
import pytest

import conftest
from _oracle import OracleContext
from scenarios import chemotaxis_2d, medium_colony
from test_gpu_parity import assert_same_state

cbm = conftest.cbm
pytestmark = pytest.mark.gpu

SIZES = {1: dict(N=600, L=200.0, n_medium=200), 2: dict(N=2000, L=64.0, n_medium=64),
         3: dict(N=3000, L=24.0, n_medium=24)}


def both(abi, kw, state):
    cfg = abi.make_config(**kw)
    g = cbm.Context(cfg)
    o = OracleContext(abi, cfg, threads=4)
    g.upload(state)
    o.upload(state)
    return g, o


def keys(dims):
    return list("xyz"[:dims]) + ["c"] + ["g" + a for a in "xyz"[:dims]]


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("bilinear", [False, True])
@pytest.mark.parametrize("dims", [1, 2, 3])
def test_medium_secretion_uptake_chemotaxis(gpu_lib, abi, dims, bilinear, prec):
    kw, st = medium_colony(abi, dims, **SIZES[dims], bilinear=bilinear,
                           precision=abi.F32 if prec == "f32" else abi.F64)
    g, o = both(abi, kw, st)
    for _ in range(3):
        g.step(15)
        o.step(15)
        a, b = g.download(), o.download()
        assert_same_state(a, b, keys(dims))
    assert np.max(a["c"]) > 0


@pytest.mark.parametrize("shape", [(37, 45, 70), (100, 33, 9), (64, 64, 200)])
def test_medium_3d_tiles_and_runs(gpu_lib, abi, shape):
    """Medium shapes that leave partial tiles in x and y and runs of z planes
    of every length (including a last run of one plane)."""
    nx, ny, nz = shape
    kw, st = medium_colony(abi, 3, N=2500, L=float(max(shape)), n_medium=1)
    kw.update(box_hi=(float(nx), float(ny), float(nz)), n_medium=(nx, ny, nz), decay=0.02)
    rng = np.random.default_rng(8)
    st = dict(x=rng.uniform(0, nx, 2500), y=rng.uniform(0, ny, 2500), z=rng.uniform(0, nz, 2500),
              c=rng.uniform(0, 1, nx * ny * nz))
    g, o = both(abi, kw, st)
    g.step(12)
    o.step(12)
    assert_same_state(g.download(), o.download(), keys(3))


@pytest.mark.parametrize("dims", [2, 3])
def test_medium_atomic_rule_paths(gpu_lib, abi, dims):
    """Secretion and uptake applied by the agent rule with atomics (a Verlet
    algorithm): exact with nearest-node sampling, 1e-5 relative with bilinear
    sampling (unequal terms added in any order)."""
    for bilinear in (False, True):
        kw, st = medium_colony(abi, dims, **SIZES[dims], bilinear=bilinear,
                               neighbors=abi.NEIGH_CLVD)
        kw.update(dt=0.02)
        g, o = both(abi, kw, st)
        g.step(20)
        o.step(20)
        a, b = g.download(), o.download()
        if not bilinear:
            assert_same_state(a, b, keys(dims))
        else:
            for k in keys(dims):
                np.testing.assert_allclose(a[k], b[k], rtol=1e-5, atol=1e-5, err_msg=k)


@pytest.mark.parametrize("dims", [1, 3])
def test_uptake_clamp_on_device(gpu_lib, abi, dims):
    """uptake dt above 1 empties the nodes under the agents; the DE step reads
    them as zero (no negative concentration), bit-exact with the checker."""
    kw, st = medium_colony(abi, dims, **SIZES[dims], uptake=30.0, secretion=0.0, chemotaxis=0.2)
    st["c"] = np.ones(SIZES[dims]["n_medium"] ** dims)
    g, o = both(abi, kw, st)
    g.step(10)
    o.step(10)
    a, b = g.download(), o.download()
    assert_same_state(a, b, keys(dims))
    assert np.min(a["c"]) >= 0 and np.min(a["c"]) < 0.5


def test_chemotaxis_2d_with_uptake(gpu_lib, abi):
    kw, st = chemotaxis_2d(abi, N=3000, L=128.0, n_medium=128)
    kw["uptake"] = 0.05
    g, o = both(abi, kw, st)
    for _ in range(4):
        g.step(25)
        o.step(25)
        assert_same_state(g.download(), o.download(), ["x", "y", "c", "gx", "gy"])


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("dims", [2, 3])
def test_secretion_runs_sparse_and_crowded(gpu_lib, abi, dims, prec):
    """The gather by runs of 32 nodes: a crowded clump (runs that more than 32
    agents touch take the per-node path), sparse agents (runs of a few
    agents, untouched runs left as they are), agents beyond the box (clamped
    stencils that put two terms on one node) and a medium width that is not
    a multiple of 32."""
    nm = {2: (150, 70), 3: (75, 30, 26)}[dims]
    L = tuple(float(v) for v in nm)
    kw, _ = medium_colony(abi, dims, N=4500, L=L[0], n_medium=1,
                          precision=abi.F32 if prec == "f32" else abi.F64)
    kw.update(box_hi=L, n_medium=nm)
    rng = np.random.default_rng(17)
    n_clump, n_sparse, n_out = 1500, 2500, 500
    lo = np.array([0.2 * v for v in L])
    clump = lo[:, None] + rng.uniform(0, 10.0, (dims, n_clump))
    sparse = rng.uniform(0, 1, (dims, n_sparse)) * np.array(L)[:, None]
    out = rng.uniform(-1.5, 1.5, (dims, n_out)) + np.where(
        rng.uniform(0, 1, (dims, n_out)) < 0.5, 0.0, np.array(L)[:, None])
    p = np.concatenate([clump, sparse, out], axis=1)
    p = p[:, rng.permutation(p.shape[1])]
    st = {k: p[d] for d, k in enumerate("xyz"[:dims])}
    st["c"] = rng.uniform(0, 1, int(np.prod(nm)))
    g, o = both(abi, kw, st)
    for _ in range(2):
        g.step(6)
        o.step(6)
        assert_same_state(g.download(), o.download(), keys(dims))


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("dx", [0.5, 0.75, 1.5625])
@pytest.mark.parametrize("dims", [2, 3])
def test_medium_spacings(gpu_lib, abi, dims, dx, prec):
    """Spacings other than 1: powers of two (dx^2 and 2 dx applied through
    their exact reciprocals) and others (divided), on medium widths whose rows
    are a multiple of 16 bytes (the TMA-fed 3D stencils) and widths that are
    not (the register-pipelined ones)."""
    for nm in {2: [(40, 30), (37, 29)], 3: [(24, 14, 12), (21, 14, 12)]}[dims]:
        L = tuple(v * dx for v in nm)
        kw, _ = medium_colony(abi, dims, N=1500, L=L[0], n_medium=1, dt=0.02,
                              precision=abi.F32 if prec == "f32" else abi.F64)
        kw.update(box_hi=L, n_medium=nm)
        rng = np.random.default_rng(23)
        st = {k: rng.uniform(0, L[d], 1500) for d, k in enumerate("xyz"[:dims])}
        st["c"] = rng.uniform(0, 1, int(np.prod(nm)))
        g, o = both(abi, kw, st)
        g.step(8)
        o.step(8)
        assert_same_state(g.download(), o.download(), keys(dims))


@pytest.mark.parametrize("shape", [(32, 5, 3), (8, 40, 2), (16, 3, 1), (40, 1, 6)])
def test_medium_3d_thin_shapes(gpu_lib, abi, shape):
    """3D media thinner than a tile (and a single plane or row): rows of a
    multiple of 16 bytes take the TMA-fed stencils, whose plane boxes then
    reach far beyond the field and read zeros there."""
    nx, ny, nz = shape
    kw, _ = medium_colony(abi, 3, N=400, L=float(max(shape)), n_medium=1)
    kw.update(box_hi=(float(nx), float(ny), float(nz)), n_medium=(nx, ny, nz))
    rng = np.random.default_rng(31)
    st = dict(x=rng.uniform(0, nx, 400), y=rng.uniform(0, ny, 400), z=rng.uniform(0, nz, 400),
              c=rng.uniform(0, 1, nx * ny * nz))
    g, o = both(abi, kw, st)
    g.step(9)
    o.step(9)
    assert_same_state(g.download(), o.download(), keys(3))
