"""Uptake of the medium by agents, on the CPU checker (runs without a GPU).

Agent i adds w_q (secretion dt - (uptake dt) c_q) to each node q of its
sampling stencil, c_q the committed value; with uptake > 0 the medium's DE
step reads the field clamped at zero.  The reference has no uptake term (a
user writes `c__[...] -= ...` in a rule, auxiliar.jl:353-365), so these are
known answers of the definition: first-order decay at one node, the mass
balance of a step, the clamp, and that uptake = 0 leaves secretion alone.
"""
import numpy as np
import pytest

from _oracle import OracleContext


def still_agents(abi, dims, n_medium, L, dt, **kw):
    """Agents that do not move (no forces, no noise, no neighbors) on a medium
    without diffusion or decay unless given."""
    base = dict(dims=dims, n_max=64, box_lo=(0.0,) * dims, box_hi=(L,) * dims, dt=dt,
                medium=1, n_medium=(n_medium,) * dims, medium_sampling=abi.MEDIUM_BILINEAR)
    base.update(kw)
    return abi.make_config(**base)


def bilinear_weights(p, L, n, dims):
    """Nodes and weights of the multilinear stencil (nodes at cell centres,
    indices clamped), the same definition as the library's."""
    dx = L / n
    i0, i1, t = [], [], []
    for d in range(dims):
        s = p[d] / dx - 0.5
        f = np.floor(s)
        t.append(s - f)
        a = int(f)
        i0.append(min(max(a, 0), n - 1))
        i1.append(min(max(a + 1, 0), n - 1))
    out = []
    for q in range(1 << dims):
        lin, mul, w = 0, 1, 1.0
        for d in range(dims):
            h = (q >> d) & 1
            lin += (i1[d] if h else i0[d]) * mul
            mul *= n
            w *= t[d] if h else 1.0 - t[d]
        out.append((lin, w))
    return out


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_uptake_at_a_node_centre_decays_geometrically(abi, dims):
    """One agent at the centre of a node takes up (uptake dt) of that node's
    content each step: c_n = c_0 (1 - uptake dt)^n, and nothing elsewhere."""
    n, L, dt, u = 8, 8.0, 0.1, 0.7
    cfg = still_agents(abi, dims, n, L, dt, uptake=u)
    c0 = np.full(n ** dims, 2.0)
    pos = {k: np.array([3.5]) for k in "xyz"[:dims]}  # centre of node 3 on every axis
    o = OracleContext(abi, cfg)
    o.upload(dict(pos, c=c0))
    node = sum(3 * n ** d for d in range(dims))
    for step in range(1, 21):
        o.step(1)
        c = o.download()["c"]
        assert abs(c[node] - 2.0 * (1 - u * dt) ** step) <= 1e-12 * 2.0
        others = np.delete(c, node)
        assert np.all(others == 2.0)


@pytest.mark.parametrize("dims", [1, 2, 3])
@pytest.mark.parametrize("sampling", ["nearest", "bilinear"])
def test_mass_balance_of_one_step(abi, dims, sampling):
    """Without diffusion and decay, one step changes the total by
    N secretion dt - uptake dt sum_q W_q c_q, W_q the summed stencil weights
    of the agents on node q (weights 1 at the nearest node)."""
    rng = np.random.default_rng(40 + dims)
    n, L, dt, s, u, N = 10, 10.0, 0.05, 0.3, 0.9, 40
    cfg = still_agents(abi, dims, n, L, dt, secretion=s, uptake=u,
                       medium_sampling=abi.MEDIUM_BILINEAR if sampling == "bilinear"
                       else abi.MEDIUM_NEAREST)
    c0 = rng.uniform(0.5, 1.5, n ** dims)
    p = rng.uniform(0, L, (dims, N))
    o = OracleContext(abi, cfg)
    o.upload(dict({k: p[d] for d, k in enumerate("xyz"[:dims])}, c=c0))
    o.step(1)
    c1 = o.download()["c"]
    W = np.zeros(n ** dims)
    for a in range(N):
        if sampling == "bilinear":
            for lin, w in bilinear_weights(p[:, a], L, n, dims):
                W[lin] += w
        else:
            q = np.minimum((p[:, a] // (L / n)).astype(int), n - 1)
            W[sum(int(q[d]) * n ** d for d in range(dims))] += 1.0
    expect = c0.sum() + N * s * dt - u * dt * np.sum(W * c0)
    assert abs(c1.sum() - expect) <= 1e-12 * c0.sum()
    np.testing.assert_allclose(c1, c0 + W * (s * dt) - (u * dt) * W * c0, rtol=1e-12, atol=1e-13)


def test_uptake_beyond_the_content_clamps_at_zero(abi):
    """uptake dt = 1.5 at a node centre would leave -0.5 c: the DE step reads
    0 there, so the node is empty after the step and stays empty."""
    cfg = still_agents(abi, 2, 6, 6.0, 0.05, uptake=30.0)
    o = OracleContext(abi, cfg)
    c0 = np.full(36, 1.0)
    o.upload(dict(x=np.array([2.5]), y=np.array([2.5]), c=c0))
    for _ in range(3):
        o.step(1)
        c = o.download()["c"]
        assert c[2 + 2 * 6] == 0.0
        assert np.all(np.delete(c, 2 + 2 * 6) == 1.0)


def test_clamp_meets_diffusion(abi):
    """With diffusion the clamped node is read as 0 by its neighbours' Laplacian."""
    n, dt, D = 5, 0.1, 1.0
    cfg = still_agents(abi, 1, n, float(n), dt, uptake=20.0, diff_D=D)
    o = OracleContext(abi, cfg)
    o.upload(dict(x=np.array([2.5]), c=np.ones(n)))
    o.step(1)
    c = o.download()["c"]
    # node 2: 1 - 2 = -1 -> 0, then 0 + dt D (1 - 0 + 1) = 0.2; nodes 1 and 3:
    # 1 + dt D (0 - 2 + 1) = 0.9; the border nodes 0 and 4 are frozen
    np.testing.assert_allclose(c, [1.0, 0.9, 0.2, 0.9, 1.0], rtol=1e-15)


def test_zero_uptake_is_plain_secretion(abi):
    """uptake = 0 gives exactly the secretion-only step (no clamp either)."""
    rng = np.random.default_rng(5)
    kw = dict(secretion=0.4, diff_D=0.5, decay=0.01)
    p = rng.uniform(0, 10, (2, 30))
    c0 = rng.uniform(-0.2, 1.0, 100)  # negative values stay: no clamp without uptake
    out = []
    for extra in ({}, {"uptake": 0.0}):
        o = OracleContext(abi, still_agents(abi, 2, 10, 10.0, 0.05, **kw, **extra))
        o.upload(dict(x=p[0], y=p[1], c=c0))
        o.step(5)
        out.append(o.download()["c"])
    np.testing.assert_array_equal(out[0], out[1])
    assert np.min(out[0]) < 0
