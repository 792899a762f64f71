"""The checker's Heun, RungeKutta4 and EulerHeun agent integrators
(src/integrators.jl:516-668,744-814) against a transcription of the
reference's step! functions, on CPU: three soft spheres in 2D with Full
neighbors (so the pair order is ascending j) and volume growth, Float64, bit
for bit.  EulerHeun reads its two draws from the shared counter-based stream."""
import numpy as np
import pytest

from conftest import cbm
import ctypes as C

from _oracle import OracleContext, load_oracle

abi = cbm._abi


def _f(x, krep=10.0, rrep=2.0, katt=1.0, ratt=3.0):
    """f(du, u): the pair sum of every agent, neighbors in ascending j."""
    n = x.shape[1]
    du = np.zeros_like(x)
    for i in range(n):
        acc = [0.0, 0.0]
        for j in range(n):
            if j == i:
                continue
            e = [x[0, i] - x[0, j], x[1, i] - x[1, j]]
            s2 = e[0] * e[0]
            s2 = s2 + e[1] * e[1]
            d = float(np.sqrt(s2))
            if d < rrep:
                F = krep * (rrep - d)
            elif d < ratt:
                F = -(katt * (d - rrep))
            else:
                continue
            sc = F / d
            acc = [acc[0] + sc * e[0], acc[1] + sc * e[1]]
        du[:, i] = acc
    return du


def _heun(x, v, g, dt):
    du = _f(x)
    h1 = x + du * dt
    du = _f(h1)
    x = (h1 + (x + du * dt)) / 2
    hv = v + g * dt
    return x, (hv + (v + g * dt)) / 2


def _rk4(x, v, g, dt):
    k1 = _f(x)
    h1 = x + k1 * dt / 2
    k2 = _f(h1)
    h1 = x + k2 * dt / 2
    k3 = _f(h1)
    h1 = x + k3 * dt
    k4 = _f(h1)
    x = x + (k1 + 2 * k2 + 2 * k3 + k4) * dt / 6
    return x, v + (g + 2 * g + 2 * g + g) * dt / 6


@pytest.mark.parametrize("name,integ,step", [("heun", abi.INT_HEUN, _heun), ("rk4", abi.INT_RK4, _rk4)])
def test_multistage_oracle_matches_transcription(name, integ, step):
    x0 = np.array([[1.0, 2.3, 2.9], [1.0, 1.4, 2.6]])
    v0 = np.array([1.0, 1.2, 1.5])
    g = np.array([0.5, 0.7, 0.9])
    kw = dict(dims=2, precision=abi.F64, n_max=3, box_lo=(0.0, 0.0), box_hi=(10.0, 10.0),
              dt=0.01, neighbors=abi.NEIGH_FULL, integrator=integ, k_rep=10.0, r_rep=2.0,
              k_att=1.0, r_att=3.0, growth=1)
    o = OracleContext(abi, abi.make_config(**kw))
    o.upload(dict(x=x0[0], y=x0[1], v=v0, g=g))
    x, v = x0.copy(), v0.copy()
    for _ in range(5):
        o.step(1)
        x, v = step(x, v, g, 0.01)
    got = o.download()
    np.testing.assert_array_equal(got["x"][:3], x[0])
    np.testing.assert_array_equal(got["y"][:3], x[1])
    np.testing.assert_array_equal(got["v"][:3], v)


def _normals(step, agent, stream, seed=7):
    lib = load_oracle(abi)
    out = np.zeros(2, np.float64)
    lib.oracle_normals(abi.F64, seed, step, agent, stream, 0, 2, out.ctypes.data)
    return out


def test_euler_heun_oracle_matches_transcription():
    """EulerHeun, the CPU branch of step!: h1 = u + f1 dt + g xi1 sqrt(dt),
    u = u + ((f1 + f2) dt + (g1 + g2) xi2 sqrt(dt)) / 2 with a fresh draw xi2
    (streams 0 and 4 of the shared generator), g = sigma for x and 0 for v."""
    x = np.array([[1.0, 2.3, 2.9], [1.0, 1.4, 2.6]])
    v = np.array([1.0, 1.2, 1.5])
    g = np.array([0.5, 0.7, 0.9])
    sig, dt = 0.3, 0.01
    kw = dict(dims=2, precision=abi.F64, n_max=3, box_lo=(0.0, 0.0), box_hi=(10.0, 10.0),
              dt=dt, seed=7, neighbors=abi.NEIGH_FULL, integrator=abi.INT_EULER_HEUN,
              sigma=sig, k_rep=10.0, r_rep=2.0, k_att=1.0, r_att=3.0, growth=1)
    o = OracleContext(abi, abi.make_config(**kw))
    o.upload(dict(x=x[0], y=x[1], v=v, g=g))
    sq = np.sqrt(dt)
    for step in range(4):
        o.step(1)
        xi1 = np.stack([_normals(step, i, 0) for i in range(3)], axis=1)
        xi2 = np.stack([_normals(step, i, 4) for i in range(3)], axis=1)
        f1 = _f(x)
        h1 = x + f1 * dt + sig * xi1 * sq
        f2 = _f(h1)
        x = x + ((f1 + f2) * dt + (sig + sig) * xi2 * sq) / 2
        v = v + ((g + g) * dt + (0.0 + 0.0) * xi2[0] * sq) / 2
    got = o.download()
    np.testing.assert_array_equal(got["x"][:3], x[0])
    np.testing.assert_array_equal(got["y"][:3], x[1])
    np.testing.assert_array_equal(got["v"][:3], v)
