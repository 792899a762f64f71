"""The checker's DGADI medium (CBMIntegrators.DGADI, src/integrators.jl:141-428,
817-937) against an independent transcription of the reference's Julia loops,
on CPU.  Julia cannot run here, so the transcription below follows
tridiagonal{1,2,3}D{x,y,z}CPU! and step!(::DGADI) statement by statement,
1-based like the source, with the arrays the reference keeps (u, u_new,
c_star, d_star, all copies of u0).  In Float32 it reproduces Julia's
promotion: `1.0 / x` with x::Float32 is Float64, and the products with it are
rounded when stored into the Float32 arrays."""
import numpy as np
import pytest

from conftest import cbm
from _oracle import OracleMedium

abi = cbm._abi


def _julia_dgadi(u0, src, n, dims, dt, box, diffusion, decay, c_max, steps, T):
    """step!(::DGADI) with the medium model f = s (c_max - u) - decay u inside."""
    nf = len(diffusion)  # arrays are indexed (l, i, j, k) as in the reference

    def arr(a):
        return np.array(a, dtype=T).reshape((nf,) + tuple(reversed(n[:dims]))).transpose(
            (0,) + tuple(range(dims, 0, -1))).copy()

    u = arr(u0)
    s = np.array(src, dtype=T).reshape(tuple(reversed(n[:dims]))).transpose(
        tuple(range(dims - 1, -1, -1))).copy()
    u_new = u.copy()  # c_star and d_star are kept per line below
    # r = dt ./ (nDims .* ((simBox[:,2] .- simBox[:,1]) ./ NMedium).^2), column [l, dims]
    dxl = (box[1][dims - 1] - box[0][dims - 1]) / float(n[dims - 1])
    r = dt / (float(dims) * (dxl * dxl))
    sub = [T(-D * r) for D in diffusion]
    sup = [T(-D * r) for D in diffusion]
    main = [T(1.0 + 2.0 * D * r) for D in diffusion]

    def line(l, get, setn, nx):
        # one line of tridiagonal*CPU!, indices 1..nx; get(i) reads x_old, setn writes x_new
        cs, ds = {}, {}
        cs[2] = sup[l] / main[l]
        ds[2] = (get(2) - sub[l] * get(1)) / main[l]
        for i in range(3, nx - 1):
            m = 1.0 / float(main[l] - sub[l] * cs[i - 1])
            cs[i] = T(float(sup[l]) * m)
            ds[i] = T(float(get(i) - sub[l] * ds[i - 1]) * m)
        m = 1.0 / float(main[l] - sub[l] * cs[nx - 2])
        ds[nx - 1] = T(float((get(nx - 1) - sup[l] * get(nx)) - sub[l] * ds[nx - 2]) * m)
        setn(nx - 1, ds[nx - 1])
        xn = {nx - 1: ds[nx - 1]}
        for i in range(nx - 2, 1, -1):
            xn[i] = ds[i] - cs[i] * xn[i + 1]
            setn(i, xn[i])

    for _ in range(steps):
        du = np.zeros_like(u)
        it = np.ndindex(*n[:dims])
        for idx in it:
            inside = all(0 < idx[d] < n[d] - 1 for d in range(dims))
            if inside:
                for l in range(nf):
                    du[(l,) + idx] = s[idx] * (T(c_max) - u[(l,) + idx]) - T(decay[l]) * u[(l,) + idx]
        u = u + du
        for a in range(dims):
            others = [d for d in range(dims) if d != a]
            ranges = [range(1, n[d] - 1) for d in others]
            for rest in np.ndindex(*[len(rg) for rg in ranges]) if others else [()]:
                pos = [0] * dims
                for d, k in zip(others, rest):
                    pos[d] = k + 1
                for l in range(nf):
                    def key(i, pos=pos, l=l, a=a):
                        p = list(pos)
                        p[a] = i - 1
                        return (l,) + tuple(p)
                    line(l, lambda i: u[key(i)], lambda i, v: u_new.__setitem__(key(i), v), n[a])
            u = u_new.copy()
    return u.transpose((0,) + tuple(range(dims, 0, -1))).reshape(nf, -1)


CASES = [
    (1, (9, 1, 1)),
    (2, (7, 6, 1)),
    (3, (5, 6, 4)),
]


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("dims,n", CASES)
def test_oracle_dgadi_matches_julia_transcription(dims, n, prec):
    rng = np.random.default_rng(40 + dims)
    T = np.float64 if prec == "f64" else np.float32
    nodes = int(np.prod(n[:dims]))
    diffusion, decay = [1.0, 2.0], [0.0, 0.3]
    box = ((0.0, 0.0, 0.0), (1.0, 2.0, 0.5))
    u0 = rng.uniform(0, 1, size=(2, nodes))
    src = (rng.uniform(size=nodes) < 0.3).astype(float)
    cfg = abi.make_medium_config(dims, n, box[0], box[1], 0.01, diffusion, decay, c_max=1.0,
                                 precision=abi.F64 if prec == "f64" else abi.F32)
    o = OracleMedium(abi, cfg)
    o.upload(u0, src)
    o.step(3)
    got, t = o.download()
    want = _julia_dgadi(u0.reshape(-1), src, list(n), dims, 0.01, box, diffusion, decay, 1.0,
                        3, T)
    assert got.dtype == T
    np.testing.assert_array_equal(got.reshape(2, -1), want)
    assert t == 0.01 + 0.01 + 0.01


def test_oracle_dgadi_line_solves_the_system():
    """One 1D step with no explicit term: the interior solves
    (1 + 2Dr) u_i - Dr (u_{i-1} + u_{i+1}) = u_i^old with the ends fixed."""
    n, D, dt = 12, 0.7, 0.05
    rng = np.random.default_rng(3)
    u0 = rng.uniform(size=n)
    cfg = abi.make_medium_config(1, (n, 1, 1), (0.0,) * 3, (1.0,) * 3, dt, [D], precision=abi.F64)
    o = OracleMedium(abi, cfg)
    o.upload(u0[None, :])
    o.step(1)
    u, _ = o.download()
    u = u[0]
    r = dt / (1.0 * (1.0 / n) ** 2)
    assert u[0] == u0[0] and u[-1] == u0[-1]
    lhs = (1 + 2 * D * r) * u[1:-1] - D * r * (u[:-2] + u[2:])
    np.testing.assert_allclose(lhs, u0[1:-1], rtol=1e-12, atol=1e-12)


def test_oracle_dgadi_border_and_no_diffusion():
    """D = 0 leaves only the explicit step; the border keeps its values."""
    n = (6, 5, 1)
    rng = np.random.default_rng(4)
    u0 = rng.uniform(size=(1, 30))
    src = rng.uniform(size=30)
    cfg = abi.make_medium_config(2, n, (0.0,) * 3, (1.0,) * 3, 0.1, [0.0], [0.25], c_max=2.0,
                                 precision=abi.F64)
    o = OracleMedium(abi, cfg)
    o.upload(u0, src)
    o.step(1)
    u, _ = o.download()
    g = u0.reshape(5, 6).copy()
    s = src.reshape(5, 6)
    inner = (slice(1, -1), slice(1, -1))
    g[inner] = g[inner] + (s[inner] * (2.0 - g[inner]) - 0.25 * g[inner])
    np.testing.assert_array_equal(u.reshape(5, 6), g)
