"""The device DGADI medium (cbm_medium_*) against the checker, bit for bit:
1D/2D/3D, Float32 and Float64, several fields with their own diffusion and
decay, a source field, unequal axes (the last axis's spacing sets r for every
axis), and the two workloads of examples/Implementation.ipynb.  Small media
run as one launch per call (a field per block, in shared memory); larger ones
take one launch per axis, staged or from global memory."""
import numpy as np
import pytest

from _oracle import OracleMedium

pytestmark = pytest.mark.gpu


def _run_both(abi, cbm, cfg, u0, src, steps):
    g = cbm._abi.DGADIMedium(cfg)
    o = OracleMedium(abi, cfg)
    g.upload(u0, src)
    o.upload(u0, src)
    out = []
    for s in steps:
        g.step(s)
        o.step(s)
        a, ta = g.download()
        b, tb = o.download()
        out.append((a, b, ta, tb))
    g.close()
    o.close()
    return out


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("dims,n", [(1, (33, 1, 1)), (2, (23, 17, 1)), (3, (13, 9, 11))])
def test_dgadi_bitexact(gpu_lib, abi, dims, n, prec):
    from conftest import cbm
    rng = np.random.default_rng(50 + dims)
    nodes = int(np.prod(n[:dims]))
    cfg = abi.make_medium_config(dims, n, (0.0, -1.0, 0.0), (1.0, 2.0, 0.7), 0.004,
                                 [1.0, 0.25, 3.0], [0.0, 0.5, 0.1], c_max=1.5,
                                 precision=abi.F32 if prec == "f32" else abi.F64)
    u0 = rng.uniform(0, 2, size=(3, nodes))
    src = rng.uniform(size=nodes) * (rng.uniform(size=nodes) < 0.2)
    for a, b, ta, tb in _run_both(abi, cbm, cfg, u0, src, [1, 4, 7]):
        assert a.dtype == b.dtype
        np.testing.assert_array_equal(a, b)
        assert ta == tb


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("dims,n", [(1, (30000, 1, 1)), (2, (900, 40, 1)), (3, (40, 30, 25))])
def test_dgadi_large_media_bitexact(gpu_lib, abi, dims, n, prec):
    """Media too large for one block's shared memory take one launch per axis:
    lines too long for a 96 KB tile of 32 lines (1D, and x in 2D) are solved
    from global memory, the others through shared-memory tiles."""
    from conftest import cbm
    rng = np.random.default_rng(60 + dims)
    nodes = int(np.prod(n[:dims]))
    cfg = abi.make_medium_config(dims, n, (0.0,) * 3, (3.0, 0.5, 1.0), 0.002, [0.8, 0.1],
                                 [0.05, 0.0], c_max=1.0,
                                 precision=abi.F32 if prec == "f32" else abi.F64)
    u0 = rng.uniform(size=(2, nodes))
    src = (rng.uniform(size=nodes) < 0.1).astype(float)
    for a, b, ta, tb in _run_both(abi, cbm, cfg, u0, src, [3, 5]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("dims,n,steps", [(2, (101, 101, 1), 50), (3, (101, 101, 101), 4)])
def test_dgadi_implementation_notebook_workload(gpu_lib, abi, dims, n, steps):
    """examples/Implementation.ipynb: co2 and co3 (D = 1 and 2) on [0,1]^dims,
    dt = 0.01, a source (vein = 1) at the central node, co2Max = 1, Float32
    as the reference's GPU platform runs it."""
    from conftest import cbm
    nodes = int(np.prod(n[:dims]))
    cfg = abi.make_medium_config(dims, n, (0.0,) * 3, (1.0,) * 3, 0.01, [1.0, 2.0],
                                 c_max=1.0, precision=abi.F32)
    src = np.zeros(tuple(reversed(n[:dims])), np.float32)
    src[tuple(round(k / 2) - 1 for k in reversed(n[:dims]))] = 1.0
    u0 = np.zeros((2, nodes), np.float32)
    (a, b, ta, tb), = _run_both(abi, cbm, cfg, u0, src.reshape(-1), [steps])
    np.testing.assert_array_equal(a, b)
    assert a.max() > 0 and np.isfinite(a).all()


def test_dgadi_errors(gpu_lib, abi):
    from conftest import cbm
    with pytest.raises(cbm._abi.CbmError):
        cbm._abi.DGADIMedium(abi.make_medium_config(2, (3, 8, 1), (0.0,) * 3, (1.0,) * 3, 0.01, [1.0]))
    m = cbm._abi.DGADIMedium(abi.make_medium_config(1, (8, 1, 1), (0.0,) * 3, (1.0,) * 3, 0.01, [1.0]))
    with pytest.raises(cbm._abi.CbmError):
        m.step(1)
    m.close()
