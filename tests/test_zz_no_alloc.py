"""cbm_cell_grid_noalloc against the context's cell grid (cbm_upload + cbm_get_grid).

The allocation-free entry point serves callers that cannot call cudaMalloc at
the moment they need a grid: code running while a framework captures the
stream into a CUDA graph, hosts whose device memory is owned by a pool
allocator (for instance a Julia process whose CUDA.jl pool holds the GPU), and
real-time loops that cannot take allocation latency.  Its scratch lives in a
static device array inside the library, shared by every call, so this test
calls it twice in a row with different inputs and checks both results.

This file is named so that pytest collects it last: the other tests have run
by the time it does, and it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import conftest
from scenarios import colony_3d

cbm = conftest.cbm
pytestmark = pytest.mark.gpu


def _bind(lib):
    f = lib.cbm_cell_grid_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                  C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double, C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_void_p]
    lib.cbm_noalloc_last_error.restype = C.c_char_p
    lib.cbm_noalloc_status.restype = C.c_int
    lib.cbm_noalloc_status.argtypes = [C.c_void_p]
    return f


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_noalloc_grid_matches_context_grid_twice(gpu_lib, abi, prec):
    import torch
    fn = _bind(gpu_lib)
    precision = abi.F32 if prec == "f32" else abi.F64
    tdt = torch.float32 if prec == "f32" else torch.float64
    for call, (N, seed) in enumerate([(20000, 7), (5000, 8)]):
        kw, st = colony_3d(abi, N=N, L=60.0, seed=seed, precision=precision,
                           neighbors=abi.NEIGH_CELL_LINKED)
        ctx = cbm.Context(abi.make_config(**kw))
        ctx.upload(st)  # builds the grid through the existing entry points
        ref = ctx.grid()
        nc = int(np.prod(ref["shape"]))
        dev = [torch.tensor(st[k], dtype=tdt, device="cuda") for k in ("x", "y", "z")]
        agent_cell = torch.full((N,), -1, dtype=torch.int32, device="cuda")
        cell_start = torch.full((nc + 1,), -1, dtype=torch.int32, device="cuda")
        cell_agents = torch.full((N,), -1, dtype=torch.int32, device="cuda")
        lo = (C.c_double * 3)(*kw["box_lo"])
        hi = (C.c_double * 3)(*kw["box_hi"])
        stream = torch.cuda.current_stream().cuda_stream
        rc = fn(dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), N, 3, precision, lo, hi,
                kw["cell_edge"], agent_cell.data_ptr(), cell_start.data_ptr(),
                cell_agents.data_ptr(), stream)
        assert rc == 0, gpu_lib.cbm_noalloc_last_error()
        # the scan's bounded waits all ended: the status of the finished call is OK
        assert gpu_lib.cbm_noalloc_status(stream) == 0, gpu_lib.cbm_noalloc_last_error()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(agent_cell.cpu().numpy(), ref["agent_cell"], err_msg=f"call {call}")
        np.testing.assert_array_equal(cell_start.cpu().numpy()[:nc], ref["cell_start"], err_msg=f"call {call}")
        assert int(cell_start[nc]) == N
        np.testing.assert_array_equal(cell_agents.cpu().numpy(), ref["cell_agents"], err_msg=f"call {call}")
        ctx.close()


def test_noalloc_rejects_sizes_beyond_the_static_array(gpu_lib, abi):
    fn = _bind(gpu_lib)
    lo = (C.c_double * 3)(0.0, 0.0, 0.0)
    hi = (C.c_double * 3)(1000.0, 1000.0, 1000.0)
    # 1000/1 + 2 cells per axis is far beyond CBM_NOALLOC_MAX_CELLS
    rc = fn(None, None, None, 0, 3, abi.F32, lo, hi, 1.0, None, None, None, None)
    assert rc == abi.CBM_ERR_ARG
    assert b"CBM_NOALLOC_MAX_CELLS" in gpu_lib.cbm_noalloc_last_error()
    rc = fn(None, None, None, 524289, 3, abi.F32, lo, hi, 100.0, None, None, None, None)
    assert rc == abi.CBM_ERR_ARG
    assert b"CBM_NOALLOC_MAX_AGENTS" in gpu_lib.cbm_noalloc_last_error()
