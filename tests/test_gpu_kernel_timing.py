"""Kernel timing inside the step graphs (cbm_set_kernel_timing /
cbm_kernel_times): every kernel of a replayed step is timed by events on the
library's stream, the timing changes no result, and the plain step graphs
captured before it are replayed again after it."""
import numpy as np
import pytest

import conftest
from scenarios import colony_3d

cbm = conftest.cbm
pytestmark = pytest.mark.gpu


def test_kernel_times_of_graph_replays(gpu_lib, abi):
    kw, st = colony_3d(abi, N=3000, L=60.0, n_max=6000, p_death=2e-3)
    cfg = abi.make_config(**kw)
    a, b = cbm.Context(cfg), cbm.Context(cfg)
    a.upload(st)
    b.upload(st)
    a.step(2)  # the plain graphs of both parities
    a.set_kernel_timing(True)
    for _ in range(4):
        a.step(1)
        times = a.kernel_times()
        names = [n for n, _ in times]
        assert len(times) == a.kernels_per_step()
        assert "k_agent_de" in names and "k_sort_place" in names
        assert all(ms > 0 for _, ms in times)
    a.set_kernel_timing(False)
    a.step(3)
    b.step(9)
    sa, sb = a.download(), b.download()
    for k in ("x", "y", "z", "v", "id"):
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)
    with pytest.raises(cbm.CbmError):
        a.kernel_times()  # timing is off again


@pytest.mark.parametrize("walls", [False, True])
def test_medium_branches_match_series(gpu_lib, abi, walls):
    """With a medium the force kernel runs on a branch of its own, in
    parallel with the medium kernels (forked at the start of the step, or
    after the agents' rule when reflecting walls need one), and a call of
    eight steps or more replays chained graphs in which the next step's
    gradient runs beside each update; with kernel timing on, and in profiled
    steps, the kernels run in series.  All give the same bits, in graph
    replays (two chains and four single steps here) and in eager steps."""
    from scenarios import medium_colony
    kw, st = medium_colony(abi, 3, N=4000, L=48.0, n_medium=48)
    if walls:
        kw["walls"] = abi.WALLS_REFLECT
    cfg = abi.make_config(**kw)
    ctxs = [cbm.Context(cfg) for _ in range(4)]
    for x in ctxs:
        x.upload(st)
    ctxs[0].step(20)                                  # chained and forked graphs
    ctxs[1].step(20, flags=abi.SYNC | abi.NO_GRAPH)   # forked eager steps
    ctxs[2].set_kernel_timing(True)                   # graphs in series
    ctxs[2].step(20)
    for _ in range(20):                               # eager steps in series
        ctxs[3].profile_step()
    ref = ctxs[0].download()
    for x in ctxs[1:]:
        s = x.download()
        for k in ("x", "y", "z", "id", "c", "gx", "gy", "gz"):
            np.testing.assert_array_equal(s[k], ref[k], err_msg=k)
