"""The batched form: every community of one persistent launch follows the
plain path's trajectory bit for bit (same CLVD list order, same expression
order, same counter-based noise keyed by the community index)."""
import numpy as np
import pytest

import conftest
from scenarios import batched_sweep, make_descs, plain_config_for

cbm = conftest.cbm
pytestmark = pytest.mark.gpu


def small_sweep(abi, n_comm=10, seed=14):
    return batched_sweep(abi, n_comm=n_comm, n_lo=150, n_hi=2500, seed=seed)


def run_plain(abi, base, desc, state, tuning, steps):
    g = cbm.Context(abi.make_config(**plain_config_for(abi, base, desc, tuning)))
    g.upload(state)
    g.step(steps)
    return g.download()


# tile_agents: 0 gathers through L1/L2; 1000 mixes staged and unstaged
# communities in one launch; 18000 stages every community
@pytest.mark.parametrize("tuning", [
    dict(threads=256, ctas_per_sm=2, skin=0.3, rebuild_threshold=0.0, tile_agents=0),
    dict(threads=128, ctas_per_sm=4, skin=0.15, rebuild_threshold=0.0, tile_agents=1000),
    dict(threads=1024, ctas_per_sm=1, skin=0.6, rebuild_threshold=0.0, tile_agents=18000),
    dict(threads=512, ctas_per_sm=2, skin=1.5, rebuild_threshold=0.2, tile_agents=9000),
    # several lanes per agent (16 and 8 agents a warp): terms still added in list order
    dict(threads=256, ctas_per_sm=2, skin=0.3, rebuild_threshold=0.0, tile_agents=0,
         lanes_per_agent=2),
    dict(threads=512, ctas_per_sm=1, skin=1.0, rebuild_threshold=0.0, tile_agents=1000,
         lanes_per_agent=4),
    dict(threads=1024, ctas_per_sm=1, skin=0.6, rebuild_threshold=0.0, tile_agents=18000,
         lanes_per_agent=2)])
def test_batch_matches_plain_path(gpu_lib, abi, tuning):
    base, descs, states = small_sweep(abi)
    b = cbm.Batch(abi.make_config(**base), make_descs(abi, descs))
    b.set_tuning(**tuning)
    for c, st in enumerate(states):
        b.upload(c, st["x"], st["y"], st["z"])
    b.step(30)
    b.step(30)  # state carries over between launches
    for c in range(len(descs)):
        got = b.download(c)
        ref = run_plain(abi, base, descs[c], states[c], tuning, 60)
        assert got["step"] == 60
        for k in "xyz":
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"community {c} {k}")


def test_batch_graph_and_eager_agree(gpu_lib, abi):
    base, descs, states = small_sweep(abi, n_comm=6, seed=15)
    out = []
    for flags in (abi.SYNC, abi.SYNC | abi.NO_GRAPH):
        b = cbm.Batch(abi.make_config(**base), make_descs(abi, descs))
        for c, st in enumerate(states):
            b.upload(c, st["x"], st["y"], st["z"])
        b.step(40, flags)
        out.append([b.download(c) for c in range(len(descs))])
    for a, r in zip(*out):
        for k in "xyz":
            np.testing.assert_array_equal(a[k], r[k])


def test_batch_autotune_restores_state(gpu_lib, abi):
    base, descs, states = small_sweep(abi, n_comm=8, seed=16)
    b = cbm.Batch(abi.make_config(**base), make_descs(abi, descs))
    for c, st in enumerate(states):
        b.upload(c, st["x"], st["y"], st["z"])
    b.step(5)
    before = [b.download(c) for c in range(len(descs))]
    t = b.autotune(trial_steps=5)
    assert t.threads in (128, 256, 512, 1024) and t.skin > 0 and t.lanes_per_agent in (1, 2, 4)
    after = [b.download(c) for c in range(len(descs))]
    for a, r in zip(after, before):
        assert a["step"] == r["step"]
        for k in "xyz":
            np.testing.assert_array_equal(a[k], r[k])
    # and the chosen tuning still reproduces the plain path
    tuning = t.as_dict()
    b2 = cbm.Batch(abi.make_config(**base), make_descs(abi, descs))
    b2.set_tuning(**tuning)
    for c, st in enumerate(states):
        b2.upload(c, st["x"], st["y"], st["z"])
    b2.step(25)
    for c in (0, 3):
        ref = run_plain(abi, base, descs[c], states[c], tuning, 25)
        np.testing.assert_array_equal(b2.download(c)["x"], ref["x"])
