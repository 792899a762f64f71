"""Sharded sweeps over ranks: the partition, the routing of communities to
ranks and the host-side gather, run as two gloo processes on the CPU."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import conftest
import _gloo_worker as W

cbm = conftest.cbm


def test_partition_is_a_balanced_disjoint_cover():
    rng = np.random.default_rng(4)
    sizes = [int(v) for v in rng.integers(500, 20001, 512)]
    for world in (1, 2, 3, 8):
        parts = cbm.partition_communities(sizes, world)
        flat = sorted(c for p in parts for c in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[c] for c in p) for p in parts]
        # LPT bound: makespan <= mean load + largest job
        assert max(loads) <= sum(sizes) / world + max(sizes)
        assert cbm.partition_communities(sizes, world) == parts  # deterministic


def test_partition_edge_cases():
    assert cbm.partition_communities([], 2) == [[], []]
    assert cbm.partition_communities([5], 3) == [[0], [], []]
    assert cbm.partition_communities([3, 3, 3, 3], 2) == [[0, 2], [1, 3]]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_sweep_world2_matches_world1(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=W.run, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = np.load(tmp_path / "gathered.npy", allow_pickle=True)
    meta = np.load(tmp_path / "meta.npy")
    assert meta[0] == 11.0  # max over ranks of (10 + rank)
    sizes, states = W.sizes_and_states()
    assert int(meta[1]) == len(sizes)
    assert all(int(s) == 7 for s in meta[2:])
    # the same sweep on one rank
    descs = [W.Desc(n, c) for c, n in enumerate(sizes)]
    one = cbm.ShardedBatch(None, descs, rank=0, world=1, factory=W.FakeBatch)
    for c, st in enumerate(states):
        one.upload(c, st["x"], st["y"], st["z"])
    one.step(7)
    ref = one.gather()
    for c in range(len(sizes)):
        np.testing.assert_array_equal(got[c], ref[c]["x"])
    mine = [list(np.load(tmp_path / f"mine{r}.npy")) for r in range(world)]
    assert sorted(mine[0] + mine[1]) == list(range(len(sizes)))
    assert not set(mine[0]) & set(mine[1])
