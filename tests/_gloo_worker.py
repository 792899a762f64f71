"""Worker of the world-size-2 gloo tests (spawned processes; CPU only)."""
import importlib.util
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_package():
    if "cbm_b200" in sys.modules:
        return sys.modules["cbm_b200"]
    pkg = os.path.join(ROOT, "cellbasedmodels.jl_b200")
    spec = importlib.util.spec_from_file_location(
        "cbm_b200", os.path.join(pkg, "__init__.py"), submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cbm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


class Desc:
    def __init__(self, n, community):
        self.n, self.community = n, community


class FakeBatch:
    """Host stand-in for the device batch: each step moves every agent of
    global community c by (c + 1) * 1e-3 along x, so a misrouted community
    shows up in the gathered state."""

    def __init__(self, cfg, descs):
        self.descs = descs
        self.state = [None] * len(descs)

    def upload(self, k, x, y, z, step=0):
        self.state[k] = dict(x=np.array(x, np.float64), y=np.array(y, np.float64),
                             z=np.array(z, np.float64), step=step)

    def step(self, n, flags=None):
        for k, s in enumerate(self.state):
            c = self.descs[k].community
            for _ in range(n):
                s["x"] = s["x"] + (c + 1) * 1e-3
            s["step"] += n

    def download(self, k):
        return dict(self.state[k])


def sizes_and_states(n_comm=13, seed=3):
    rng = np.random.default_rng(seed)
    sizes = [int(v) for v in rng.integers(5, 40, n_comm)]
    states = [dict(x=rng.uniform(0, 1, n), y=rng.uniform(0, 1, n), z=rng.uniform(0, 1, n))
              for n in sizes]
    return sizes, states


def run(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cbm = load_package()
        sizes, states = sizes_and_states()
        descs = [Desc(n, c) for c, n in enumerate(sizes)]
        sb = cbm.ShardedBatch(None, descs, rank=rank, world=world, factory=FakeBatch)
        for c, st in enumerate(states):
            sb.upload(c, st["x"], st["y"], st["z"])
        sb.step(7)
        got = sb.gather(dist)
        slowest = cbm.sweep.max_over_ranks(dist, 10.0 + rank)
        if rank == 0:
            np.save(os.path.join(out_dir, "gathered.npy"),
                    np.array([got[c]["x"] for c in range(len(sizes))], dtype=object),
                    allow_pickle=True)
            np.save(os.path.join(out_dir, "meta.npy"),
                    np.array([slowest, len(got)] + [got[c]["step"] for c in range(len(sizes))]))
        np.save(os.path.join(out_dir, f"mine{rank}.npy"), np.array(sb.mine))
    finally:
        dist.barrier()
        dist.destroy_process_group()


FIT_SEARCH = {"k_rep": [5.0, 10.0, 20.0], "sigma": [0.0, 0.1]}
FIT_DEFAULTS = dict(r_rep=2.0, k_att=1.0, r_att=3.0)


def fit_state(i, point):
    rng = np.random.default_rng(100 + i)
    n = 10 + 3 * i
    return dict(x=rng.uniform(0, 1, n), y=rng.uniform(0, 1, n), z=rng.uniform(0, 1, n))


def fit_loss(point, st):
    return float(np.mean(st["x"])) + point["sigma"]


def run_fit(rank, world, port, out_dir):
    """batched_grid_search sharded over two gloo ranks with the host batch."""
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cbm = load_package()
        rows = cbm.fitting.batched_grid_search(
            None, FIT_SEARCH, fit_state, fit_loss, 5, (0.0,) * 3, (1.0,) * 3, FIT_DEFAULTS,
            return_all=True, rank=rank, world=world, dist=dist, factory=FakeBatch)
        np.save(os.path.join(out_dir, f"fit{rank}.npy"),
                np.array([[r["k_rep"], r["sigma"], r["_score_"]] for r in rows]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


SWARM_SEARCH = {"k_rep": (5.0, 20.0), "sigma": (0.0, 0.1)}


def swarm_rows(rank=0, world=1, dist=None):
    """swarm_algorithm over the host batch; every rank runs the same driver
    with the same seed and scores its share of each generation."""
    cbm = load_package()
    ev = cbm.fitting.BatchedEvaluator(None, fit_state(0, None), fit_loss, 5, (0.0,) * 3,
                                      (1.0,) * 3, FIT_DEFAULTS, rank=rank, world=world,
                                      dist=dist, factory=FakeBatch)
    rows = cbm.fitting.swarm_algorithm(None, SWARM_SEARCH, population=6, stop_max_generations=3,
                                       rng=np.random.default_rng(2), evaluate_population=ev,
                                       return_all=True)
    return np.array([[r["k_rep"], r["sigma"], r["_score_"]] for r in rows])


def run_swarm(rank, world, port, out_dir):
    """The swarm driver with each generation partitioned over two gloo ranks."""
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        np.save(os.path.join(out_dir, f"swarm{rank}.npy"), swarm_rows(rank, world, dist))
    finally:
        dist.barrier()
        dist.destroy_process_group()
