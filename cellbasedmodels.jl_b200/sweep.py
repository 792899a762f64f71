"""Parameter sweeps over several GPUs: independent communities partitioned
across ranks (one process per GPU), with no data-path collective.

The reference's fitting drivers evaluate one whole simulation per parameter
set (src/fitting/gridSearch.jl:19-65, swarm.jl, genetic.jl); those runs are
independent, so a sweep shards by community.  Each rank advances its share in
one persistent launch (`Batch`), and the only exchanges are host-side: the
final gather of the states and the max over ranks of the device time.

Noise is keyed by the community's global index (`cbm_community_desc.community`),
so a community's trajectory does not depend on the rank that runs it or on
the number of ranks.
"""
import numpy as np


def partition_communities(sizes, world):
    """Longest-processing-time assignment of communities to `world` ranks by
    agent count.  Returns one sorted list of global community indices per
    rank; ties go to the lowest rank, so every rank computes the same answer
    without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda c: (-int(sizes[c]), c))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for c in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(c)
        load[r] += int(sizes[c])
    return [sorted(p) for p in parts]


def _default_factory(cfg, descs):
    from ._abi import Batch
    return Batch(cfg, descs)


class ShardedBatch:
    """The communities of this rank, advanced by one local batch.

    `descs` are the descriptors of ALL communities (ctypes `CbmCommunityDesc`
    or anything with `n`); `rank`/`world` choose this rank's share.  `factory`
    builds the local batch from (cfg, local descriptors) — the GPU `Batch` by
    default."""

    def __init__(self, cfg, descs, rank=0, world=1, factory=None):
        self.rank, self.world = int(rank), int(world)
        sizes = [int(d.n) for d in descs]
        self.parts = partition_communities(sizes, self.world)
        self.mine = self.parts[self.rank]
        self.local_of = {c: k for k, c in enumerate(self.mine)}
        self.n_agents = sum(sizes[c] for c in self.mine)
        self.batch = (factory or _default_factory)(cfg, [descs[c] for c in self.mine]) \
            if self.mine else None

    def owns(self, c):
        return c in self.local_of

    def upload(self, c, x, y, z, step=0):
        if self.owns(c):
            self.batch.upload(self.local_of[c], x, y, z, step=step)

    def step(self, n, flags=None):
        if self.batch is not None:
            if flags is None:
                self.batch.step(n)
            else:
                self.batch.step(n, flags)

    def download_local(self):
        """{global index: state} of this rank's communities."""
        if self.batch is None:
            return {}
        return {c: self.batch.download(k) for k, c in enumerate(self.mine)}

    def gather(self, dist=None, dst=0):
        """All communities' states on rank `dst` (None elsewhere).  Host-side
        gather over the process group (gloo or nccl object collectives)."""
        mine = self.download_local()
        if dist is None or self.world == 1:
            return mine
        box = [None] * self.world if self.rank == dst else None
        dist.gather_object(mine, box, dst=dst)
        if self.rank != dst:
            return None
        out = {}
        for part in box:
            out.update(part)
        return out


def max_over_ranks(dist, value):
    """Maximum of a float over the process group (host value; the device time
    of a rank is read from CUDA events before this call)."""
    if dist is None:
        return float(value)
    box = [None] * dist.get_world_size()
    dist.all_gather_object(box, float(value))
    return float(np.max(box))
