"""cbm_b200 — the B200 platform for CellBasedModels.jl's per-step path.

Python mirror of the reference's user interface for this path, on top of the
C ABI in include/cbm_b200.h (libcbm_b200.so):

    abm = ABM(3, force=SoftSpheres(k=10, a=1, r=1),
              neighborsAlg=CBMNeighbors.CLVD(skin=3.3, nMaxNeighbors=64, cellEdge=3.3),
              agentAlg=CBMIntegrators.EM(), sigma=0.05,
              growth=Growth(vDiv=2.0, sep=0.5), pDeath=1e-4, platform=B200("f32"))
    com = Community(abm, N=10_000, dt=0.005, simBox=[[0, 400]] * 3, x=..., y=..., z=..., v=..., g=...)
    evolve(com, steps=100, saveEach=10, preallocateAgents=990_000)

Names follow src/CellBasedModels.jl: ABM (src/AgentStructure/agentStructure.jl:90),
Community (src/CommunityStructure/communityStructure.jl:71), evolve!/step!
(src/CommunityStructure/step.jl:96-155), loadToPlatform!/bringFromPlatform!
(communityStructure.jl:606-712), CBMNeighbors (src/neighbors.jl),
CBMIntegrators (src/integrators.jl).  The model family is fixed (soft-sphere
repulsion/adhesion, walls, growth/division/death, FTCS medium with secretion
and chemotaxis); the reference's free-form Julia rule text is not accepted.
There is no CPU fallback: without the built library or a CUDA device every
call raises.
"""
from types import SimpleNamespace

import numpy as np

from . import _abi, fitting, sweep  # noqa: F401
from ._abi import (Adjoint, Batch, CbmConfig, CbmError, Context, DGADIMedium,  # noqa: F401
                   Rods2D, load_library, make_config, make_medium_config, make_rods_config)
from .sweep import ShardedBatch, partition_communities  # noqa: F401

__all__ = ["ABM", "Community", "evolve", "step", "loadToPlatform", "bringFromPlatform",
           "agentStepRule", "agentStepDE", "mediumStepRule", "mediumStepDE", "update",
           "computeNeighbors", "CBMNeighbors", "CBMIntegrators", "SoftSpheres", "Growth",
           "Medium", "B200", "Context", "Batch", "Adjoint", "ShardedBatch",
           "partition_communities", "CbmError", "make_config", "load_library",
           "DGADIMedium", "make_medium_config", "Rods2D", "make_rods_config", "fitting"]


# ---- algorithm descriptors (src/neighbors.jl, src/integrators.jl) -------------
class _Neighbors:
    Full = staticmethod(lambda: dict(neighbors=_abi.NEIGH_FULL))
    CellLinked = staticmethod(lambda cellEdge: dict(neighbors=_abi.NEIGH_CELL_LINKED,
                                                    cell_edge=float(cellEdge)))
    VerletDisplacement = staticmethod(
        lambda skin, nMaxNeighbors, rebuildThreshold=0.0: dict(
            neighbors=_abi.NEIGH_VERLET_DISPLACEMENT, skin=float(skin),
            n_max_neighbors=int(nMaxNeighbors), rebuild_threshold=float(rebuildThreshold)))
    CLVD = staticmethod(
        lambda skin, nMaxNeighbors, cellEdge, rebuildThreshold=0.0: dict(
            neighbors=_abi.NEIGH_CLVD, skin=float(skin), n_max_neighbors=int(nMaxNeighbors),
            cell_edge=float(cellEdge), rebuild_threshold=float(rebuildThreshold)))


class _Integrators:
    Euler = staticmethod(lambda: dict(integrator=_abi.INT_EULER))
    EM = staticmethod(lambda: dict(integrator=_abi.INT_EM))
    # ODE integrators with 2 and 4 evaluations of f per step (integrators.jl:516-668)
    Heun = staticmethod(lambda: dict(integrator=_abi.INT_HEUN))
    RungeKutta4 = staticmethod(lambda: dict(integrator=_abi.INT_RK4))
    # SDE integrator with 2 evaluations of f per step (integrators.jl:744-814)
    EulerHeun = staticmethod(lambda: dict(integrator=_abi.INT_EULER_HEUN))


CBMNeighbors = _Neighbors()
CBMIntegrators = _Integrators()


def SoftSpheres(k, a, r, lagged=False):
    """F = k(2r-d) for d<2r, -a(d-2r) for 2r<=d<3r (force_mode DIRECT unless lagged)."""
    return dict(k_rep=float(k), r_rep=2.0 * r, k_att=float(a), r_att=3.0 * r,
                att_form=_abi.ATT_FROM_REP,
                force_mode=_abi.FORCE_LAGGED if lagged else _abi.FORCE_DIRECT)


def Growth(vDiv, sep):
    return dict(growth=1, fate=_abi.FATE_VOLUME, v_div=float(vDiv), div_sep=float(sep))


def Medium(NMedium, D, decay=0.0, secretion=0.0, chemotaxis=0.0, bilinear=False):
    return dict(medium=1, n_medium=tuple(int(n) for n in NMedium), diff_D=float(D),
                decay=float(decay), secretion=float(secretion), chemotaxis=float(chemotaxis),
                medium_sampling=_abi.MEDIUM_BILINEAR if bilinear else _abi.MEDIUM_NEAREST)


def B200(precision="f32"):
    return dict(precision=_abi.F64 if precision in ("f64", "float64", 64) else _abi.F32)


class ABM:
    """The model: dimensions, the interaction family and its algorithms."""

    def __init__(self, dims, force=None, neighborsAlg=None, agentAlg=None, sigma=0.0,
                 growth=None, pDeath=0.0, medium=None, walls=None, platform=None, seed=0,
                 **extra):
        self.dims = int(dims)
        cfg = dict(dims=self.dims)
        for part in (force, neighborsAlg, agentAlg, growth, medium, walls, platform or B200()):
            if part:
                cfg.update(part)
        if pDeath:
            cfg["p_death"] = float(pDeath)
            cfg.setdefault("fate", _abi.FATE_VOLUME)
        cfg["sigma"] = float(sigma)
        cfg["seed"] = int(seed)
        cfg.update(extra)
        self.cfg = cfg


class Community:
    """Agents, medium and time of one simulation (communityStructure.jl:71-186)."""

    def __init__(self, abm, N, dt, simBox, t=0.0, **fields):
        self.abm = abm
        self.N = int(N)
        self.dt = float(dt)
        self.t = float(t)
        self.simBox = np.asarray(simBox, dtype=np.float64).reshape(abm.dims, 2)
        self.fields = {k: np.asarray(v) for k, v in fields.items()}
        self.step_count = 0
        self.id_max = self.N
        self.pastTimes = []
        self._ctx = None

    def __getattr__(self, k):
        f = self.__dict__.get("fields", {})
        if k in f:
            return f[k]
        raise AttributeError(k)

    @property
    def loaded(self):
        return self._ctx is not None


def loadToPlatform(com, preallocateAgents=0):
    """loadToPlatform! (communityStructure.jl:606-654)."""
    if com._ctx is not None:
        return
    kw = dict(com.abm.cfg)
    kw.update(n_max=com.N + int(preallocateAgents), dt=com.dt,
              box_lo=tuple(com.simBox[:, 0]), box_hi=tuple(com.simBox[:, 1]))
    cfg = make_config(**kw)
    ctx = Context(cfg)
    state = dict(com.fields)
    state["N"] = com.N
    ctx.upload(state, t=com.t, step=com.step_count, id_max=com.id_max)
    com._ctx = ctx


def bringFromPlatform(com):
    """bringFromPlatform! (communityStructure.jl:663-712)."""
    if com._ctx is None:
        return
    s = com._ctx.download()
    _absorb(com, s)
    com._ctx.close()
    com._ctx = None


def _absorb(com, s):
    com.N, com.t, com.step_count, com.id_max = s["N"], s["t"], s["step"], s["id_max"]
    keep = ("x", "y", "z")[: com.abm.dims] + ("id", "parent")
    cfg = com.abm.cfg
    if cfg.get("growth"):
        keep += ("v", "g")
    if cfg.get("force_mode") == _abi.FORCE_LAGGED:
        keep += ("fx", "fy", "fz")[: com.abm.dims]
    if cfg.get("medium"):
        keep += ("c",) + ("gx", "gy", "gz")[: com.abm.dims]
    com.fields = {k: s[k] for k in keep if k in s}


def _need(com):
    if com._ctx is None:
        raise RuntimeError("Community must be loaded to platform with loadToPlatform before "
                           "being able to compute any step.")
    return com._ctx


def agentStepRule(com):
    _need(com).stage("agent_rule")


def agentStepDE(com):
    _need(com).stage("agent_de")


def mediumStepRule(com):
    _need(com).stage("medium_rule")


def mediumStepDE(com):
    _need(com).stage("medium_de")


def update(com):
    _need(com).stage("update")


def computeNeighbors(com):
    _need(com).stage("neighbors")


def step(com, n=1):
    """step! (step.jl:96-107), n times, as graph replays."""
    _need(com).step(n, _abi.SYNC)


def saveRAM(com):
    """saveRAM! (IO.jl:6-33): snapshot of the committed state."""
    s = _need(com).download()
    snap = SimpleNamespace(N=s["N"], t=s["t"], **{k: v for k, v in s.items()
                                                  if isinstance(v, np.ndarray)})
    com.pastTimes.append(snap)
    return snap


def evolve(com, steps, saveEach=1, preallocateAgents=0, saveCurrentState=False,
           progressMessage=None):
    """evolve! (step.jl:124-155)."""
    loadToPlatform(com, preallocateAgents=preallocateAgents)
    if saveCurrentState:
        saveRAM(com)
    done = 0
    while done < steps:
        n = min(saveEach, steps - done)
        step(com, n)
        done += n
        if done % saveEach == 0:
            if progressMessage:
                progressMessage(com)
            saveRAM(com)
    bringFromPlatform(com)
