"""
    CellBasedModelsB200

The B200 platform of CellBasedModels.jl: the per-step hot path (cell grid and
Verlet lists, the pairwise ODE/SDE step, division and death with compaction,
the explicit medium) runs on one NVIDIA B200 through the C ABI of
`libcbm_b200` (include/cbm_b200.h).  The ABM / Community definitions stay the
reference's; a community is evolved with

    dev = B200(precision=Float32, force=SoftSpheres(k=10, a=1, r=1), sigma=0.05,
               growth=Growth(vDiv=2, sep=0.5), pDeath=1e-4)
    evolve!(com, dev; steps=1000, saveEach=100, preallocateAgents=10^6)

(a method of the reference's own `evolve!`) with its keywords and save points (`saveRAM!`,
`saveJLD2`).  Also: batched sweeps for the fitting drivers (`run_batch`,
`gridSearch_b200`), trajectory gradients through a ChainRulesCore `rrule`
(`trajectory_loss`), the implicit DGADI medium (`DGADIMedium`), the rod
models (`evolve_rods!`) and the allocation-free grid for callers that must
not allocate (`cbm_cell_grid_noalloc`).
"""
module CellBasedModelsB200

using CellBasedModels
using ChainRulesCore
# The stepping API gains methods whose second argument is the B200 platform;
# the reference's one-argument methods are untouched.
import CellBasedModels: loadToPlatform!, bringFromPlatform!, step!, evolve!, agentStepRule!,
                        agentStepDE!, mediumStepRule!, mediumStepDE!, modelStepRule!,
                        modelStepDE!, update!, computeNeighbors!

export B200, SoftSpheres, Growth, Medium, CbmError
export BatchPoint, run_batch, gridSearch_b200
export AdjointProblem, trajectory_loss
export DGADIMedium, evolve_rods!

include("abi.jl")
include("platform.jl")
include("stepping.jl")
include("batch.jl")
include("adjoint.jl")
include("medium.jl")
include("rods.jl")

end
