# The stepping interface of CellBasedModels (src/CommunityStructure/step.jl)
# for the B200 platform: the stage functions, step! and evolve! with its save
# points (saveRAM! / saveJLD2, src/CommunityStructure/IO.jl:6-121).  The
# reference's functions take an untyped community and dispatch on its
# platform inside (typeof(platform) <: CPU / GPU), so these are methods of the
# same functions with the platform as a second argument; the reference's
# one-argument methods are untouched.

checkloaded(dev::B200) = dev.ctx == C_NULL && error(
    "Community must be loaded to platform with `loadToPlatform!` before being able to compute any step.")

"""agentStepRule! (step.jl:6-14): rule of the agents (walls, secretion, uptake, division, death)."""
agentStepRule!(com, dev::B200) = (checkloaded(dev); cbm_agent_step_rule(dev.ctx))
"""agentStepDE! (step.jl:48-56): neighbor forces and the agent integrator."""
agentStepDE!(com, dev::B200) = (checkloaded(dev); cbm_agent_step_de(dev.ctx))
"""mediumStepRule! (step.jl:34-42): gradient of the committed medium."""
mediumStepRule!(com, dev::B200) = (checkloaded(dev); cbm_medium_step_rule(dev.ctx))
"""mediumStepDE! (step.jl:76-84): FTCS step of the medium."""
mediumStepDE!(com, dev::B200) = (checkloaded(dev); cbm_medium_step_de(dev.ctx))
"""modelStepRule! / modelStepDE!: the model family has no model-scope variables."""
modelStepRule!(com, dev::B200) = checkloaded(dev)
modelStepDE!(com, dev::B200) = checkloaded(dev)
"""update! (update.jl:201-298): compaction, commit of the new values, N, t."""
update!(com, dev::B200) = (checkloaded(dev); cbm_update(dev.ctx))
"""computeNeighbors! (neighbors.jl): rebuild of the grid or of the Verlet list."""
computeNeighbors!(com, dev::B200) = (checkloaded(dev); cbm_compute_neighbors(dev.ctx))

"""
    step!(com, dev::B200)

One `step!` (step.jl:96-107): rule, DE, medium, update, neighbors, as one
replay of the context's CUDA graph.
"""
step!(com, dev::B200) = (checkloaded(dev); cbm_step(dev.ctx, 1))

"""
    evolve!(com, dev::B200; steps, saveEach=1, saveToFile=false, fileName=nothing,
            overwrite=false, saveCurrentState=false, preallocateAgents=0,
            progressMessage=(com)->nothing)

`evolve!` (step.jl:124-155) on the B200 platform, with the reference's
keywords.  Between save points the device runs `saveEach` steps as graph
replays with no host round trip; at each save point the committed state is
downloaded into the community's host arrays and saved by the reference's
own `saveRAM!` or `saveJLD2`.  The community is brought back at the end.
"""
function evolve!(com, dev::B200; steps, saveEach=1, saveToFile=false, fileName=nothing,
                 overwrite=false, saveCurrentState=false, preallocateAgents=0,
                 progressMessage=(com) -> nothing)
    if saveToFile && fileName === nothing
        error("Key argument fileName has to be specified with a valid name.")
    end
    loadToPlatform!(com, dev; preallocateAgents=preallocateAgents)
    save() = (download!(com, dev);
              saveToFile ? CellBasedModels.saveJLD2(fileName, com; overwrite=overwrite) :
                           CellBasedModels.saveRAM!(com))
    saveCurrentState && save()
    done = 0
    while done < steps
        chunk = min(saveEach - done % saveEach, steps - done)
        cbm_step(dev.ctx, chunk)
        done += chunk
        if done % saveEach == 0
            progressMessage(com)
            save()
        end
    end
    bringFromPlatform!(com, dev)
end
