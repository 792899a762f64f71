# CBMModels.rods2D and rods2dGrowth (src/models/rods.jl:61-163) on a rods
# context of the library (cbm_rods_*): the contact force rodForces
# (rods.jl:21-59) over CBMMetrics.rodIntersection (src/metrics.jl:137-246),
# with fx, fy, W and pressure assigned inside the ODE and read lagged, as the
# reference's code generator has them.  Neighbors are CellLinked or Full.

const ROD_SYMBOLS = (:x, :y, :vx, :vy, :theta, :ω, :d, :l, :m, :fx, :fy, :W, :pressure, :lTarget)

"""
    rods_config(com; precision=Float64, seed=0)

The `cbm_rods_config` of a rods2D / rods2dGrowth community: model parameters
from the community's fields, neighbors from its ABM.
"""
function rods_config(com; precision=Float64, seed=0)
    nb = com.abm.neighbors
    full = nb isa CellBasedModels.CBMNeighbors.Full
    growth = hasproperty(com, :lTarget)
    box = Array{Float64}(com.simBox)
    CbmRodsConfig(precision == Float64 ? CBM_F64 : CBM_F32,
                  full ? CBM_NEIGH_FULL : CBM_NEIGH_CELL_LINKED, Int64(com.nMax_ === nothing ? com.N : com.nMax_),
                  (box[1, 1], box[2, 1]), (box[1, 2], box[2, 2]),
                  full ? 0.0 : Float64(nb.cellEdge), Float64(com.dt),
                  com.kn[1], com.γn[1], com.γt[1], com.μcc[1], com.μcw[1], com.β[1], com.βω[1],
                  Int32(growth ? 1 : 0), Int32(0),
                  growth ? com.growth[1] : 0.0, growth ? com.α[1] : 0.0,
                  growth ? com.σlTarget[1] : 0.0, growth ? com.lMax[1] : 0.0, UInt64(seed))
end

"""
    evolve_rods!(com; steps, preallocateAgents=0, precision=Float64, seed=0)

`steps` Euler steps of a rods2D / rods2dGrowth community on the device,
with the community's arrays updated at the end (growth changes N).
"""
function evolve_rods!(com; steps, preallocateAgents=0, precision=Float64, seed=0)
    N = com.N
    cap = N + preallocateAgents
    cfg = rods_config(com; precision=precision, seed=seed)
    cfg = CbmRodsConfig(cfg.precision, cfg.neighbors, Int64(cap), cfg.box_lo, cfg.box_hi,
                        cfg.cell_edge, cfg.dt, cfg.kn, cfg.gamma_n, cfg.gamma_t, cfg.mu_cc,
                        cfg.mu_cw, cfg.beta, cfg.beta_w, cfg.growth_model, cfg.pad0, cfg.growth,
                        cfg.alpha, cfg.sigma_l_target, cfg.l_max, cfg.seed)
    r = cbm_rods_create(cfg)
    try
        cols = [hasproperty(com, s) ? Array{precision}(vcat(getproperty(com, s)[1:N],
                                                             zeros(precision, cap - N))) :
                                      nothing for s in ROD_SYMBOLS]
        ptrs = Ptr{Cvoid}[c === nothing ? C_NULL : pointer(c) for c in cols]
        ptrs[13] = C_NULL  # pressure is read by download only
        GC.@preserve cols cbm_rods_upload(r, N, ptrs)
        cbm_rods_step(r, steps)
        ptrs = Ptr{Cvoid}[c === nothing ? C_NULL : pointer(c) for c in cols]
        n = GC.@preserve cols cbm_rods_download(r, ptrs)
        for (s, c) in zip(ROD_SYMBOLS, cols)
            c === nothing || (com.parameters[s] = c[1:n])
        end
        setfield!(com, :N, Int(n))
        n
    finally
        cbm_rods_destroy(r)
    end
end
