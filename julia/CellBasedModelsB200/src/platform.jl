# The B200 platform: a device context per community, the model family it runs,
# and the exchange of the community's host arrays with the device
# (loadToPlatform! / bringFromPlatform!, communityStructure.jl:606-712).
#
# The reference compiles each model's Julia rule and DE texts into CPU or CUDA
# code (functionDE.jl:13-117).  A C ABI cannot run those closures, so the B200
# platform runs a fixed interaction family whose parameters describe the
# model: soft-sphere repulsion/adhesion, Euler or Euler-Maruyama, walls,
# growth with division and death, and an FTCS medium with secretion, uptake
# and chemotaxis.  The model texts each configuration corresponds to are
# listed in INTEGRATION.md.

"""
    SoftSpheres(; k, a, r, lagged=false, to_attraction=false)

Pair force `k(2r - d)` for `d < 2r`, then `-a(d - 2r)` up to the cutoff `3r`
(`to_attraction=true`: the `Aggregation.md` form with cutoff `r_att`);
`lagged=true` reads the committed force `fx` (`dt(x) = fx`).
"""
Base.@kwdef struct SoftSpheres
    k::Float64
    a::Float64
    r::Float64
    r_att::Float64 = 3r
    lagged::Bool = false
    to_attraction::Bool = false
end

"""`Growth(; vDiv, sep)`: `dt(v) = g`, division at `v >= vDiv` into daughters at `±sep`."""
Base.@kwdef struct Growth
    vDiv::Float64
    sep::Float64
end

"""
    Medium(; D, decay=0, secretion=0, uptake=0, chemotaxis=0, bilinear=false)

The medium variable `c` on the community's `NMedium` grid: FTCS
`dt(c) = D ∇²c - decay c` inside, frozen border; agents add
`w (secretion dt - uptake dt c)` at their stencil (nearest node, or the
multilinear stencil with `bilinear=true`) and drift by
`chemotaxis ∇c / (1 + |∇c|)`.
"""
Base.@kwdef struct Medium
    D::Float64
    decay::Float64 = 0.0
    secretion::Float64 = 0.0
    uptake::Float64 = 0.0
    chemotaxis::Float64 = 0.0
    bilinear::Bool = false
end

"""
    B200(; precision=Float32, force, sigma=0, growth=nothing, pDeath=0, walls=:none,
         wallForce=0, wallRange=0, drift=0, medium=nothing, seed=0, rebuildThreshold=0)

The B200 platform of one community.  `force` (a `SoftSpheres`), `sigma` (EM
noise amplitude), `growth`, `pDeath`, `walls` (`:none`, `:reflect`, `:push`),
`drift` (`dt(x) += -drift x`) and `medium` describe the model; the neighbor
algorithm and the integrator are taken from the `ABM` (`neighborsAlg`,
`agentAlg`).  `seed` keys the counter-based random stream of the library.
"""
mutable struct B200 <: CellBasedModels.Platform
    precision::DataType
    force::SoftSpheres
    sigma::Float64
    growth::Union{Nothing,Growth}
    pDeath::Float64
    walls::Symbol
    wallForce::Float64
    wallRange::Float64
    drift::Float64
    medium::Union{Nothing,Medium}
    seed::UInt64
    rebuildThreshold::Float64
    ctx::Ptr{Cvoid}
    nMax::Int
end

function B200(; precision=Float32, force, sigma=0.0, growth=nothing, pDeath=0.0, walls=:none,
              wallForce=0.0, wallRange=0.0, drift=0.0, medium=nothing, seed=0,
              rebuildThreshold=0.0)
    precision in (Float32, Float64) || error("B200 runs Float32 or Float64")
    walls in (:none, :reflect, :push) || error("walls must be :none, :reflect or :push")
    B200(precision, force, Float64(sigma), growth, Float64(pDeath), walls, Float64(wallForce),
         Float64(wallRange), Float64(drift), medium, UInt64(seed), Float64(rebuildThreshold),
         C_NULL, 0)
end

# CellBasedModels calls these at load and after each CPU/GPU step; the B200
# platform keeps its launch shapes inside the library.
CellBasedModels.platformSetup!(::B200, com) = nothing
CellBasedModels.platformUpdate!(::B200, com) = nothing

neighbor_code(n) =
    n isa CellBasedModels.CBMNeighbors.Full ? CBM_NEIGH_FULL :
    n isa CellBasedModels.CBMNeighbors.CellLinked ? CBM_NEIGH_CELL_LINKED :
    n isa CellBasedModels.CBMNeighbors.VerletDisplacement ? CBM_NEIGH_VERLET_DISPLACEMENT :
    n isa CellBasedModels.CBMNeighbors.CLVD ? CBM_NEIGH_CLVD :
    error("B200: neighbor algorithm $(typeof(n)) is not supported")

integrator_code(a) =
    a isa CellBasedModels.CBMIntegrators.Euler ? CBM_INT_EULER :
    a isa CellBasedModels.CBMIntegrators.EM ? CBM_INT_EM :
    a isa CellBasedModels.CBMIntegrators.Heun ? CBM_INT_HEUN :
    a isa CellBasedModels.CBMIntegrators.RungeKutta4 ? CBM_INT_RK4 :
    a isa CellBasedModels.CBMIntegrators.EulerHeun ? CBM_INT_EULER_HEUN :
    error("B200: integrator $(typeof(a)) is not supported")

pad3(v, fill) = ntuple(d -> d <= length(v) ? v[d] : fill, 3)

"""
    cbm_config_from(com, dev; n_max)

The `cbm_config` of a community: dimensions, simBox, dt and NMedium from the
`Community`, neighbor algorithm and integrator from its `ABM`, the model
parameters from the platform `dev`.
"""
function cbm_config_from(com, dev::B200; n_max::Integer)
    abm = com.abm
    dims = abm.dims
    nb = abm.neighbors
    code = neighbor_code(nb)
    cell_edge = hasproperty(nb, :cellEdge) ? Float64(nb.cellEdge) : 1.0
    skin = hasproperty(nb, :skin) ? Float64(nb.skin) : 1.0
    nmaxn = hasproperty(nb, :nMaxNeighbors) ? Int32(nb.nMaxNeighbors) : Int32(32)
    box = Array{Float64}(com.simBox)
    f = dev.force
    m = dev.medium
    nm = m === nothing ? (1, 1, 1) : pad3(Int32.(collect(com.NMedium)), Int32(1))
    CbmConfig(Int32(dims), dev.precision == Float64 ? CBM_F64 : CBM_F32, Int64(n_max),
              pad3(box[:, 1], 0.0), pad3(box[:, 2], 0.0), Float64(com.dt),
              dev.seed, UInt32(0), code, nmaxn,
              integrator_code(abm.agentAlg), cell_edge, skin, dev.rebuildThreshold,
              dev.sigma, f.lagged ? CBM_FORCE_LAGGED : CBM_FORCE_DIRECT,
              f.to_attraction ? CBM_ATT_TO_ATT : CBM_ATT_FROM_REP,
              f.k, 2f.r, f.a, f.r_att,
              dev.walls === :reflect ? CBM_WALLS_REFLECT : dev.walls === :push ? CBM_WALLS_PUSH : CBM_WALLS_NONE,
              dev.growth === nothing && dev.pDeath == 0 ? CBM_FATE_NONE : CBM_FATE_VOLUME,
              dev.wallForce, dev.wallRange, dev.drift,
              Int32(dev.growth === nothing ? 0 : 1), Int32(m === nothing ? 0 : 1),
              dev.growth === nothing ? 0.0 : dev.growth.vDiv,
              dev.growth === nothing ? 0.0 : dev.growth.sep, dev.pDeath,
              NTuple{3,Int32}(nm),
              m === nothing || !m.bilinear ? CBM_MEDIUM_NEAREST : CBM_MEDIUM_BILINEAR,
              m === nothing ? 0.0 : m.D, m === nothing ? 0.0 : m.decay,
              m === nothing ? 0.0 : m.secretion, m === nothing ? 0.0 : m.chemotaxis,
              m === nothing ? 0.0 : m.uptake)
end

"""
    HostState

The community's agent and medium arrays on the host, in the platform's
precision, with room for `capacity` agents: what `cbm_upload` reads and
`cbm_download` writes.  Keys follow the model: `:x, :y, :z`, `:v, :g`
(growth), `:fx, :fy, :fz` (lagged force), `:parent`, `:c, :gx, :gy, :gz`
(medium).
"""
struct HostState
    arrays::Dict{Symbol,Array}
    id::Vector{Int64}
    parent::Vector{Int64}
end

agent_symbols(dims) = (:x, :y, :z)[1:dims]

function HostState(com, dev::B200, capacity::Integer)
    T = dev.precision
    dims = com.abm.dims
    N = com.N
    arrays = Dict{Symbol,Array}()
    for s in agent_symbols(dims)
        a = zeros(T, capacity)
        a[1:N] .= getproperty(com, s)[1:N]
        arrays[s] = a
    end
    if dev.growth !== nothing
        for s in (:v, :g)
            a = zeros(T, capacity)
            a[1:N] .= getproperty(com, s)[1:N]
            arrays[s] = a
        end
    end
    if dev.force.lagged
        for s in (:fx, :fy, :fz)[1:dims]
            arrays[s] = zeros(T, capacity)
        end
    end
    if dev.medium !== nothing
        n = prod(com.NMedium)
        arrays[:c] = Array{T}(reshape(getproperty(com, :c), :))
        for s in (:gx, :gy, :gz)[1:dims]
            arrays[s] = zeros(T, n)
        end
    end
    id = zeros(Int64, capacity)
    id[1:N] .= Array{Int64}(com.id)[1:N]
    parent = zeros(Int64, capacity)
    if hasproperty(com, :parent)
        parent[1:N] .= getproperty(com, :parent)[1:N]
    end
    HostState(arrays, id, parent)
end

ptr_or_null(d, s) = haskey(d, s) ? Ptr{Cvoid}(pointer(d[s])) : C_NULL

"""The `cbm_state_view` of a host state (keep `h` alive while the view is used)."""
function state_view(h::HostState; N, t=0.0, step=0, id_max=0)
    a = h.arrays
    v = CbmStateView()
    v.N = N
    v.capacity = length(h.id)
    v.t = t
    v.step = step
    v.id_max = id_max
    v.pos = (ptr_or_null(a, :x), ptr_or_null(a, :y), ptr_or_null(a, :z))
    v.v = ptr_or_null(a, :v)
    v.g = ptr_or_null(a, :g)
    v.f = (ptr_or_null(a, :fx), ptr_or_null(a, :fy), ptr_or_null(a, :fz))
    v.id = pointer(h.id)
    v.parent = pointer(h.parent)
    v.medium_c = ptr_or_null(a, :c)
    v.medium_grad = (ptr_or_null(a, :gx), ptr_or_null(a, :gy), ptr_or_null(a, :gz))
    v
end

"""
    loadToPlatform!(com, dev::B200; preallocateAgents=0)

`loadToPlatform!` (communityStructure.jl:606-654) for the B200 platform:
creates the device context with capacity `N + preallocateAgents`, uploads
the community, and builds the neighbor structure (the reference's first
`computeNeighbors!`).  The host arrays stay the community's own.
"""
function loadToPlatform!(com, dev::B200; preallocateAgents::Integer=0)
    dev.ctx == C_NULL || error("B200: this platform already holds a loaded community")
    n_max = com.N + preallocateAgents
    cfg = cbm_config_from(com, dev; n_max=n_max)
    dev.ctx = cbm_create(cfg)
    dev.nMax = n_max
    h = HostState(com, dev, max(com.N, 1))
    idmax = com.N == 0 ? 0 : maximum(Array{Int64}(com.id)[1:com.N])
    GC.@preserve h cbm_upload(dev.ctx, state_view(h; N=com.N, t=Float64(com.t), id_max=idmax))
    setfield!(com, :loaded, true)
    nothing
end

"""
    download!(com, dev::B200)

Copies the committed device state into the community's host arrays and sets
`N`, `t` and `id`: the data half of `bringFromPlatform!`, used at every save
point.
"""
function download!(com, dev::B200)
    h = HostState(com.abm.dims, dev, dev.nMax, com)
    v = state_view(h; N=0)
    GC.@preserve h cbm_download(dev.ctx, v, CBM_VIEW_COMMITTED)
    N = Int(v.N)
    for (s, a) in h.arrays
        if s in (:c, :gx, :gy, :gz)
            dst = com.parameters[s]
            copyto!(dst, reshape(a, size(dst)))
        else
            com.parameters[s] = Array{eltype(com.parameters[s])}(a[1:N])
        end
    end
    if haskey(com.parameters, :parent)
        com.parameters[:parent] = h.parent[1:N]
    end
    setfield!(com, :N, N)
    setfield!(com, :t, v.t)
    setfield!(com, :id, h.id[1:N])
    nothing
end

# a host state with room for `capacity` agents, for downloads
function HostState(dims::Integer, dev::B200, capacity::Integer, com)
    T = dev.precision
    arrays = Dict{Symbol,Array}()
    for s in agent_symbols(dims)
        arrays[s] = zeros(T, capacity)
    end
    if dev.growth !== nothing
        arrays[:v] = zeros(T, capacity)
        arrays[:g] = zeros(T, capacity)
    end
    if dev.force.lagged
        for s in (:fx, :fy, :fz)[1:dims]
            arrays[s] = zeros(T, capacity)
        end
    end
    if dev.medium !== nothing
        n = prod(com.NMedium)
        arrays[:c] = zeros(T, n)
        for s in (:gx, :gy, :gz)[1:dims]
            arrays[s] = zeros(T, n)
        end
    end
    HostState(arrays, zeros(Int64, capacity), zeros(Int64, capacity))
end

"""
    bringFromPlatform!(com, dev::B200)

`bringFromPlatform!` (communityStructure.jl:663-712) for the B200 platform:
downloads the committed state into the community and releases the device
context.
"""
function bringFromPlatform!(com, dev::B200)
    dev.ctx == C_NULL && error("B200: no community is loaded on this platform")
    download!(com, dev)
    cbm_destroy(dev.ctx)
    dev.ctx = C_NULL
    setfield!(com, :loaded, false)
    nothing
end
