# Batched sweeps: many independent 3D soft-sphere communities (EM, CLVD,
# Float32) advanced by one persistent launch of the library (cbm_batch_*).
# This is the workload of the fitting drivers (src/fitting/gridSearch.jl,
# swarmAlgorithm.jl, geneticAlgorithm.jl, beeColonyAlgorithm.jl), which run
# one whole simulation per parameter set: a generation becomes one batch.

"""
    BatchPoint(; x, y, z, simBox, k, a, σ, r=1.0, r_att=3r)

One community of a batch: its initial positions, box and force/noise
parameters.
"""
Base.@kwdef struct BatchPoint
    x::Vector{Float32}
    y::Vector{Float32}
    z::Vector{Float32}
    simBox::Matrix{Float64}
    k::Float64
    a::Float64
    σ::Float64
    r::Float64 = 1.0
    r_att::Float64 = 3r
end

"""
    run_batch(points; dt, steps, seed=0, autotune=true, first_community=0)

Advances every `BatchPoint` by `steps` Euler-Maruyama steps in one launch and
returns the final positions of each, `(x, y, z)` tuples.  Community `c` of
the batch draws its noise as community `first_community + c` of the stream,
so that a community's trajectory is the one `evolve!` gives on the B200
platform with that community index.
"""
function run_batch(points::Vector{BatchPoint}; dt, steps, seed=0, autotune=true, first_community=0)
    base = CbmConfig(Int32(3), CBM_F32, Int64(1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), Float64(dt),
                     UInt64(seed), UInt32(0), CBM_NEIGH_CLVD, Int32(256), CBM_INT_EM, 3.3, 3.3, 0.15,
                     0.0, CBM_FORCE_DIRECT, CBM_ATT_FROM_REP, 10.0, 2.0, 1.0, 3.0, CBM_WALLS_NONE,
                     CBM_FATE_NONE, 0.0, 0.0, 0.0, Int32(0), Int32(0), 0.0, 0.0, 0.0,
                     (Int32(1), Int32(1), Int32(1)), CBM_MEDIUM_NEAREST, 0.0, 0.0, 0.0, 0.0, 0.0)
    descs = [CbmCommunityDesc(length(p.x), pad3(p.simBox[:, 1], 0.0), pad3(p.simBox[:, 2], 0.0),
                              p.k, 2p.r, p.a, p.r_att, p.σ, UInt32(first_community + i - 1), Int32(0))
             for (i, p) in enumerate(points)]
    b = cbm_batch_create(base, descs)
    try
        for (i, p) in enumerate(points)
            v = CbmStateView()
            v.N = length(p.x)
            v.capacity = length(p.x)
            v.pos = (pointer(p.x), pointer(p.y), pointer(p.z))
            GC.@preserve p cbm_batch_upload(b, i - 1, v)
        end
        autotune && cbm_batch_autotune(b)
        cbm_batch_step(b, steps)
        out = Vector{NTuple{3,Vector{Float32}}}(undef, length(points))
        for (i, p) in enumerate(points)
            n = length(p.x)
            x, y, z = zeros(Float32, n), zeros(Float32, n), zeros(Float32, n)
            v = CbmStateView()
            v.capacity = n
            v.pos = (pointer(x), pointer(y), pointer(z))
            GC.@preserve x y z cbm_batch_download(b, i - 1, v)
            out[i] = (x, y, z)
        end
        out
    finally
        cbm_batch_destroy(b)
    end
end

"""
    gridSearch_b200(points, loss; dt, steps, kwargs...)

`CBMFitting.gridSearch` (src/fitting/gridSearch.jl:19-65) with one batched
launch for all grid points: `loss(final_positions, point)` scores each
point, and the scores come back in the points' order.
"""
function gridSearch_b200(points::Vector{BatchPoint}, loss; dt, steps, kwargs...)
    finals = run_batch(points; dt=dt, steps=steps, kwargs...)
    [loss(f, p) for (f, p) in zip(finals, points)]
end
