# The implicit medium: CBMIntegrators.DGADI (src/integrators.jl:817-937) on a
# medium context of the library (cbm_medium_*).  The model is fixed:
# dt(c_k) = s (c_max - c_k) - λ_k c_k inside (@mediumInside), with s a static
# source field (the mediumODE of examples/Implementation.ipynb with λ = 0).
# As in the reference, the explicit part is added without a factor dt, every
# axis uses the last axis's r = dt / (dims dx^2), and the border keeps its
# initial values.

"""
    DGADIMedium(; NMedium, simBox, dt, D, decay=zeros, c_max=0, precision=Float32)

A device medium of `length(D)` fields (at most 8) on `NMedium` nodes.
"""
mutable struct DGADIMedium
    h::Ptr{Cvoid}
    n::NTuple{3,Int32}
    n_fields::Int
    precision::DataType
end

function DGADIMedium(; NMedium, simBox, dt, D, decay=zeros(length(D)), c_max=0.0, precision=Float32)
    dims = length(NMedium)
    nf = length(D)
    1 <= nf <= CBM_MEDIUM_MAX_FIELDS || error("DGADI: 1 to $CBM_MEDIUM_MAX_FIELDS fields")
    box = Array{Float64}(simBox)
    n = pad3(Int32.(collect(NMedium)), Int32(1))
    cfg = CbmMediumConfig(Int32(dims), precision == Float64 ? CBM_F64 : CBM_F32, NTuple{3,Int32}(n),
                          Int32(nf), pad3(box[:, 1], 0.0), pad3(box[:, 2], 0.0), Float64(dt),
                          ntuple(k -> k <= nf ? Float64(D[k]) : 0.0, 8),
                          ntuple(k -> k <= nf ? Float64(decay[k]) : 0.0, 8), Float64(c_max))
    DGADIMedium(cbm_medium_create(cfg), NTuple{3,Int32}(n), nf, precision)
end

"""
    upload!(m, u, source=nothing)

`u`: the reference's medium array `(nVars, NX, NY, NZ)`; the library keeps
fields one after another, x fastest, so it is permuted on the way in.
"""
function upload!(m::DGADIMedium, u::AbstractArray, source=nothing)
    dims = ndims(u) - 1
    fields = Array{m.precision}(permutedims(u, (2:(dims + 1)..., 1)))
    src = source === nothing ? nothing : Array{m.precision}(source)
    cbm_medium_upload(m.h, fields, src)
end

"""`step!(m, n)`: n DGADI steps on the device."""
step!(m::DGADIMedium, n::Integer=1) = cbm_medium_step(m.h, n)

"""`download_fields(m, dims)`: the fields as the reference's `(nVars, NX, NY, NZ)` array, and t."""
function download_fields(m::DGADIMedium, dims::Integer)
    fields = zeros(m.precision, m.n[1:dims]..., m.n_fields)
    t = cbm_medium_download!(m.h, fields)
    permutedims(fields, (dims + 1, 1:dims...)), t
end

close!(m::DGADIMedium) = (m.h == C_NULL || cbm_medium_destroy(m.h); m.h = C_NULL; nothing)
