# The C ABI of libcbm_b200 (include/cbm_b200.h): constants, mirrors of the C
# structures (field order and sizes exactly those of the header), and one
# `ccall` wrapper per entry point.  Host arrays passed to a call are borrowed
# for the duration of that call only: every caller keeps them alive with
# `GC.@preserve`.  Indices returned by the grid and neighbor queries are
# 0-based.

"""Path of the shared library; `ENV["CBM_B200_LIB"]` overrides the in-tree build."""
const LIBCBM = get(ENV, "CBM_B200_LIB",
                   joinpath(@__DIR__, "..", "..", "..", "cellbasedmodels.jl_b200", "libcbm_b200.so"))

# ---- status codes ------------------------------------------------------------
const CBM_OK = Int32(0)
const CBM_ERR_ARG = Int32(1)
const CBM_ERR_CUDA = Int32(2)
const CBM_ERR_AGENT_OVERFLOW = Int32(3)
const CBM_ERR_NEIGHBOR_OVERFLOW = Int32(4)
const CBM_ERR_TIMEOUT = Int32(5)
const CBM_ERR_STATE = Int32(6)
const CBM_ERR_NOMEM = Int32(7)

# ---- enumerations --------------------------------------------------------------
const CBM_F32 = Int32(0)
const CBM_F64 = Int32(1)
const CBM_NEIGH_NONE = Int32(0)
const CBM_NEIGH_FULL = Int32(1)
const CBM_NEIGH_CELL_LINKED = Int32(2)
const CBM_NEIGH_VERLET_DISPLACEMENT = Int32(3)
const CBM_NEIGH_CLVD = Int32(4)
const CBM_INT_EULER = Int32(0)
const CBM_INT_EM = Int32(1)
const CBM_INT_HEUN = Int32(2)
const CBM_INT_RK4 = Int32(3)
const CBM_INT_EULER_HEUN = Int32(4)
const CBM_FORCE_DIRECT = Int32(0)
const CBM_FORCE_LAGGED = Int32(1)
const CBM_ATT_FROM_REP = Int32(0)
const CBM_ATT_TO_ATT = Int32(1)
const CBM_WALLS_NONE = Int32(0)
const CBM_WALLS_REFLECT = Int32(1)
const CBM_WALLS_PUSH = Int32(2)
const CBM_FATE_NONE = Int32(0)
const CBM_FATE_VOLUME = Int32(1)
const CBM_FATE_ID_PARITY = Int32(2)
const CBM_MEDIUM_NEAREST = Int32(0)
const CBM_MEDIUM_BILINEAR = Int32(1)
const CBM_SYNC = Int32(1)
const CBM_NO_GRAPH = Int32(2)
const CBM_VIEW_COMMITTED = Int32(0)
const CBM_VIEW_NEW = Int32(1)
const CBM_MEDIUM_MAX_FIELDS = 8
const CBM_RODS_FIELDS = 14
const CBM_NOALLOC_MAX_AGENTS = 524288
const CBM_NOALLOC_MAX_CELLS = 1048576

# ---- structures ------------------------------------------------------------------
"""Mirror of `cbm_config`: the model family and its parameters (ABM + Community)."""
struct CbmConfig
    dims::Int32; precision::Int32; n_max::Int64
    box_lo::NTuple{3,Float64}; box_hi::NTuple{3,Float64}; dt::Float64
    seed::UInt64; community::UInt32; neighbors::Int32; n_max_neighbors::Int32
    integrator::Int32; cell_edge::Float64; skin::Float64; rebuild_threshold::Float64
    sigma::Float64; force_mode::Int32; att_form::Int32
    k_rep::Float64; r_rep::Float64; k_att::Float64; r_att::Float64
    walls::Int32; fate::Int32; wall_force::Float64; wall_range::Float64
    drift_linear::Float64; growth::Int32; medium::Int32; v_div::Float64
    div_sep::Float64; p_death::Float64; n_medium::NTuple{3,Int32}
    medium_sampling::Int32; diff_D::Float64; decay::Float64; secretion::Float64
    chemotaxis::Float64; uptake::Float64
end

"""Mirror of `cbm_state_view`: pointers to host arrays of one community state."""
mutable struct CbmStateView
    N::Int64; capacity::Int64; t::Float64; step::Int64; id_max::Int64
    pos::NTuple{3,Ptr{Cvoid}}; v::Ptr{Cvoid}; g::Ptr{Cvoid}
    f::NTuple{3,Ptr{Cvoid}}; id::Ptr{Int64}; parent::Ptr{Int64}
    medium_c::Ptr{Cvoid}; medium_grad::NTuple{3,Ptr{Cvoid}}
end

CbmStateView() = CbmStateView(0, 0, 0.0, 0, 0, (C_NULL, C_NULL, C_NULL), C_NULL, C_NULL,
                              (C_NULL, C_NULL, C_NULL), Ptr{Int64}(C_NULL), Ptr{Int64}(C_NULL),
                              C_NULL, (C_NULL, C_NULL, C_NULL))

"""Mirror of `cbm_community_desc`: one community of a batched sweep."""
struct CbmCommunityDesc
    n::Int64; box_lo::NTuple{3,Float64}; box_hi::NTuple{3,Float64}
    k_rep::Float64; r_rep::Float64; k_att::Float64; r_att::Float64; sigma::Float64
    community::UInt32; pad::Int32
end

"""Mirror of `cbm_batch_tuning`."""
struct CbmBatchTuning
    threads::Int32; ctas_per_sm::Int32; skin::Float64; rebuild_threshold::Float64
    tile_agents::Int32; lanes_per_agent::Int32
end

"""Mirror of `cbm_medium_config` (the implicit DGADI medium)."""
struct CbmMediumConfig
    dims::Int32; precision::Int32; n::NTuple{3,Int32}; n_fields::Int32
    box_lo::NTuple{3,Float64}; box_hi::NTuple{3,Float64}; dt::Float64
    diffusion::NTuple{8,Float64}; decay::NTuple{8,Float64}; c_max::Float64
end

"""Mirror of `cbm_rods_config` (rods2D / rods2dGrowth)."""
struct CbmRodsConfig
    precision::Int32; neighbors::Int32; n_max::Int64
    box_lo::NTuple{2,Float64}; box_hi::NTuple{2,Float64}; cell_edge::Float64; dt::Float64
    kn::Float64; gamma_n::Float64; gamma_t::Float64; mu_cc::Float64; mu_cw::Float64
    beta::Float64; beta_w::Float64
    growth_model::Int32; pad0::Int32
    growth::Float64; alpha::Float64; sigma_l_target::Float64; l_max::Float64; seed::UInt64
end

# ---- errors ------------------------------------------------------------------------
"""A non-zero status of a libcbm_b200 call, with the library's message."""
struct CbmError <: Exception
    code::Int32
    msg::String
end
Base.showerror(io::IO, e::CbmError) = print(io, "libcbm_b200 status ", e.code, ": ", e.msg)

cbm_version() = unsafe_string(ccall((:cbm_version, LIBCBM), Cstring, ()))
cbm_last_error(ctx) = unsafe_string(ccall((:cbm_last_error, LIBCBM), Cstring, (Ptr{Cvoid},), ctx))
check(rc, ctx) = rc == CBM_OK ? nothing : throw(CbmError(rc, cbm_last_error(ctx)))

# ---- one community: lifetime, exchange, stepping --------------------------------------
function cbm_create(cfg::CbmConfig)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:cbm_create, LIBCBM), Cint, (Ref{Ptr{Cvoid}}, Ref{CbmConfig}), out, cfg)
    check(rc, C_NULL)
    out[]
end
cbm_destroy(ctx) = ccall((:cbm_destroy, LIBCBM), Cvoid, (Ptr{Cvoid},), ctx)
cbm_upload(ctx, v::CbmStateView) =
    check(ccall((:cbm_upload, LIBCBM), Cint, (Ptr{Cvoid}, Ref{CbmStateView}), ctx, v), ctx)
cbm_download(ctx, v::CbmStateView, which=CBM_VIEW_COMMITTED) =
    check(ccall((:cbm_download, LIBCBM), Cint, (Ptr{Cvoid}, Ref{CbmStateView}, Int32), ctx, v, which), ctx)
cbm_step(ctx, n, flags=CBM_SYNC) =
    check(ccall((:cbm_step, LIBCBM), Cint, (Ptr{Cvoid}, Int32, Int32), ctx, n, flags), ctx)
# parity runs: noise increments given by the caller, `dims x N` column-major (i*dims + d)
cbm_step_noise(ctx, ξ::Matrix, flags=CBM_SYNC) =
    GC.@preserve ξ check(ccall((:cbm_step_noise, LIBCBM), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Int32),
                               ctx, ξ, flags), ctx)
cbm_agent_step_rule(ctx) = check(ccall((:cbm_agent_step_rule, LIBCBM), Cint, (Ptr{Cvoid},), ctx), ctx)
cbm_agent_step_de(ctx) = check(ccall((:cbm_agent_step_de, LIBCBM), Cint, (Ptr{Cvoid},), ctx), ctx)
cbm_medium_step_rule(ctx) = check(ccall((:cbm_medium_step_rule, LIBCBM), Cint, (Ptr{Cvoid},), ctx), ctx)
cbm_medium_step_de(ctx) = check(ccall((:cbm_medium_step_de, LIBCBM), Cint, (Ptr{Cvoid},), ctx), ctx)
cbm_update(ctx) = check(ccall((:cbm_update, LIBCBM), Cint, (Ptr{Cvoid},), ctx), ctx)
cbm_compute_neighbors(ctx) = check(ccall((:cbm_compute_neighbors, LIBCBM), Cint, (Ptr{Cvoid},), ctx), ctx)
cbm_sync(ctx) = check(ccall((:cbm_sync, LIBCBM), Cint, (Ptr{Cvoid},), ctx), ctx)

function cbm_get_counters(ctx)
    N, a, r, m, s = Ref{Int64}(0), Ref{Int64}(0), Ref{Int64}(0), Ref{Int64}(0), Ref{Int64}(0)
    fl = Ref{Int32}(0)
    check(ccall((:cbm_get_counters, LIBCBM), Cint,
                (Ptr{Cvoid}, Ref{Int64}, Ref{Int64}, Ref{Int64}, Ref{Int64}, Ref{Int32}, Ref{Int64}),
                ctx, N, a, r, m, fl, s), ctx)
    (N=N[], NAdd=a[], NRemove=r[], idMax=m[], flagRecomputeNeighbors=fl[], step=s[])
end
function cbm_grid_shape(ctx)
    n3 = zeros(Int32, 3)
    check(ccall((:cbm_grid_shape, LIBCBM), Cint, (Ptr{Cvoid}, Ptr{Int32}), ctx, n3), ctx)
    Tuple(n3)
end
cbm_get_grid(ctx, agent_cell, cell_start, cell_count, cell_agents) =
    check(ccall((:cbm_get_grid, LIBCBM), Cint,
                (Ptr{Cvoid}, Ptr{Int32}, Ptr{Int32}, Ptr{Int32}, Ptr{Int32}),
                ctx, agent_cell, cell_start, cell_count, cell_agents), ctx)
cbm_get_neighbors(ctx, counts::Vector{Int32}, list::Vector{Int32}) =
    check(ccall((:cbm_get_neighbors, LIBCBM), Cint, (Ptr{Cvoid}, Ptr{Int32}, Ptr{Int32}, Int64),
                ctx, counts, list, length(list)), ctx)
cbm_count_neighbors(ctx, radius, out::Vector{Int32}) =
    check(ccall((:cbm_count_neighbors, LIBCBM), Cint, (Ptr{Cvoid}, Float64, Ptr{Int32}),
                ctx, radius, out), ctx)
cbm_rng_fill(ctx, kind, a, b, out::Vector, step=0) =
    check(ccall((:cbm_rng_fill, LIBCBM), Cint, (Ptr{Cvoid}, Int32, Float64, Float64, Int64, Int64, Ptr{Cvoid}),
                ctx, kind, a, b, length(out), step, out), ctx)
cbm_stream(ctx) = ccall((:cbm_stream, LIBCBM), Ptr{Cvoid}, (Ptr{Cvoid},), ctx)
cbm_kernels_per_step(ctx) = ccall((:cbm_kernels_per_step, LIBCBM), Cint, (Ptr{Cvoid},), ctx)
function cbm_profile_step(ctx, max_kernels=32)
    ms = zeros(Float32, max_kernels)
    names = fill(Ptr{UInt8}(C_NULL), max_kernels)
    n = Ref{Int32}(0)
    check(ccall((:cbm_profile_step, LIBCBM), Cint, (Ptr{Cvoid}, Int32, Ptr{Float32}, Ptr{Ptr{UInt8}}, Ref{Int32}),
                ctx, max_kernels, ms, names, n), ctx)
    [(unsafe_string(names[k]), ms[k]) for k in 1:n[]]
end

"""Kernel timing inside the step graphs on (true) or off; graphs are captured again."""
cbm_set_kernel_timing(ctx, on::Bool) =
    check(ccall((:cbm_set_kernel_timing, LIBCBM), Cint, (Ptr{Cvoid}, Int32), ctx, on ? 1 : 0), ctx)
"""Durations (ms) and names of the kernels of the last graph-replayed step."""
function cbm_kernel_times(ctx, max_kernels=32)
    ms = zeros(Float32, max_kernels)
    names = fill(Ptr{UInt8}(C_NULL), max_kernels)
    n = Ref{Int32}(0)
    check(ccall((:cbm_kernel_times, LIBCBM), Cint, (Ptr{Cvoid}, Int32, Ptr{Float32}, Ptr{Ptr{UInt8}}, Ref{Int32}),
                ctx, max_kernels, ms, names, n), ctx)
    [(unsafe_string(names[k]), ms[k]) for k in 1:min(n[], max_kernels)]
end

# ---- batched communities ------------------------------------------------------------
cbm_batch_last_error(b) = unsafe_string(ccall((:cbm_batch_last_error, LIBCBM), Cstring, (Ptr{Cvoid},), b))
bcheck(rc, b) = rc == CBM_OK ? nothing : throw(CbmError(rc, cbm_batch_last_error(b)))
function cbm_batch_create(base::CbmConfig, descs::Vector{CbmCommunityDesc})
    out = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:cbm_batch_create, LIBCBM), Cint,
               (Ref{Ptr{Cvoid}}, Ref{CbmConfig}, Int32, Ptr{CbmCommunityDesc}),
               out, base, length(descs), descs)
    bcheck(rc, C_NULL)
    out[]
end
cbm_batch_destroy(b) = ccall((:cbm_batch_destroy, LIBCBM), Cvoid, (Ptr{Cvoid},), b)
cbm_batch_upload(b, c, v::CbmStateView) =
    bcheck(ccall((:cbm_batch_upload, LIBCBM), Cint, (Ptr{Cvoid}, Int32, Ref{CbmStateView}), b, c, v), b)
cbm_batch_download(b, c, v::CbmStateView) =
    bcheck(ccall((:cbm_batch_download, LIBCBM), Cint, (Ptr{Cvoid}, Int32, Ref{CbmStateView}), b, c, v), b)
cbm_batch_step(b, n, flags=CBM_SYNC) =
    bcheck(ccall((:cbm_batch_step, LIBCBM), Cint, (Ptr{Cvoid}, Int32, Int32), b, n, flags), b)
cbm_batch_set_tuning(b, t::CbmBatchTuning) =
    bcheck(ccall((:cbm_batch_set_tuning, LIBCBM), Cint, (Ptr{Cvoid}, Ref{CbmBatchTuning}), b, t), b)
function cbm_batch_get_tuning(b)
    t = Ref{CbmBatchTuning}(CbmBatchTuning(0, 0, 0.0, 0.0, 0, 0))
    bcheck(ccall((:cbm_batch_get_tuning, LIBCBM), Cint, (Ptr{Cvoid}, Ref{CbmBatchTuning}), b, t), b)
    t[]
end
function cbm_batch_autotune(b, trial_steps=20)
    t = Ref{CbmBatchTuning}(CbmBatchTuning(0, 0, 0.0, 0.0, 0, 0))
    bcheck(ccall((:cbm_batch_autotune, LIBCBM), Cint, (Ptr{Cvoid}, Int32, Ref{CbmBatchTuning}),
                 b, trial_steps, t), b)
    t[]
end
cbm_batch_stream(b) = ccall((:cbm_batch_stream, LIBCBM), Ptr{Cvoid}, (Ptr{Cvoid},), b)

# ---- adjoint -------------------------------------------------------------------------
cbm_adjoint_last_error(a) = unsafe_string(ccall((:cbm_adjoint_last_error, LIBCBM), Cstring, (Ptr{Cvoid},), a))
acheck(rc, a) = rc == CBM_OK ? nothing : throw(CbmError(rc, cbm_adjoint_last_error(a)))
function cbm_adjoint_create(cfg::CbmConfig)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:cbm_adjoint_create, LIBCBM), Cint, (Ref{Ptr{Cvoid}}, Ref{CbmConfig}), out, cfg)
    acheck(rc, C_NULL)
    out[]
end
cbm_adjoint_destroy(a) = ccall((:cbm_adjoint_destroy, LIBCBM), Cvoid, (Ptr{Cvoid},), a)
function cbm_adjoint_forward(a, x0::NTuple{3,Vector{Float64}}, steps)
    n = length(x0[1])
    xT = ntuple(_ -> zeros(Float64, n), 3)
    px = Ptr{Cvoid}[pointer(v) for v in x0]
    pT = Ptr{Cvoid}[pointer(v) for v in xT]
    GC.@preserve x0 xT px pT acheck(ccall((:cbm_adjoint_forward, LIBCBM), Cint,
        (Ptr{Cvoid}, Int64, Ptr{Ptr{Cvoid}}, Int32, Ptr{Ptr{Cvoid}}), a, n, px, steps, pT), a)
    xT
end
function cbm_adjoint_run(a, x0::NTuple{3,Vector{Float64}}, target::NTuple{3,Vector{Float64}}, steps,
                         checkpoint_every)
    n = length(x0[1])
    loss = Ref{Float64}(0.0)
    dθ = zeros(Float64, 3)
    dx0 = ntuple(_ -> zeros(Float64, n), 3)
    px = Ptr{Cvoid}[pointer(v) for v in x0]
    pt = Ptr{Cvoid}[pointer(v) for v in target]
    pd = Ptr{Cvoid}[pointer(v) for v in dx0]
    GC.@preserve x0 target dx0 px pt pd acheck(ccall((:cbm_adjoint_run, LIBCBM), Cint,
        (Ptr{Cvoid}, Int64, Ptr{Ptr{Cvoid}}, Int32, Int32, Ptr{Ptr{Cvoid}}, Ref{Float64},
         Ptr{Float64}, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}),
        a, n, px, steps, checkpoint_every, pt, loss, dθ, pd, C_NULL), a)
    (loss=loss[], dθ=dθ, dx0=dx0)
end
cbm_adjoint_stream(a) = ccall((:cbm_adjoint_stream, LIBCBM), Ptr{Cvoid}, (Ptr{Cvoid},), a)

# ---- implicit medium (DGADI) ------------------------------------------------------------
cbm_medium_last_error(m) = unsafe_string(ccall((:cbm_medium_last_error, LIBCBM), Cstring, (Ptr{Cvoid},), m))
mcheck(rc, m) = rc == CBM_OK ? nothing : throw(CbmError(rc, cbm_medium_last_error(m)))
function cbm_medium_create(cfg::CbmMediumConfig)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:cbm_medium_create, LIBCBM), Cint, (Ref{Ptr{Cvoid}}, Ref{CbmMediumConfig}), out, cfg)
    mcheck(rc, C_NULL)
    out[]
end
cbm_medium_destroy(m) = ccall((:cbm_medium_destroy, LIBCBM), Cvoid, (Ptr{Cvoid},), m)
# fields: Array{T}(undef, NX, NY, NZ, n_fields) (x fastest, then the field index)
cbm_medium_upload(m, fields::Array, source) =
    GC.@preserve fields source mcheck(ccall((:cbm_medium_upload, LIBCBM), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}), m, fields, source === nothing ? C_NULL : pointer(source)), m)
cbm_medium_step(m, n, flags=CBM_SYNC) =
    mcheck(ccall((:cbm_medium_step, LIBCBM), Cint, (Ptr{Cvoid}, Int32, Int32), m, n, flags), m)
function cbm_medium_download!(m, fields::Array)
    t = Ref{Float64}(0.0)
    GC.@preserve fields mcheck(ccall((:cbm_medium_download, LIBCBM), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ref{Float64}), m, fields, t), m)
    t[]
end
cbm_medium_stream(m) = ccall((:cbm_medium_stream, LIBCBM), Ptr{Cvoid}, (Ptr{Cvoid},), m)

# ---- rods2D / rods2dGrowth --------------------------------------------------------------
cbm_rods_last_error(r) = unsafe_string(ccall((:cbm_rods_last_error, LIBCBM), Cstring, (Ptr{Cvoid},), r))
rcheck(rc, r) = rc == CBM_OK ? nothing : throw(CbmError(rc, cbm_rods_last_error(r)))
function cbm_rods_create(cfg::CbmRodsConfig)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:cbm_rods_create, LIBCBM), Cint, (Ref{Ptr{Cvoid}}, Ref{CbmRodsConfig}), out, cfg)
    rcheck(rc, C_NULL)
    out[]
end
cbm_rods_destroy(r) = ccall((:cbm_rods_destroy, LIBCBM), Cvoid, (Ptr{Cvoid},), r)
cbm_rods_upload(r, n, ptrs::Vector{Ptr{Cvoid}}) =
    rcheck(ccall((:cbm_rods_upload, LIBCBM), Cint, (Ptr{Cvoid}, Int64, Ptr{Ptr{Cvoid}}), r, n, ptrs), r)
cbm_rods_step(r, n, flags=CBM_SYNC) =
    rcheck(ccall((:cbm_rods_step, LIBCBM), Cint, (Ptr{Cvoid}, Int32, Int32), r, n, flags), r)
function cbm_rods_download(r, ptrs::Vector{Ptr{Cvoid}})
    n = Ref{Int64}(0)
    rcheck(ccall((:cbm_rods_download, LIBCBM), Cint, (Ptr{Cvoid}, Ptr{Ptr{Cvoid}}, Ref{Int64}), r, ptrs, n), r)
    n[]
end
cbm_rods_stream(r) = ccall((:cbm_rods_stream, LIBCBM), Ptr{Cvoid}, (Ptr{Cvoid},), r)

# ---- allocation-free cell grid ------------------------------------------------------------
cbm_noalloc_last_error() = unsafe_string(ccall((:cbm_noalloc_last_error, LIBCBM), Cstring, ()))
"""
    cbm_cell_grid_noalloc(x, y, z, n, dims, precision, lo, hi, edge, agent_cell, cell_start, cell_agents, stream)

The CellLinked grid of `n` device-resident positions without any device
allocation (pointers from CUDA.jl arrays, for a process whose CUDA.jl pool
owns the GPU or while a stream is captured).  Its scratch is a static device
array of the library: at most `CBM_NOALLOC_MAX_AGENTS` agents and
`CBM_NOALLOC_MAX_CELLS` cells, and calls that overlap on one GPU race.
"""
cbm_cell_grid_noalloc(x, y, z, n, dims, precision, lo::NTuple{3,Float64}, hi::NTuple{3,Float64},
                      edge, agent_cell, cell_start, cell_agents, stream) =
    ccall((:cbm_cell_grid_noalloc, LIBCBM), Cint,
          (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Int32, Int32, Int32, Ref{NTuple{3,Float64}},
           Ref{NTuple{3,Float64}}, Float64, Ptr{Int32}, Ptr{Int32}, Ptr{Int32}, Ptr{Cvoid}),
          x, y, z, n, dims, precision, lo, hi, edge, agent_cell, cell_start, cell_agents, stream)
"""Status of the last `cbm_cell_grid_noalloc` on this device (waits for `stream`)."""
cbm_noalloc_status(stream) = ccall((:cbm_noalloc_status, LIBCBM), Cint, (Ptr{Cvoid},), stream)
