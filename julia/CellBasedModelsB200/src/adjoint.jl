# Gradients of a trajectory loss through the hand-written adjoint of the
# library (cbm_adjoint_*): the soft-sphere Euler ODE in 3D, Float64, with
# θ = (k, a, 2r).  `trajectory_loss` is the forward map followed by the mean
# squared error against a target; its ChainRulesCore `rrule` returns the loss
# and a pullback built from one checkpointed reverse sweep.

"""
    AdjointProblem(; dt, simBox, cellEdge, r_att)

The fixed part of the differentiable problem: time step, simBox (3x2),
CellLinked cell edge and the interaction cutoff, which the derivative holds
fixed (pairs crossing the cutoff are a measure-zero event at which the loss
is not differentiable).
"""
Base.@kwdef struct AdjointProblem
    dt::Float64
    simBox::Matrix{Float64}
    cellEdge::Float64
    r_att::Float64
end

function adjoint_config(p::AdjointProblem, θ, n)
    k, a, ρ = θ
    box = p.simBox
    CbmConfig(Int32(3), CBM_F64, Int64(n), pad3(box[:, 1], 0.0), pad3(box[:, 2], 0.0), p.dt,
              UInt64(0), UInt32(0), CBM_NEIGH_CELL_LINKED, Int32(32), CBM_INT_EULER,
              max(p.cellEdge, p.r_att), 1.0, 0.0, 0.0, CBM_FORCE_DIRECT, CBM_ATT_FROM_REP,
              Float64(k), Float64(ρ), Float64(a), p.r_att, CBM_WALLS_NONE, CBM_FATE_NONE, 0.0, 0.0,
              0.0, Int32(0), Int32(0), 0.0, 0.0, 0.0, (Int32(1), Int32(1), Int32(1)),
              CBM_MEDIUM_NEAREST, 0.0, 0.0, 0.0, 0.0, 0.0)
end

function with_adjoint(f, p::AdjointProblem, θ, n)
    a = cbm_adjoint_create(adjoint_config(p, θ, n))
    try
        f(a)
    finally
        cbm_adjoint_destroy(a)
    end
end

"""
    trajectory_loss(θ, x0, target; problem, steps, K=20)

`mean((x_T - target)^2)` over the three coordinates of every agent, with
`x_T` the positions after `steps` Euler steps from `x0` (a tuple of three
vectors) under θ = (k, a, 2r).
"""
function trajectory_loss(θ, x0::NTuple{3,Vector{Float64}}, target::NTuple{3,Vector{Float64}};
                         problem::AdjointProblem, steps::Integer, K::Integer=20)
    n = length(x0[1])
    xT = with_adjoint(a -> cbm_adjoint_forward(a, x0, steps), problem, θ, n)
    sum(sum(abs2, xT[d] .- target[d]) for d in 1:3) / (3n)
end

function ChainRulesCore.rrule(::typeof(trajectory_loss), θ, x0::NTuple{3,Vector{Float64}},
                              target::NTuple{3,Vector{Float64}};
                              problem::AdjointProblem, steps::Integer, K::Integer=20)
    n = length(x0[1])
    res = with_adjoint(a -> cbm_adjoint_run(a, x0, target, steps, K), problem, θ, n)
    function trajectory_loss_pullback(ȳ)
        dθ = ȳ .* res.dθ
        dx0 = map(g -> ȳ .* g, res.dx0)
        (NoTangent(), dθ, dx0, NoTangent())
    end
    res.loss, trajectory_loss_pullback
end
