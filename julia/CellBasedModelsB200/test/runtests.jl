# Checks for a machine with Julia, CellBasedModels.jl and a B200: the B200
# platform against the reference's own CPU platform on the 2D aggregation
# model (Float64, CellLinked, reflecting walls, Euler), and the binding of
# every entry point.  The repository's Python tests drive the same C ABI
# through ctypes on machines without Julia.
using Test
using CellBasedModels
using CellBasedModelsB200

@testset "library" begin
    @test startswith(CellBasedModelsB200.cbm_version(), "cbm_b200")
end

@testset "2D aggregation against the CPU platform" begin
    r, k, a = 1.0, 10.0, 1.0
    model = ABM(2,
        agent = Dict(),
        agentODE = quote
            @loopOverNeighbors i2 begin
                d = CBMMetrics.euclidean(x, x[i2], y, y[i2])
                if d < 2 * $r
                    F = $k * (2 * $r - d)
                elseif d < 3 * $r
                    F = -($a * (d - 2 * $r))
                else
                    F = 0.0
                end
                if d < 3 * $r
                    s = F / d
                    dt(x) += s * (x - x[i2]); dt(y) += s * (y - y[i2])
                end
            end
        end,
        agentRule = quote
            if x < 0.0; x = -x elseif x > 100.0; x = 200.0 - x end
            if y < 0.0; y = -y elseif y > 100.0; y = 200.0 - y end
        end,
        neighborsAlg = CBMNeighbors.CellLinked(cellEdge=3.0),
        agentAlg = CBMIntegrators.Euler(),
        platform = CPU())
    N = 4096
    x0, y0 = 100 .* rand(N), 100 .* rand(N)
    ref = Community(model, N=N, dt=0.01, simBox=[0 100; 0 100.0], x=copy(x0), y=copy(y0))
    evolve!(ref, steps=100)
    com = Community(model, N=N, dt=0.01, simBox=[0 100; 0 100.0], x=copy(x0), y=copy(y0))
    dev = B200(precision=Float64, force=SoftSpheres(k=k, a=a, r=r), walls=:reflect)
    evolve!(com, dev; steps=100)
    @test com.x ≈ ref.x rtol=1e-10
    @test com.y ≈ ref.y rtol=1e-10
end
