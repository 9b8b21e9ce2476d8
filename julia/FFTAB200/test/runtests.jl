# Parity of the GPU plans with FFTA's own CPU transforms on the same inputs
# (the configurations' shapes at test sizes), plus FFTA's error behaviour.
# Needs a CUDA device and FFTA.jl in the test environment.
using Test, Random, LinearAlgebra
using AbstractFFTs
using CUDA
import FFTA
using FFTAB200

relerr(a, b) = norm(a - b) / max(norm(b), floatmin(real(eltype(b))))
tol(T, n) = 4 * eps(real(T)) * max(1.0, log2(n))

@testset "FFTAB200" begin
    if !CUDA.functional()
        @info "no CUDA device: the GPU parity tests are skipped"
        @test_skip false
    else
        Random.seed!(1)
        @testset "1D N=$N $T" for (N, T) in ((1024, ComplexF64), (4096, ComplexF32),
                                             (19683, ComplexF32), (27648, ComplexF64),
                                             (1009, ComplexF32), (1000, ComplexF64))
            x = randn(T, N, 8)
            for (gpu, cpu) in ((plan_fft, FFTA.plan_fft), (plan_bfft, FFTA.plan_bfft))
                p = gpu(CuArray(x), 1)
                y = Array(p * CuArray(x))
                ref = cpu(x, 1) * x
                @test relerr(y, ref) <= tol(T, N)
            end
        end
        @testset "2D $sz" for sz in ((1000, 1000), (2187, 2048))
            X = randn(ComplexF32, sz...)
            y = Array(plan_fft(CuArray(X), 1:2) * CuArray(X))
            @test relerr(y, FFTA.fft(X)) <= tol(ComplexF32, prod(sz))
        end
        @testset "real" begin
            x = randn(Float32, 4096, 16)
            y = Array(plan_rfft(CuArray(x), 1) * CuArray(x))
            @test relerr(y, FFTA.rfft(x, 1)) <= tol(Float32, 4096)
        end
        @testset "errors (test/argument_checking.jl)" begin
            x = CuArray(randn(ComplexF32, 8, 4))
            p = plan_fft(x, 1)
            @test_throws DimensionMismatch mul!(similar(x, 8, 5), p, x)
            @test_throws DimensionMismatch p * CuArray(randn(ComplexF32, 9, 4))
            @test_throws DomainError size(p, 0)
            @test_throws ArgumentError plan_fft(CuArray(randn(ComplexF16, 8)), 1)
        end
    end
end
