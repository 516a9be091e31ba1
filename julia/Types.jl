# Types.jl (drop-in for src/Types.jl, 2D) -- Config, FieldState, Operators,
# Step1Cache and BDFCoeff with the reference's names and fields, over libvsav.
#
# Include this set instead of the reference's (scripts/Main.jl:42-52 picks the
# implementation by its include list):
#     for f in ("Types.jl", "SpectralUtils.jl", "Utils.jl", "Init.jl", "Solvers.jl", "simulation.jl")
#         include(joinpath(<repo>/julia, f))
#     end
# Differences from the reference, all deliberate:
#   * Operators holds the device handle (and the host k-tables), not FFTW plans
#     and scratch arrays;
#   * the device holds the time levels: FieldState objects are host mirrors
#     (upload_state! / download_state!, vsav_core.jl);
#   * Step1Cache and the step results are lazy device views.

include(joinpath(@__DIR__, "vsav_core.jl"))

# ---- 1. Config (src/Types.jl:27-134) -------------------------------------------

struct Config
    N::Int
    epsilon::Float64
    M_phi::Float64
    M0_psi::Float64
    eta::Float64
    gamma_surf::Float64
    gamma_area::Int
    gamma_bend::Float64
    gamma_in::Int
    beta_in::Int
    psi_in_v::Vector{Float64}
    gamma_out::Int
    beta_out::Int
    psi_out_v::Vector{Float64}
    lamda::Int
    S1::Float64
    S2::Float64
    S3::Float64
    S4::Float64
    C1::Float64
    C2::Float64
    C3::Float64
    dt::Float64
    T::Float64
    Nt::Int
    Nx::Int
    Ny::Int
    Lx::Float64
    Ly::Float64
    dx::Float64
    dy::Float64
    tol::Float64
    goal::Symbol
    spe_len::Int
end

"""Keyword constructor; derives Nt = round(T/dt), dx = Lx/Nx, dy = Ly/Ny and
the half-spectrum length (Nx÷2+1)·Ny·N as the reference does."""
function Config(; N, epsilon, M_phi, M0_psi, eta, gamma_surf, gamma_area, gamma_bend,
                gamma_in, beta_in, psi_in_v::Vector{Float64}, gamma_out, beta_out, psi_out_v::Vector{Float64},
                lamda, S1, S2, S3, S4, C1, C2, C3, dt, T, Nx, Ny, Lx, Ly, tol, goal)
    return Config(N, epsilon, M_phi, M0_psi, eta, gamma_surf, gamma_area, gamma_bend,
                  gamma_in, beta_in, psi_in_v, gamma_out, beta_out, psi_out_v, lamda,
                  S1, S2, S3, S4, C1, C2, C3, dt, T, round(Int, T / dt),
                  Nx, Ny, Lx, Ly, Lx / Nx, Ly / Ny, tol, goal, (Nx ÷ 2 + 1) * Ny * N)
end
Base.broadcastable(c::Config) = Ref(c)

# ---- 2. FieldState (src/Types.jl:167-265): the host mirror of one time level ----

mutable struct FieldState
    phi::Array{Float64, 3}         # Nx × Ny × N
    phi_hat::Array{ComplexF64, 3}  # (Nx÷2+1) × Ny × N
    psi::Array{Float64, 3}
    psi_hat::Array{ComplexF64, 3}
    u::Array{Float64, 3}           # Nx × Ny × 2
    u_hat::Array{ComplexF64, 3}
    p::Matrix{Float64}             # Nx × Ny
    p_hat::Matrix{ComplexF64}
    mu::Array{Float64, 3}
    mu_hat::Array{ComplexF64, 3}
    nu::Array{Float64, 3}
    nu_hat::Array{ComplexF64, 3}
    Q::Float64
    R1::Float64
    R2::Float64
    R3::Float64
    A0::Vector{Float64}
    dt::Float64
end

function FieldState(Nx::Int, Ny::Int, N::Int)
    Nk = Nx ÷ 2 + 1
    r(k) = zeros(Float64, Nx, Ny, k)
    c(k) = zeros(ComplexF64, Nk, Ny, k)
    return FieldState(r(N), c(N), r(N), c(N), r(2), c(2), zeros(Nx, Ny), zeros(ComplexF64, Nk, Ny),
                      r(N), c(N), r(N), c(N), 0.0, 0.0, 0.0, 0.0, [0.0], 0.0)
end
empty_state(conf::Config) = FieldState(conf.Nx, conf.Ny, conf.N)

"""Deep copy of every host array and scalar of `src` into `dest` (the
reference's update_state!).  The device levels advance with advance_state!."""
function update_state!(dest::FieldState, src::FieldState)
    for name in STATE_ARRAYS
        copyto!(getfield(dest, name), getfield(src, name))
    end
    dest.Q, dest.R1, dest.R2, dest.R3 = src.Q, src.R1, src.R2, src.R3
    dest.A0 = copy(src.A0)
    dest.dt = src.dt
    return dest
end

# ---- 3. Operators (src/Types.jl:298-342) ----------------------------------------

mutable struct Operators
    h::Ptr{Cvoid}                  # libvsav handle: plans, buffers and both time levels
    ndim::Int
    Nx::Int
    Ny::Int
    Nz::Int
    N::Int
    K::NTuple{2, Matrix{Float64}}
    D1::NTuple{2, Matrix{ComplexF64}}
    D1_full::NTuple{2, Matrix{ComplexF64}}
    Laplacian::Matrix{Float64}
    Laplacian_full::Matrix{Float64}
    Biharmonic::Matrix{Float64}
    gen::Int                       # bumped whenever the device state changes
end

# ---- Step1Cache (src/Types.jl:358-385): 16 device views ---------------------------

struct Step1Cache
    ops::Any
    views::Any                     # NamedTuple of the 16 fields, or nothing before the first Step 1
end
Step1Cache(Nx::Int, Ny::Int, N::Int) = Step1Cache(nothing, nothing)
function Base.getproperty(c::Step1Cache, s::Symbol)
    s in (:ops, :views) && return getfield(c, s)
    v = getfield(c, :views)
    v === nothing && error("Step1Cache is empty until solve_step1 has run")
    return getproperty(v, s)
end

# ---- 4. BDFCoeff (src/Types.jl:407-426) ------------------------------------------

struct BDFCoeff
    a::Float64
    b::Float64
    c::Float64
end
BDFCoeff(::Val{1}) = BDFCoeff(1.0, -1.0, 0.0)
BDFCoeff(::Val{2}) = BDFCoeff(1.5, -2.0, 0.5)
bdf_coeff(n::Int) = n == 1 ? BDFCoeff(Val(1)) : BDFCoeff(Val(2))
