# Types_3d.jl (drop-in for src/Types_3d.jl, 3D) -- Config, FieldState, Operators,
# Step1Cache and BDFCoeff with the reference's names and fields, over libvsav.
#
# Include this set instead of the reference's (scripts/Main.jl:42-52 picks the
# implementation by its include list):
#     for f in ("Types_3d.jl", "SpectralUtils_3d.jl", "Utils_3d.jl", "Init_3d.jl", "Solvers_3d.jl",
#               "simulation.jl")
#         include(joinpath(<repo>/julia, f))
#     end
# Differences from the reference, all deliberate:
#   * Operators holds the device handle (and the host k-tables), not FFTW plans
#     and scratch arrays;
#   * the device holds the time levels: FieldState objects are host mirrors
#     (upload_state! / download_state!, vsav_core.jl);
#   * Step1Cache and the step results are lazy device views.

include(joinpath(@__DIR__, "vsav_core.jl"))

# ---- 1. Config (src/Types_3d.jl:27-140) -------------------------------------------

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
    Nz::Int
    Lx::Float64
    Ly::Float64
    Lz::Float64
    dx::Float64
    dy::Float64
    dz::Float64
    tol::Float64
    goal::Symbol
    spe_len::Int
end

"""Keyword constructor; derives Nt = round(T/dt), dx, dy, dz and the
half-spectrum length (Nx÷2+1)·Ny·Nz·N as the reference does."""
function Config(; N, epsilon, M_phi, M0_psi, eta, gamma_surf, gamma_area, gamma_bend,
                gamma_in, beta_in, psi_in_v::Vector{Float64}, gamma_out, beta_out, psi_out_v::Vector{Float64},
                lamda, S1, S2, S3, S4, C1, C2, C3, dt, T, Nx, Ny, Nz, Lx, Ly, Lz, tol, goal)
    return Config(N, epsilon, M_phi, M0_psi, eta, gamma_surf, gamma_area, gamma_bend,
                  gamma_in, beta_in, psi_in_v, gamma_out, beta_out, psi_out_v, lamda,
                  S1, S2, S3, S4, C1, C2, C3, dt, T, round(Int, T / dt),
                  Nx, Ny, Nz, Lx, Ly, Lz, Lx / Nx, Ly / Ny, Lz / Nz, tol, goal, (Nx ÷ 2 + 1) * Ny * Nz * N)
end
Base.broadcastable(c::Config) = Ref(c)

# ---- 2. FieldState (src/Types_3d.jl:172-270): the host mirror of one time level ----

mutable struct FieldState
    phi::Array{Float64, 4}         # Nx × Ny × Nz × N
    phi_hat::Array{ComplexF64, 4}  # (Nx÷2+1) × Ny × Nz × N
    psi::Array{Float64, 4}
    psi_hat::Array{ComplexF64, 4}
    u::Array{Float64, 4}           # Nx × Ny × Nz × 3
    u_hat::Array{ComplexF64, 4}
    p::Array{Float64, 3}           # Nx × Ny × Nz
    p_hat::Array{ComplexF64, 3}
    mu::Array{Float64, 4}
    mu_hat::Array{ComplexF64, 4}
    nu::Array{Float64, 4}
    nu_hat::Array{ComplexF64, 4}
    Q::Float64
    R1::Float64
    R2::Float64
    R3::Float64
    A0::Vector{Float64}
    dt::Float64
end

function FieldState(Nx::Int, Ny::Int, Nz::Int, N::Int)
    Nk = Nx ÷ 2 + 1
    r(k) = zeros(Float64, Nx, Ny, Nz, k)
    c(k) = zeros(ComplexF64, Nk, Ny, Nz, k)
    return FieldState(r(N), c(N), r(N), c(N), r(3), c(3), zeros(Nx, Ny, Nz), zeros(ComplexF64, Nk, Ny, Nz),
                      r(N), c(N), r(N), c(N), 0.0, 0.0, 0.0, 0.0, [0.0], 0.0)
end
empty_state(conf::Config) = FieldState(conf.Nx, conf.Ny, conf.Nz, conf.N)

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

# ---- 3. Operators (src/Types_3d.jl:304-350) ----------------------------------------

mutable struct Operators
    h::Ptr{Cvoid}                  # libvsav handle: plans, buffers and both time levels
    ndim::Int
    Nx::Int
    Ny::Int
    Nz::Int
    N::Int
    K::NTuple{3, Array{Float64, 3}}
    D1::NTuple{3, Array{ComplexF64, 3}}
    D1_full::NTuple{3, Array{ComplexF64, 3}}
    Laplacian::Array{Float64, 3}
    Laplacian_full::Array{Float64, 3}
    Biharmonic::Array{Float64, 3}
    gen::Int                       # bumped whenever the device state changes
end

# ---- Step1Cache (src/Types_3d.jl:361-390): 16 device views ---------------------------

struct Step1Cache
    ops::Any
    views::Any                     # NamedTuple of the 16 fields, or nothing before the first Step 1
end
Step1Cache(Nx::Int, Ny::Int, Nz::Int, N::Int) = Step1Cache(nothing, nothing)
function Base.getproperty(c::Step1Cache, s::Symbol)
    s in (:ops, :views) && return getfield(c, s)
    v = getfield(c, :views)
    v === nothing && error("Step1Cache is empty until solve_step1 has run")
    return getproperty(v, s)
end

# ---- 4. BDFCoeff (src/Types_3d.jl:410-430) ------------------------------------------

struct BDFCoeff
    a::Float64
    b::Float64
    c::Float64
end
BDFCoeff(::Val{1}) = BDFCoeff(1.0, -1.0, 0.0)
BDFCoeff(::Val{2}) = BDFCoeff(1.5, -2.0, 0.5)
bdf_coeff(n::Int) = n == 1 ? BDFCoeff(Val(1)) : BDFCoeff(Val(2))
