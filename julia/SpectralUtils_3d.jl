# SpectralUtils_3d.jl (drop-in for src/SpectralUtils_3d.jl, 3D) -- build_operators,
# to_spectral!, to_physical! and mult! over libvsav's batched 3D FFT kernels.

vsav_rfreq(n::Int, L::Float64) = [2π * j / L for j in 0:(n ÷ 2)]
vsav_freq(n::Int, L::Float64) = [2π * (j < n ÷ 2 ? j : j - n) / L for j in 0:(n - 1)]

"""build_operators(cfg) (src/SpectralUtils_3d.jl:36-160): the device handle and
the host k-tables in the reference's 3D shapes (kx (Nx÷2+1)×1×1, kx0 Nx×1×1,
ky 1×Ny×1, kz 1×1×Nz; fftfreq Nyquist negative along y and z).  Keyword
arguments go to vsav_open (psi3d_variable = true selects the variable-mobility
ψ solve, an option without a reference counterpart)."""
function build_operators(cfg::Config; kwargs...)
    h, nd = vsav_open(cfg; kwargs...)
    kx = reshape(vsav_rfreq(cfg.Nx, cfg.Lx), :, 1, 1)
    kx0 = reshape(vsav_freq(cfg.Nx, cfg.Lx), :, 1, 1)
    ky = reshape(vsav_freq(cfg.Ny, cfg.Ly), 1, :, 1)
    kz = reshape(vsav_freq(cfg.Nz, cfg.Lz), 1, 1, :)
    K2 = kx .^ 2 .+ ky .^ 2 .+ kz .^ 2
    i0(k) = complex.(0.0, k)
    ops = Operators(h, nd, cfg.Nx, cfg.Ny, cfg.Nz, cfg.N, (kx, ky, kz), (i0(kx), i0(ky), i0(kz)),
                    (i0(kx0), i0(ky), i0(kz)), -K2, -(kx0 .^ 2 .+ ky .^ 2 .+ kz .^ 2), K2 .^ 2, 0)
    finalizer(vsav_close!, ops)
    return ops
end

nfields(A::AbstractArray, per::Int) = length(A) ÷ per

"""to_spectral!(buffer, u, ops): rfft of every Nx × Ny × Nz block of u."""
function to_spectral!(buffer::AbstractArray{ComplexF64}, u::AbstractArray{Float64}, ops::Operators)
    uc = Array{Float64}(u)
    out = Array{ComplexF64}(undef, size(buffer))
    GC.@preserve uc out vsav_check(ops.h, vsav_transform(ops.h, 0, nfields(uc, ops.Nx * ops.Ny * ops.Nz),
                                                         pointer(uc), as_f64ptr(out)))
    copyto!(buffer, out)
    return buffer
end

"""to_physical!(buffer, u_hat, ops): normalised 3D irfft (c2r convention of FFTW)."""
function to_physical!(buffer::AbstractArray{Float64}, u_hat::AbstractArray{ComplexF64}, ops::Operators;
                      mult::Integer = 0)
    uc = Array{ComplexF64}(u_hat)
    out = Array{Float64}(undef, size(buffer))
    kind = mult == 0 ? 1 : 10 + mult
    GC.@preserve uc out vsav_check(ops.h, vsav_transform(ops.h, kind,
                                                         nfields(uc, (ops.Nx ÷ 2 + 1) * ops.Ny * ops.Nz),
                                                         as_f64ptr(uc), pointer(out)))
    copyto!(buffer, out)
    return buffer
end

"""mult!(buffer, u_hat, v_hat, ops) (src/SpectralUtils_3d.jl:164-173)."""
function mult!(buffer::AbstractArray{ComplexF64}, u_hat::AbstractArray{ComplexF64},
               v_hat::AbstractArray{ComplexF64}, ops::Operators)
    sz = (ops.Nx, ops.Ny, ops.Nz, nfields(u_hat, (ops.Nx ÷ 2 + 1) * ops.Ny * ops.Nz))
    u = to_physical!(zeros(sz), u_hat, ops)
    v = to_physical!(zeros(sz), v_hat, ops)
    return to_spectral!(buffer, u .* v, ops)
end
