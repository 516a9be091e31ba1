# SpectralUtils.jl (drop-in for src/SpectralUtils.jl, 2D) -- build_operators,
# to_spectral!, to_physical! and mult! over libvsav's batched FFT kernels.

# wavenumbers 2π·rfftfreq(n, n/L) and 2π·fftfreq(n, n/L) (Nyquist positive / negative)
vsav_rfreq(n::Int, L::Float64) = [2π * j / L for j in 0:(n ÷ 2)]
vsav_freq(n::Int, L::Float64) = [2π * (j < n ÷ 2 ? j : j - n) / L for j in 0:(n - 1)]

"""build_operators(cfg) (src/SpectralUtils.jl:36-118): the device handle (FFT
kernel variants autotuned at creation, all buffers, both time levels) and the
host k-tables K, D1, D1_full, Laplacian, Laplacian_full, Biharmonic with the
reference's shapes and Nyquist conventions.  precision and friends are
passed to vsav_open (vsav_core.jl)."""
function build_operators(cfg::Config; kwargs...)
    h, nd = vsav_open(cfg; kwargs...)
    kx = reshape(vsav_rfreq(cfg.Nx, cfg.Lx), :, 1)
    kx0 = reshape(vsav_freq(cfg.Nx, cfg.Lx), :, 1)
    ky = reshape(vsav_freq(cfg.Ny, cfg.Ly), 1, :)
    # the reference's shapes: kx (Nx÷2+1)×1, kx0 Nx×1, ky 1×Ny, the operators broadcast to full size
    K2 = kx .^ 2 .+ ky .^ 2
    ops = Operators(h, nd, cfg.Nx, cfg.Ny, 1, cfg.N, (kx, ky),
                    (complex.(0.0, kx), complex.(0.0, ky)), (complex.(0.0, kx0), complex.(0.0, ky)),
                    -K2, -(kx0 .^ 2 .+ ky .^ 2), K2 .^ 2, 0)
    finalizer(vsav_close!, ops)
    return ops
end

nfields(A::AbstractArray, per::Int) = length(A) ÷ per

"""to_spectral!(buffer, u, ops): rfft of every Nx × Ny slice of u (at most 3N slices)."""
function to_spectral!(buffer::AbstractArray{ComplexF64}, u::AbstractArray{Float64}, ops::Operators)
    uc = Array{Float64}(u)
    out = Array{ComplexF64}(undef, size(buffer))
    GC.@preserve uc out vsav_check(ops.h, vsav_transform(ops.h, 0, nfields(uc, ops.Nx * ops.Ny), pointer(uc),
                                                         as_f64ptr(out)))
    copyto!(buffer, out)
    return buffer
end

"""to_physical!(buffer, u_hat, ops): normalised irfft (FFTW's c2r convention:
only Re of the kx = 0 and kx = Nx/2 bins) of every half-spectrum slice."""
function to_physical!(buffer::AbstractArray{Float64}, u_hat::AbstractArray{ComplexF64}, ops::Operators;
                      mult::Integer = 0)
    uc = Array{ComplexF64}(u_hat)
    out = Array{Float64}(undef, size(buffer))
    kind = mult == 0 ? 1 : 10 + mult               # 10+m: irfft of multiplier m (1 D1x, 2 D1y, 4 Lap, 5 Bih)
    GC.@preserve uc out vsav_check(ops.h, vsav_transform(ops.h, kind, nfields(uc, (ops.Nx ÷ 2 + 1) * ops.Ny),
                                                         as_f64ptr(uc), pointer(out)))
    copyto!(buffer, out)
    return buffer
end

"""mult!(buffer, u_hat, v_hat, ops) (src/SpectralUtils.jl:158-167): the
spectrum of the pointwise product of the two fields."""
function mult!(buffer::AbstractArray{ComplexF64}, u_hat::AbstractArray{ComplexF64},
               v_hat::AbstractArray{ComplexF64}, ops::Operators)
    sz = (ops.Nx, ops.Ny, nfields(u_hat, (ops.Nx ÷ 2 + 1) * ops.Ny))
    u = to_physical!(zeros(sz), u_hat, ops)
    v = to_physical!(zeros(sz), v_hat, ops)
    return to_spectral!(buffer, u .* v, ops)
end
