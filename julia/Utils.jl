# Utils.jl (drop-in for src/Utils.jl, 2D and 3D) -- the pointwise helpers and
# energy densities on host arrays (their spectral derivatives through
# libvsav's transforms), and the monitor quantities of the device state.
#
# The SAV functionals the time step needs (get_W1..3, get_H1..3, get_MG,
# get_omega) run on the device inside vsav_init_state and vsav_step1/2; they
# have no host version here.

g(phi) = @. 0.25 * (phi^2 - 1.0)^2                    # double well
g_prime(phi) = @. phi * (phi^2 - 1.0)
p_phi(phi) = @. -0.5 * phi^3 + 1.5 * phi              # interpolation function
p_phi_prime(phi) = @. -1.5 * phi^2 + 1.5
get_M_psi(phi, conf) = @. 0.1 * (1.0 - conf.M0_psi * (phi^2 - 1.0)^2)

cell_volume(conf) = hasproperty(conf, :Nz) ? conf.dx * conf.dy * conf.dz : conf.dx * conf.dy
integrate(f, conf) = sum(f) * cell_volume(conf)
integrate_sq(f, conf) = sum(abs2, f) * cell_volume(conf)

# derivative / Laplacian of phi on the host grid through the device transforms
function spectral_apply(phi::AbstractArray{Float64}, ops, mult::Integer)
    phi_hat = to_spectral!(zeros(ComplexF64, spectral(ops)..., size(phi)[end]), phi, ops)
    return to_physical!(zeros(size(phi)), phi_hat, ops; mult = mult)
end

"""f_surf: (3√2/4) g(φ)/ε + ε |∇φ|²/2.  The 3D reference omits ∂z (src/Utils_3d.jl:38-41),
and so does this density in 3D."""
function f_surf(phi::AbstractArray{Float64}, ops, conf)
    gx = spectral_apply(phi, ops, 1)
    gy = spectral_apply(phi, ops, 2)
    ε = conf.epsilon
    return @. (3 * sqrt(2) / 4) * (g(phi) / ε) + ε * (gx^2 + gy^2) / 2
end

"""f_bend: (3√2/(16ε)) (g'(φ)/ε − ε Δφ)²."""
function f_bend(phi::AbstractArray{Float64}, ops, conf)
    lap = spectral_apply(phi, ops, 4)
    ε = conf.epsilon
    return @. (3 * sqrt(2) / (16ε)) * (g_prime(phi) / ε - ε * lap)^2
end

"""f_osmotic: the p(φ)-weighted inside / outside osmotic densities."""
function f_osmotic(phi, psi, conf)
    P = p_phi(phi)
    sh = ntuple(i -> i == ndims(phi) ? length(conf.psi_in_v) : 1, ndims(phi))
    pin = reshape(conf.psi_in_v, sh)
    pout = reshape(conf.psi_out_v, sh)
    f_in = @. 0.5 * conf.gamma_in * (psi - pin)^2 + conf.beta_in
    f_out = @. 0.5 * conf.gamma_out * (psi - pout)^2 + conf.beta_out
    return @. ((1 + P) / 2) * f_in + ((1 - P) / 2) * f_out
end

"""calculate_area: ∫ f_surf per vesicle field (host array phi)."""
function calculate_area(phi::AbstractArray{Float64}, ops, conf)
    s = f_surf(phi, ops, conf)
    return [integrate(selectdim(s, ndims(s), n), conf) for n in 1:conf.N]
end

"""compute_modified_energy(present, old, ops, conf) (src/Utils.jl:96-141) of
the DEVICE state's present and old levels, which the host mirrors `present`
and `old` are expected to copy."""
compute_modified_energy(present, old, ops, conf) = device_monitor(ops)[1]
