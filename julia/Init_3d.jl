# Init_3d.jl (drop-in for src/Init_3d.jl, 3D) -- set_para_base and
# generate_initial_condition, the latter evaluated on the device.

"""set_para_base(dt, T): the reference's default 3D parameter set (one
vesicle, 128³, unit box, ε = 0.01, growth goal; S1..S4 from ε and γ_bend)."""
function set_para_base(dt::Float64, T::Float64)
    N = 1
    goal = :g
    epsilon = 0.01
    gamma_bend = 0.1
    gamma_in = gamma_out = 1e5
    psi_in_v, psi_out_v = if N == 1
        (goal === :s ? [0.1] : [0.65]), [0.8]
    elseif N == 2
        [0.65, 0.65], [0.8, 0.8]
    else
        [0.1, 0.65, 0.5], [0.8, 0.6, 0.4]
    end
    return Config(N = N, epsilon = epsilon, M_phi = 1.0, M0_psi = 0.5, eta = 1.0,
                  gamma_surf = 1.0, gamma_area = 5e4, gamma_bend = gamma_bend,
                  gamma_in = gamma_in, beta_in = 0.0, psi_in_v = psi_in_v,
                  gamma_out = gamma_out, beta_out = 0.0, psi_out_v = psi_out_v, lamda = 1.0,
                  S1 = (3 * sqrt(2) / 8) * epsilon * gamma_bend, S2 = 0.0,
                  S3 = gamma_bend / epsilon^3, S4 = min(gamma_in, gamma_out),
                  C1 = 1.0, C2 = 5.0e5, C3 = 1.0e6, dt = dt, T = T,
                  Nx = 128, Ny = 128, Nz = 128, Lx = 1.0, Ly = 1.0, Lz = 1.0, tol = 1e-12, goal = goal)
end

"""generate_initial_condition(conf, ops, state_type) (src/Init_3d.jl:67-152) on
the device, followed there by the SAV initialisation of src/simulation.jl:25-53.
Returns the present level as a host FieldState."""
function generate_initial_condition(conf, ops, state_type::Int)
    vsav_check(ops.h, vsav_generate_initial_condition(ops.h, state_type, Int32(first(String(conf.goal))), C_NULL))
    ops.gen += 1
    return download_state(ops, conf)
end
