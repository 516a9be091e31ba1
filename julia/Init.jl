# Init.jl (drop-in for src/Init.jl, 2D) -- set_para_base and
# generate_initial_condition, the latter evaluated on the device.

"""set_para_base(dt, T): the reference's default 2D parameter set (one
vesicle, 256², unit box, ε = 0.01, shrinkage goal; S1..S4 from ε and
γ_bend as src/Init.jl:40-43 derives them)."""
function set_para_base(dt::Float64, T::Float64)
    N = 1
    goal = :s
    epsilon = 0.01
    gamma_bend = 0.1
    gamma_in = gamma_out = 1e5
    psi_in_v, psi_out_v = if N == 1
        (goal === :g ? [0.65] : goal === :s ? [0.1] : error("what's the goal? now it is $goal")), [0.8]
    elseif N == 2
        (goal === :g ? [0.65, 0.65] : goal === :s ? [0.1, 0.1] : error("what's the goal? now it is $goal")), [0.8, 0.8]
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
                  Nx = 256, Ny = 256, Lx = 1.0 * N, Ly = 1.0, tol = 1e-12, goal = goal)
end

"""generate_initial_condition(conf, ops, state_type) (src/Init.jl:74-216):
the reference's shapes evaluated on the device, followed there by the rest of
the initialisation of src/simulation.jl:25-53 (A0, R1..R3 = sqrt(W + C),
Q = 1, μ and ν, old = present).  Returns the present level as a host
FieldState.  state_type 4 draws its 20 uniforms here, in the order the
reference draws them (aₙ, pₙ for n = 1..10), so the blob is the reference's."""
function generate_initial_condition(conf, ops, state_type::Int)
    blob = state_type == 4 ? [rand() for _ in 1:20] : Float64[]
    GC.@preserve blob vsav_check(ops.h, vsav_generate_initial_condition(ops.h, state_type, Int32(first(String(conf.goal))),
                                                                        isempty(blob) ? C_NULL : pointer(blob)))
    ops.gen += 1
    return download_state(ops, conf)
end
