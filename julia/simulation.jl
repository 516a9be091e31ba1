# simulation.jl (drop-in for src/simulation.jl, 2D and 3D) -- run_simulation
# with the reference's arguments, time grid, save schedule and return value
# (src/simulation.jl:2-155); the time loop runs on the device.
using Printf

"""run_simulation(dt_val, T_val, state_type; save_path, save_interval) ->
(present, energy_history, area_ratio_history, Dt).

Parameters from set_para_base, the two-phase time grid of
src/simulation.jl:15-19, the initial condition and its SAV initialisation on
the device, then every step (Steps 1-7, state update, modified energy, area
ratio) on the device, between save points in one vsav_run call each.  At a
save point the present level is downloaded and written as
save_path/MAT/state_2d_t<time>.mat (state_3d_ in 3D) when MAT.jl's matwrite
is loaded, and φ summed over the vesicles is plotted when visualize.jl's
plot_field is loaded, as in the reference.  `present` is the final state as a
host FieldState."""
function run_simulation(dt_val::Float64, T_val::Float64, state_type::Int;
                        save_path::String = "./results", save_interval::Float64 = 0.001)
    conf = set_para_base(dt_val, T_val)
    ops = build_operators(conf)
    mkpath(save_path)
    mat_folder = joinpath(save_path, "MAT")
    mkpath(mat_folder)
    Dt = time_grid(conf.dt, T_val)
    present = generate_initial_condition(conf, ops, state_type)
    @info "simulation starts: initial area = $(present.A0), steps = $(length(Dt) - 1)"
    three_d = hasproperty(conf, :Nz)
    function save(state, n)
        t_str = @sprintf("%.2e", Dt[n])
        data = Dict("phi" => state.phi, "psi" => state.psi, "mu" => state.mu, "nu" => state.nu,
                    "p" => state.p, "u" => state.u, "R1" => state.R1, "R2" => state.R2, "R3" => state.R3,
                    "Q" => state.Q)
        if !three_d && isdefined(Main, :plot_field)
            phi_plot = dropdims(sum(state.phi, dims = 3), dims = 3) .+ conf.N .- 1
            Main.plot_field(phi_plot, conf, title = @sprintf("phi  (t = %.2e)", Dt[n]),
                            filename = joinpath(save_path, "phi_t$(t_str).png"))
        end
        if isdefined(Main, :matwrite)
            Main.matwrite(joinpath(mat_folder, (three_d ? "state_3d_t" : "state_2d_t") * t_str * ".mat"), data)
        end
    end
    energy_history, area_ratio_history = device_time_loop(ops, conf, Dt, save_interval, save)
    present = download_state(ops, conf)
    return present, energy_history, area_ratio_history, Dt
end
