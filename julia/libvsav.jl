# libvsav.jl -- one Julia binding per function of include/vsav.h.
#
# Every function below is a direct `ccall` into libvsav.so with the argument
# and return types of its C prototype (int32_t -> Int32, int64_t -> Int64,
# double -> Float64, int -> Cint, const char* result -> Cstring, opaque
# handles -> Ptr{Cvoid}, arrays -> Ptr{element type}).  The higher-level
# drop-in files (Types.jl, SpectralUtils.jl, Utils.jl, Init.jl, Solvers.jl,
# simulation.jl and their _3d twins) call only these.
#
# The library path can be overridden with the environment variable LIBVSAV.

const libvsav = get(ENV, "LIBVSAV",
                    normpath(joinpath(@__DIR__, "..", "julia-vesicles-growth-and-shrinkage_b200", "vsav", "libvsav.so")))

# ---- C structs (field order and types as in include/vsav.h) -----------------

struct VsavConfig
    ndim::Int32
    Nx::Int32
    Ny::Int32
    Nz::Int32
    N::Int32
    epsilon::Float64
    M_phi::Float64
    M0_psi::Float64
    eta::Float64
    gamma_surf::Float64
    gamma_area::Float64
    gamma_bend::Float64
    gamma_in::Float64
    beta_in::Float64
    gamma_out::Float64
    beta_out::Float64
    lamda::Float64
    S1::Float64
    S2::Float64
    S3::Float64
    S4::Float64
    C1::Float64
    C2::Float64
    C3::Float64
    dt::Float64
    T::Float64
    Lx::Float64
    Ly::Float64
    Lz::Float64
    tol::Float64
    psi_in_v::Ptr{Float64}
    psi_out_v::Ptr{Float64}
end

mutable struct VsavOptions
    precision::Int32
    psi_form::Int32
    psi_precond::Int32
    psi_itmax::Int32
    psi_rtol::Float64
    psi_atol::Float64
    n_runs::Int32
    run_sizes::Ptr{Int32}
    device::Int32
    graph::Int32
    psi3d_variable::Int32
    psi_stop::Int32
    psi_check::Int32
end
VsavOptions() = VsavOptions(0, 0, 0, 20, 1e-12, 1e-14, 1, C_NULL, 0, 1, 0, 0, 0)

mutable struct VsavStatus
    err_flags::Int32
    psi_systems::Int32
    psi_max_iters::Int32
    psi_not_converged::Int32
end
VsavStatus() = VsavStatus(0, 0, 0, 0)

struct VsavShape2D
    cx::Float64
    cy::Float64
    a::Float64
    b::Float64
    rot::Float64
    psi_in::Float64
    psi_out::Float64
    nmodes::Int32
    m::NTuple{8, Int32}
    amp::NTuple{8, Float64}
    phase::NTuple{8, Float64}
end

# ---- constants --------------------------------------------------------------

const VSAV_OK = 0
const VSAV_E_INVALID = -1
const VSAV_E_CUDA = -2
const VSAV_E_WC_NEGATIVE = -3
const VSAV_E_NONFINITE = -4
const VSAV_W_NOT_CONVERGED = 1
const VSAV_FP64 = 0
const VSAV_FP32 = 1
const VSAV_MIXED = 2
const VSAV_PSI_FULL = 0
const VSAV_PSI_HALF = 1
const VSAV_PRESENT = 0
const VSAV_OLD = 1
const VSAV_FIELD = Dict(:phi => 0, :phi_hat => 1, :psi => 2, :psi_hat => 3, :u => 4, :u_hat => 5,
                        :p => 6, :p_hat => 7, :mu => 8, :mu_hat => 9, :nu => 10, :nu_hat => 11)
const VSAV_EXPORT_PHI_SUM = 0
const VSAV_EXPORT_SPEED = 1
const VSAV_EXPORT_FIELD = 100

# ---- handle life cycle --------------------------------------------------------

vsav_create(cfg, opt, out) =
    ccall((:vsav_create, libvsav), Cint, (Ref{VsavConfig}, Ref{VsavOptions}, Ptr{Ptr{Cvoid}}), cfg, opt, out)
vsav_destroy(h) = ccall((:vsav_destroy, libvsav), Cint, (Ptr{Cvoid},), h)
vsav_last_error(h) = ccall((:vsav_last_error, libvsav), Cstring, (Ptr{Cvoid},), h)
vsav_create_error() = ccall((:vsav_create_error, libvsav), Cstring, ())
vsav_default_options(opt, cfg) =
    ccall((:vsav_default_options, libvsav), Cvoid, (Ref{VsavOptions}, Ref{VsavConfig}), opt, cfg)

# ---- FieldState upload / download -------------------------------------------

vsav_set_field(h, level, field, data) =
    ccall((:vsav_set_field, libvsav), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}), h, level, field, data)
vsav_get_field(h, level, field, data) =
    ccall((:vsav_get_field, libvsav), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}), h, level, field, data)
vsav_export_f32(h, level, what, data) =
    ccall((:vsav_export_f32, libvsav), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Float32}), h, level, what, data)
vsav_set_scalars(h, level, q4) =
    ccall((:vsav_set_scalars, libvsav), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}), h, level, q4)
vsav_get_scalars(h, level, q4) =
    ccall((:vsav_get_scalars, libvsav), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}), h, level, q4)
vsav_set_dt(h, dt) = ccall((:vsav_set_dt, libvsav), Cint, (Ptr{Cvoid}, Ptr{Float64}), h, dt)
vsav_get_dt(h, dt) = ccall((:vsav_get_dt, libvsav), Cint, (Ptr{Cvoid}, Ptr{Float64}), h, dt)
vsav_set_A0(h, A0) = ccall((:vsav_set_A0, libvsav), Cint, (Ptr{Cvoid}, Ptr{Float64}), h, A0)
vsav_get_A0(h, A0) = ccall((:vsav_get_A0, libvsav), Cint, (Ptr{Cvoid}, Ptr{Float64}), h, A0)

# ---- initialisation ---------------------------------------------------------

vsav_init_state(h, hats_given) = ccall((:vsav_init_state, libvsav), Cint, (Ptr{Cvoid}, Int32), h, hats_given)
vsav_generate_initial_condition(h, state_type, goal, blob_u) =
    ccall((:vsav_generate_initial_condition, libvsav), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}),
          h, state_type, goal, blob_u)
vsav_init_shapes2d(h, shapes) =
    ccall((:vsav_init_shapes2d, libvsav), Cint, (Ptr{Cvoid}, Ptr{VsavShape2D}), h, shapes)

# ---- the seven steps, the state update and the loop ----------------------------

vsav_step1(h, n, st) = ccall((:vsav_step1, libvsav), Cint, (Ptr{Cvoid}, Int32, Ref{VsavStatus}), h, n, st)
vsav_step2(h, n) = ccall((:vsav_step2, libvsav), Cint, (Ptr{Cvoid}, Int32), h, n)
vsav_step3(h) = ccall((:vsav_step3, libvsav), Cint, (Ptr{Cvoid},), h)
vsav_step4(h, n) = ccall((:vsav_step4, libvsav), Cint, (Ptr{Cvoid}, Int32), h, n)
vsav_step5(h, n) = ccall((:vsav_step5, libvsav), Cint, (Ptr{Cvoid}, Int32), h, n)
vsav_step6(h) = ccall((:vsav_step6, libvsav), Cint, (Ptr{Cvoid},), h)
vsav_step7(h, n) = ccall((:vsav_step7, libvsav), Cint, (Ptr{Cvoid}, Int32), h, n)
vsav_update_state(h) = ccall((:vsav_update_state, libvsav), Cint, (Ptr{Cvoid},), h)
vsav_run(h, n0, nsteps, dt, energy, area_ratio, st) =
    ccall((:vsav_run, libvsav), Cint,
          (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ref{VsavStatus}),
          h, n0, nsteps, dt, energy, area_ratio, st)
vsav_time_run(h, n0, nsteps, dt, monitor, device_ms) =
    ccall((:vsav_time_run, libvsav), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}, Int32, Ptr{Float64}),
          h, n0, nsteps, dt, monitor, device_ms)

# ---- measurement --------------------------------------------------------------

vsav_profile(h, enable) = ccall((:vsav_profile, libvsav), Cint, (Ptr{Cvoid}, Int32), h, enable)
vsav_launch_count() = ccall((:vsav_launch_count, libvsav), Int64, ())
vsav_profile_read(h, kclass, out3) =
    ccall((:vsav_profile_read, libvsav), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}), h, kclass, out3)
vsav_get_tuning(h, buf, cap, needed) =
    ccall((:vsav_get_tuning, libvsav), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Int64, Ptr{Int64}), h, buf, cap, needed)

# ---- monitor, intermediates, transforms ----------------------------------------

vsav_monitor(h, energy, area_ratio) =
    ccall((:vsav_monitor, libvsav), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}), h, energy, area_ratio)
vsav_get_work(h, what, idx, out) =
    ccall((:vsav_get_work, libvsav), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}), h, what, idx, out)
vsav_get_scalar_work(h, what, out) =
    ccall((:vsav_get_scalar_work, libvsav), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}), h, what, out)
vsav_transform(h, kind, nf, inp, out) =
    ccall((:vsav_transform, libvsav), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}, Ptr{Float64}),
          h, kind, nf, inp, out)

# ---- learned psi preconditioner -----------------------------------------------

vsav_net_create(cap_pixels, device, out) =
    ccall((:vsav_net_create, libvsav), Cint, (Int64, Int32, Ptr{Ptr{Cvoid}}), cap_pixels, device, out)
vsav_net_destroy(net) = ccall((:vsav_net_destroy, libvsav), Cint, (Ptr{Cvoid},), net)
vsav_net_last_error(net) = ccall((:vsav_net_last_error, libvsav), Cstring, (Ptr{Cvoid},), net)
vsav_net_nparams() = ccall((:vsav_net_nparams, libvsav), Cint, ())
vsav_net_set_params(net, theta) =
    ccall((:vsav_net_set_params, libvsav), Cint, (Ptr{Cvoid}, Ptr{Float64}), net, theta)
vsav_net_get_params(net, theta, rounded) =
    ccall((:vsav_net_get_params, libvsav), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int32), net, theta, rounded)
vsav_net_forward(net, x, B, H, W, periodic, impl, out) =
    ccall((:vsav_net_forward, libvsav), Cint,
          (Ptr{Cvoid}, Ptr{Float32}, Int32, Int32, Int32, Int32, Int32, Ptr{Float32}),
          net, x, B, H, W, periodic, impl, out)
vsav_net_grad(net, x, t, B, H, W, periodic, loss_kind, op_c0, loss, grad) =
    ccall((:vsav_net_grad, libvsav), Cint,
          (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Int32, Int32, Int32, Int32, Int32, Float64, Ptr{Float64},
           Ptr{Float64}),
          net, x, t, B, H, W, periodic, loss_kind, op_c0, loss, grad)
vsav_net_train(net, x, t, w, ncrops, S, batch, nsteps, lr, seed, flip, loss_kind, op_c0, losses) =
    ccall((:vsav_net_train, libvsav), Cint,
          (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Int64, Int32, Int32, Int32, Float64, UInt64,
           Int32, Int32, Float64, Ptr{Float64}),
          net, x, t, w, ncrops, S, batch, nsteps, lr, seed, flip, loss_kind, op_c0, losses)
vsav_net_eval(net, x, t, w, ncrops, S, batch, loss_kind, op_c0, loss) =
    ccall((:vsav_net_eval, libvsav), Cint,
          (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Int64, Int32, Int32, Int32, Float64,
           Ptr{Float64}),
          net, x, t, w, ncrops, S, batch, loss_kind, op_c0, loss)
vsav_set_psi_net(h, theta) = ccall((:vsav_set_psi_net, libvsav), Cint, (Ptr{Cvoid}, Ptr{Float64}), h, theta)
vsav_psi_harvest(h, max_snapshots) =
    ccall((:vsav_psi_harvest, libvsav), Cint, (Ptr{Cvoid}, Int32), h, max_snapshots)
vsav_psi_harvest_read(h, out, capacity, nsnap, nfloats) =
    ccall((:vsav_psi_harvest_read, libvsav), Cint, (Ptr{Cvoid}, Ptr{Float32}, Int64, Ptr{Int32}, Ptr{Int64}),
          h, out, capacity, nsnap, nfloats)

# ---- allocation-free inverse FFT ----------------------------------------------

vsav_irfft2d_f32_noalloc(spec, out, nf, Nx, Ny, Lx, Ly, mult, stream) =
    ccall((:vsav_irfft2d_f32_noalloc, libvsav), Cint,
          (Ptr{Float32}, Ptr{Float32}, Int32, Int32, Int32, Float64, Float64, Int32, Ptr{Cvoid}),
          spec, out, nf, Nx, Ny, Lx, Ly, mult, stream)
vsav_noalloc_error() = ccall((:vsav_noalloc_error, libvsav), Cstring, ())
