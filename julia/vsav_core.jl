# vsav_core.jl -- the part of the drop-in shared by the 2D and the 3D file sets.
#
# The reference keeps every field in host arrays and runs FFTW and Krylov.jl on
# the CPU.  With the drop-in the state lives on the GPU, inside the handle that
# `Operators` wraps; host `FieldState`s are mirrors that move only through
# `upload_state!` / `download_state!`.  The step functions keep the reference's
# names, arguments and return shapes (src/Solvers.jl:14-498,
# src/Solvers_3d.jl:14-467): scalar results (the Step-2 R values, Q, the new
# R1..R3) are plain Float64s, field results are `DeviceView`s -- lazy
# descriptions of a device array that are downloaded when used (`Array(v)`,
# broadcasting, `copyto!`).  A view is valid until the state advances
# (`advance_state!` or `vsav_run`); using it later raises an error.
#
# Every C call goes through libvsav.jl.

include(joinpath(@__DIR__, "libvsav.jl"))

# ---- errors ------------------------------------------------------------------

"""Raise the library's error text for rc < 0 (W + C < 0 becomes the reference's
"FATAL" error, src/Utils.jl:162,180,188); warn on an unconverged psi solve as
src/Solvers.jl:76 does."""
function vsav_check(h::Ptr{Cvoid}, rc::Integer)
    if rc == VSAV_W_NOT_CONVERGED
        @warn "BiCGSTAB did not converge within itmax (psi solve)"
    elseif rc < 0
        msg = h == C_NULL ? unsafe_string(vsav_create_error()) : unsafe_string(vsav_last_error(h))
        error(rc == VSAV_E_WC_NEGATIVE ? "FATAL: W+C<0 ($msg)" : "libvsav error $rc: $msg")
    end
    return rc
end

as_f64ptr(A::Array{Float64}) = pointer(A)
as_f64ptr(A::Array{ComplexF64}) = Ptr{Float64}(pointer(A))

# ---- lazy device views ---------------------------------------------------------

"""A field result that stays on the device.  `Array(v)` downloads it;
broadcasting and `copyto!` download it implicitly."""
struct DeviceView{T, N}
    ops::Any                      # the Operators whose handle holds the data
    gen::Int                      # state generation the view belongs to
    dims::NTuple{N, Int}
    fill!::Function               # fill!(A::Array{T,N}) copies the data into A
end

Base.size(v::DeviceView) = v.dims
Base.eltype(::Type{DeviceView{T, N}}) where {T, N} = T
function Base.Array(v::DeviceView{T, N}) where {T, N}
    v.gen == v.ops.gen || error("stale device view: the state advanced after this step result was made")
    A = Array{T, N}(undef, v.dims)
    v.fill!(A)
    return A
end
Base.collect(v::DeviceView) = Array(v)
Base.Broadcast.broadcastable(v::DeviceView) = Array(v)
Base.copyto!(A::Array, v::DeviceView) = copyto!(A, Array(v))

# shapes in Julia's column-major order (the C ABI's [..][Ny][Nx] buffers)
spatial(ops) = ops.ndim == 2 ? (ops.Nx, ops.Ny) : (ops.Nx, ops.Ny, ops.Nz)
spectral(ops) = ops.ndim == 2 ? (ops.Nx ÷ 2 + 1, ops.Ny) : (ops.Nx ÷ 2 + 1, ops.Ny, ops.Nz)

# a view of vsav_get_work(what, idx): Step1Cache (0), Step 3 (1), u_tilde_hat (2), u_tilde (3)
function work_view(ops, what::Integer, idx::Integer)
    T = what == 3 ? Float64 : ComplexF64
    dims = what <= 1 ? (spectral(ops)..., ops.N) :
           what == 2 ? (spectral(ops)..., ops.ndim) : (spatial(ops)..., ops.ndim)
    return DeviceView{T, length(dims)}(ops, ops.gen, dims,
        A -> GC.@preserve A vsav_check(ops.h, vsav_get_work(ops.h, what, idx, as_f64ptr(A))))
end

# a view of a field of one time level (vsav_get_field)
function field_view(ops, level::Integer, name::Symbol)
    hat = endswith(String(name), "_hat")
    T = hat ? ComplexF64 : Float64
    base = hat ? spectral(ops) : spatial(ops)
    dims = name in (:u, :u_hat) ? (base..., ops.ndim) : name in (:p, :p_hat) ? base : (base..., ops.N)
    return DeviceView{T, length(dims)}(ops, ops.gen, dims,
        A -> GC.@preserve A vsav_check(ops.h, vsav_get_field(ops.h, level, VSAV_FIELD[name], as_f64ptr(A))))
end

# ---- the handle ----------------------------------------------------------------

"""Build the device handle for `conf`.  precision: VSAV_FP64 (the reference's
arithmetic), VSAV_FP32 or VSAV_MIXED; the psi BiCGSTAB settings default to the
reference's (itmax 20, rtol conf.tol, atol 1e-14; src/Solvers.jl:73-75)."""
function vsav_open(conf; precision::Integer = VSAV_FP64, psi_form::Integer = VSAV_PSI_FULL,
                   psi_precond::Integer = 0, device::Integer = 0, graph::Bool = true,
                   psi3d_variable::Bool = false)
    nd = hasproperty(conf, :Nz) ? 3 : 2
    psi_in = Vector{Float64}(conf.psi_in_v)
    psi_out = Vector{Float64}(conf.psi_out_v)
    cfg = VsavConfig(nd, conf.Nx, conf.Ny, nd == 3 ? conf.Nz : 1, conf.N,
                     conf.epsilon, conf.M_phi, conf.M0_psi, conf.eta,
                     conf.gamma_surf, conf.gamma_area, conf.gamma_bend,
                     conf.gamma_in, conf.beta_in, conf.gamma_out, conf.beta_out, conf.lamda,
                     conf.S1, conf.S2, conf.S3, conf.S4, conf.C1, conf.C2, conf.C3,
                     conf.dt, conf.T, conf.Lx, conf.Ly, nd == 3 ? conf.Lz : 0.0, conf.tol,
                     pointer(psi_in), pointer(psi_out))
    opt = VsavOptions()
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve psi_in psi_out begin
        vsav_default_options(opt, cfg)
        opt.precision = precision
        opt.psi_form = psi_form
        opt.psi_precond = psi_precond
        opt.device = device
        opt.graph = graph ? 1 : 0
        opt.psi3d_variable = psi3d_variable ? 1 : 0
        vsav_check(C_NULL, vsav_create(cfg, opt, h))
    end
    return h[], nd
end

vsav_close!(ops) = (ops.h != C_NULL && vsav_destroy(ops.h); ops.h = C_NULL; nothing)

# ---- FieldState transfer ---------------------------------------------------------

const STATE_ARRAYS = (:phi, :phi_hat, :psi, :psi_hat, :u, :u_hat, :p, :p_hat, :mu, :mu_hat, :nu, :nu_hat)

"""Copy a host FieldState into time level `level` of the device state
(fields, Q/R1/R2/R3; A0 and dt as well for the present level)."""
function upload_state!(ops, state, level::Integer = VSAV_PRESENT)
    for name in STATE_ARRAYS
        A = getfield(state, name)
        GC.@preserve A vsav_check(ops.h, vsav_set_field(ops.h, level, VSAV_FIELD[name], as_f64ptr(A)))
    end
    q = [state.Q, state.R1, state.R2, state.R3]
    vsav_check(ops.h, vsav_set_scalars(ops.h, level, q))
    if level == VSAV_PRESENT
        A0 = Vector{Float64}(state.A0)
        length(A0) == ops.N && vsav_check(ops.h, vsav_set_A0(ops.h, A0))
        vsav_check(ops.h, vsav_set_dt(ops.h, [state.dt]))
    end
    ops.gen += 1
    return ops
end

"""Fill a host FieldState from time level `level` of the device state."""
function download_state!(state, ops, level::Integer = VSAV_PRESENT)
    for name in STATE_ARRAYS
        A = getfield(state, name)
        GC.@preserve A vsav_check(ops.h, vsav_get_field(ops.h, level, VSAV_FIELD[name], as_f64ptr(A)))
    end
    q = zeros(4)
    vsav_check(ops.h, vsav_get_scalars(ops.h, level, q))
    state.Q, state.R1, state.R2, state.R3 = q
    A0 = zeros(ops.N)
    vsav_check(ops.h, vsav_get_A0(ops.h, A0))
    state.A0 = A0
    dt = zeros(1)
    vsav_check(ops.h, vsav_get_dt(ops.h, dt))
    state.dt = dt[1]
    return state
end

"""A new host FieldState holding time level `level` of the device state."""
download_state(ops, conf, level::Integer = VSAV_PRESENT) = download_state!(empty_state(conf), ops, level)

"""The state update of src/simulation.jl:88-110 on the device: old <- present,
present <- the Step 6/7 results, the six inverse transforms.  Invalidates
every earlier DeviceView."""
function advance_state!(ops)
    vsav_check(ops.h, vsav_update_state(ops.h))
    ops.gen += 1
    return ops
end

# ---- the seven steps (src/Solvers.jl / src/Solvers_3d.jl) -----------------------

bdf_index(bdf) = bdf.a == 1.0 ? 1 : 2       # vsav_step* take the step index: 1 -> BDF1, else BDF2

# the Step1Cache field order of vsav_get_work(0, idx)
const STEP1_FIELDS = (:phi_11, :phi_12, :phi_13, :phi_14, :phi_21, :psi_11, :psi_12, :psi_21,
                      :mu_11, :mu_12, :mu_13, :mu_14, :mu_21, :nu_11, :nu_12, :nu_21)

function step1_views(ops)
    return NamedTuple{STEP1_FIELDS}(Tuple(work_view(ops, 0, i - 1) for i in 1:16))
end

function step1!(present, ops, dt, bdf)
    present.dt = dt
    vsav_check(ops.h, vsav_set_dt(ops.h, [dt]))
    st = VsavStatus()
    vsav_check(ops.h, vsav_step1(ops.h, bdf_index(bdf), st))
    return st
end

function step2_result(ops, bdf)
    vsav_check(ops.h, vsav_step2(ops.h, bdf_index(bdf)))
    r = zeros(6)
    vsav_check(ops.h, vsav_get_scalar_work(ops.h, 0, r))
    # src/Solvers.jl:230-233
    return (R_11_np1 = r[1], R_21_np1 = r[2], R_31_np1 = r[3],
            R_12_np1 = r[4], R_22_np1 = r[5], R_32_np1 = r[6], ops = ops)
end

function step3_result(ops)
    vsav_check(ops.h, vsav_step3(ops.h))
    v(i) = work_view(ops, 1, i)                     # order phi1 psi1 phi2 psi2 mu1 nu1 mu2 nu2
    # src/Solvers.jl:257-258
    return (phi_1_hat = v(0), mu_1_hat = v(4), psi_1_hat = v(1), nu_1_hat = v(5),
            phi_2_hat = v(2), mu_2_hat = v(6), psi_2_hat = v(3), nu_2_hat = v(7), ops = ops)
end

function step4_result(ops, bdf)
    vsav_check(ops.h, vsav_step4(ops.h, bdf_index(bdf)))
    # src/Solvers.jl:331-336
    return (u_tilde_1_hat = work_view(ops, 2, 0), u_tilde_2_hat = work_view(ops, 2, 1),
            u_tilde_1 = work_view(ops, 3, 0), u_tilde_2 = work_view(ops, 3, 1), ops = ops)
end

function step5_result(ops, bdf)
    vsav_check(ops.h, vsav_step5(ops.h, bdf_index(bdf)))
    q = zeros(1)
    vsav_check(ops.h, vsav_get_scalar_work(ops.h, 1, q))
    return q[1]                                      # src/Solvers.jl:422
end

# Steps 6 and 7 write the new level into the old level's storage, where the
# views below read it until advance_state! swaps the levels.
function step6_result(ops, step4_res, Q_np1)
    vsav_check(ops.h, vsav_step6(ops.h))
    q = zeros(4)
    vsav_check(ops.h, vsav_get_scalars(ops.h, VSAV_OLD, q))
    u1, u2 = step4_res.u_tilde_1_hat, step4_res.u_tilde_2_hat
    ut = DeviceView{ComplexF64, length(u1.dims)}(ops, ops.gen, u1.dims, A -> (A .= Array(u1) .+ Q_np1 .* Array(u2)))
    # src/Solvers.jl:447-452
    return (phi_hat = field_view(ops, VSAV_OLD, :phi_hat), psi_hat = field_view(ops, VSAV_OLD, :psi_hat),
            mu_hat = field_view(ops, VSAV_OLD, :mu_hat), nu_hat = field_view(ops, VSAV_OLD, :nu_hat),
            R1 = q[2], R2 = q[3], R3 = q[4], u_tilde_hat = ut, ops = ops)
end

function step7_result(ops, bdf)
    vsav_check(ops.h, vsav_step7(ops.h, bdf_index(bdf)))
    # src/Solvers.jl:494-497
    return (u_hat = field_view(ops, VSAV_OLD, :u_hat), p_hat = field_view(ops, VSAV_OLD, :p_hat))
end

# ---- monitor ---------------------------------------------------------------------

"""compute_modified_energy and the area ratio of src/simulation.jl:146-148 for
the device's present and old levels."""
function device_monitor(ops)
    e = zeros(1)
    a = zeros(1)
    vsav_check(ops.h, vsav_monitor(ops.h, e, a))
    return e[1], a[1]
end

"""calculate_area of the device's present phi (per vesicle, after a monitor)."""
function device_area(ops)
    device_monitor(ops)
    A = zeros(ops.N)
    vsav_check(ops.h, vsav_get_scalar_work(ops.h, 3, A))
    return A
end

# ---- run_simulation (src/simulation.jl:2-155) -------------------------------------

"""The two-phase time grid of src/simulation.jl:15-19: steps of 1e-7 up to
1e-5, then steps of conf.dt up to T."""
function time_grid(dt::Float64, T::Float64)
    t1 = collect(range(0.0, 1e-5, step = 1e-7))
    t2 = collect(range(1e-5, T, step = dt))
    return vcat(t1, t2[2:end])
end

"""The time loop of run_simulation on the device: the step of index n runs
with dt = Dt[n+1] - Dt[n]; between two save points one vsav_run advances all
steps (each replayed as one CUDA graph) and monitors after every step.  The
state after step n is saved under the label Dt[n] when
floor((Dt[n] + 1e-12) / save_interval) grows (src/simulation.jl:112-143);
`save(state, n)` receives the downloaded present level."""
function device_time_loop(ops, conf, Dt::Vector{Float64}, save_interval::Float64, save)
    Nt = length(Dt)
    energy_history = Float64[]
    area_ratio_history = Float64[]
    save_idx(n) = floor(Int, (Dt[n] + 1e-12) / save_interval)
    last_save_idx = -1
    n = 1
    st = VsavStatus()
    while n <= Nt - 1
        # advance to the next step whose save index grows (or to the end)
        m = n
        while m < Nt - 1 && !(save_idx(m) > last_save_idx)
            m += 1
        end
        k = m - n + 1
        dts = [Dt[j + 1] - Dt[j] for j in n:m]
        e = zeros(k)
        a = zeros(k)
        vsav_check(ops.h, vsav_run(ops.h, n, k, dts, e, a, st))
        ops.gen += 1
        append!(energy_history, e)
        append!(area_ratio_history, a)
        if save_idx(m) > last_save_idx
            save(download_state(ops, conf), m)
            last_save_idx = save_idx(m)
        end
        n = m + 1
    end
    return energy_history, area_ratio_history
end
