/* libvsav -- B200 (sm_100a) pseudo-spectral SAV time step for the vesicle
 * growth/shrinkage model of Forstylime/Julia-Vesicles-growth-and-shrinkage.
 *
 * C ABI: plain pointers and sizes.  Every array argument is float64 (complex
 * = interleaved re,im) in C order with x fastest, which is the memory order
 * of the reference's column-major Julia arrays:
 *   phi, psi, mu, nu        Julia (Nx,Ny[,Nz],N)      -> [V][Nz][Ny][Nx]
 *   phi_hat ... nu_hat      Julia (Nx÷2+1,Ny[,Nz],N)  -> [V][Nz][Ny][Nx/2+1] complex
 *   u / u_hat               Julia (Nx,Ny[,Nz],nd)     -> [R][nd][Nz][Ny][Nx]  (one block per run)
 *   p / p_hat               Julia (Nx,Ny[,Nz])        -> [R][Nz][Ny][Nx]
 * V = total vesicle fields of all runs, R = number of independent runs
 * (R = 1 reproduces the reference; Nz = 1 in 2D).
 * Host or device pointers are both accepted where data is copied in or out.
 * All functions return 0 on success or a negative VSAV_E_* code; the text of
 * the last error of a handle is returned by vsav_last_error().
 * One handle = one CUDA stream; a handle is not thread safe.
 */
#ifndef VSAV_H
#define VSAV_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VSAV_OK 0
#define VSAV_E_INVALID (-1)       /* bad argument or unsupported size */
#define VSAV_E_CUDA (-2)          /* CUDA runtime error (text in vsav_last_error) */
#define VSAV_E_WC_NEGATIVE (-3)   /* W_i + C_i < 0 (Utils.jl:162,180,188 "FATAL: W+C<0") */
#define VSAV_E_NONFINITE (-4)     /* NaN/Inf in the SAV scalars */
#define VSAV_W_NOT_CONVERGED 1    /* psi BiCGSTAB hit itmax (Solvers.jl:76 @warn); result still valid */

typedef struct vsav_handle vsav_handle;

/* Config (src/Types.jl:27-134, src/Types_3d.jl:27-140).  Fields the reference
 * types as Int (gamma_area, gamma_in, beta_in, gamma_out, beta_out, lamda) are
 * taken as double.  psi_in_v/psi_out_v have one entry per vesicle field (V). */
typedef struct vsav_config {
  int32_t ndim;                 /* 2 or 3 */
  int32_t Nx, Ny, Nz;           /* powers of two; Nz ignored in 2D */
  int32_t N;                    /* vesicle fields per run when n_runs == 1 */
  double epsilon, M_phi, M0_psi, eta;
  double gamma_surf, gamma_area, gamma_bend;
  double gamma_in, beta_in, gamma_out, beta_out, lamda;
  double S1, S2, S3, S4, C1, C2, C3;
  double dt, T;
  double Lx, Ly, Lz;
  double tol;
  const double* psi_in_v;       /* [V] */
  const double* psi_out_v;      /* [V] */
} vsav_config;

#define VSAV_FP64 0             /* every field and transform in FP64 */
#define VSAV_FP32 1             /* FP32 fields/FFTs; FP64 SAV inner products, 3x3 and Q solves */
#define VSAV_MIXED 2            /* FP64 fields/FFTs; the psi BiCGSTAB (2D, or 3D with psi3d_variable) in FP32
                                   with FP64 iterative refinement */
#define VSAV_PSI_FULL 0         /* psi BiCGSTAB on full complex spectra: the reference's form */
#define VSAV_PSI_HALF 1         /* psi BiCGSTAB on half spectra of real fields (Nyquist-projected) */

typedef struct vsav_options {
  int32_t precision;            /* VSAV_FP64 | VSAV_FP32 */
  int32_t psi_form;             /* VSAV_PSI_FULL | VSAV_PSI_HALF */
  int32_t psi_precond;          /* 0 = diagonal spectral on the left, Krylov.jl form (Solvers.jl:57,73-75);
                                   1 = flexible right-preconditioned BiCGSTAB, diagonal;
                                   2 = flexible, diagonal + learned correction (vsav_set_psi_net) */
  int32_t psi_itmax;            /* Solvers.jl:75 uses 20 */
  double psi_rtol;              /* Solvers.jl:75 uses conf.tol */
  double psi_atol;              /* Solvers.jl:74 uses 1e-14 */
  int32_t n_runs;               /* R >= 1 */
  const int32_t* run_sizes;     /* [R] vesicle fields per run (NULL: R == 1 with N fields) */
  int32_t device;               /* CUDA device ordinal */
  int32_t graph;                /* 1 (default): vsav_run replays each time step after the first as one
                                   CUDA graph (Krylov loops as conditional nodes); 0: eager launches */
  int32_t psi3d_variable;       /* 3D only.  0 (default): psi by the reference's constant-M0_psi spectral
                                   division (Solvers_3d.jl:28-30); 1: the 2D scheme's variable mobility
                                   M_psi(phi*) (Utils_3d.jl:20) and its diagonal-preconditioned BiCGSTAB
                                   (Solvers.jl:26-81) on 3D full spectra -- no counterpart in the reference */
  int32_t psi_stop;             /* 0 (default): stop the psi BiCGSTAB on the preconditioned residual,
                                   ||M^-1 r|| <= atol + rtol ||M^-1 b|| (Krylov.jl's left-preconditioned rule,
                                   Solvers.jl:73-75); 1: on the true residual ||b - A x|| <= atol + rtol ||b||.
                                   The flexible solvers (psi_precond 1, 2) always stop on the true residual */
  int32_t psi_check;            /* 1: after every psi solve, measure ||b - A x|| / ||b|| per system in the
                                   handle's arithmetic (FP64 for VSAV_MIXED): one more operator application
                                   per solve; read with vsav_get_scalar_work(h, 6, out[3R]) */
} vsav_options;

/* field ids (FieldState, src/Types.jl:167-201) */
enum {
  VSAV_PHI = 0, VSAV_PHI_HAT, VSAV_PSI, VSAV_PSI_HAT, VSAV_U, VSAV_U_HAT,
  VSAV_P, VSAV_P_HAT, VSAV_MU, VSAV_MU_HAT, VSAV_NU, VSAV_NU_HAT
};
#define VSAV_PRESENT 0
#define VSAV_OLD 1

typedef struct vsav_status {
  int32_t err_flags;            /* bit0: W1+C1<0, bit1: W2+C2<0, bit2: W3+C3<0 */
  int32_t psi_systems;          /* BiCGSTAB systems solved in the last Step 1 (3 per run) */
  int32_t psi_max_iters;
  int32_t psi_not_converged;
} vsav_status;

/* build_operators(cfg) (SpectralUtils.jl:36-118) + the FieldState/Step1Cache
 * allocations: everything on the device. */
int vsav_create(const vsav_config* cfg, const vsav_options* opt, vsav_handle** out);
int vsav_destroy(vsav_handle* h);
const char* vsav_last_error(const vsav_handle* h);
/* text of the last failed vsav_create on this thread */
const char* vsav_create_error(void);
/* defaults for vsav_options (FP64, FULL psi, reference BiCGSTAB settings) */
void vsav_default_options(vsav_options* opt, const vsav_config* cfg);

/* FieldState upload/download (Types.jl:167-201), level VSAV_PRESENT / VSAV_OLD */
int vsav_set_field(vsav_handle* h, int32_t level, int32_t field, const double* data);
int vsav_get_field(vsav_handle* h, int32_t level, int32_t field, double* data);

/* Float32 frames for headless visualisation (the arrays scripts/visualize.jl
 * plots; no counterpart in the C sense -- the reference draws them with
 * CairoMakie):  VSAV_EXPORT_PHI_SUM, per run, the sum of its vesicle fields
 * + N - 1 (the phi_plot of simulation.jl:124 / Main.jl:119), [R][Nz][Ny][Nx];
 * VSAV_EXPORT_SPEED, per run, |u| (visualize.jl:71-73); VSAV_EXPORT_FIELD +
 * a physical field id (VSAV_PHI, VSAV_PSI, VSAV_U, VSAV_P, VSAV_MU, VSAV_NU), the
 * field as float32 in vsav_get_field's layout.  Computed and narrowed on the
 * device; only float32 crosses to the host. */
#define VSAV_EXPORT_PHI_SUM 0
#define VSAV_EXPORT_SPEED 1
#define VSAV_EXPORT_FIELD 100
int vsav_export_f32(vsav_handle* h, int32_t level, int32_t what, float* data);
/* scalars Q, R1, R2, R3 per run: q4[R][4] */
int vsav_set_scalars(vsav_handle* h, int32_t level, const double* q4);
int vsav_get_scalars(vsav_handle* h, int32_t level, double* q4);
/* present.dt per run (simulation.jl:73) */
int vsav_set_dt(vsav_handle* h, const double* dt);
int vsav_get_dt(vsav_handle* h, double* dt);
/* present.A0 per vesicle field */
int vsav_set_A0(vsav_handle* h, const double* A0);
int vsav_get_A0(vsav_handle* h, double* A0);

/* simulation.jl:22-53: hats of phi/psi/u/p from the physical fields (unless
 * hats_given), A0 = calculate_area(phi), R_i = sqrt(W_i + C_i), Q = 1, initial
 * mu/nu, old = deepcopy(present). */
int vsav_init_state(vsav_handle* h, int32_t hats_given);

/* generate_initial_condition(conf, ops, state_type) (Init.jl:74-216,
 * Init_3d.jl:67-152) evaluated on the device, then vsav_init_state(h, 0) (the
 * rest of simulation.jl:22-53).  goal: 'g' or 's' (Config.goal).  Every run of
 * the handle gets the shapes of its own N: 2D state_type 1 ellipse, 2 smoothed
 * triangle, 3 star, 4 random blob (N = 1), 7/8 stars (N = 2, 3); 3D state_type 1
 * ellipsoid (N = 1); the other types the reference accepts leave phi = 0.
 * psi = -0.1 phi + 0.7 (goal s) or -0.35 phi + 0.45.  blob_u: [R][20], the
 * uniform draws of state_type 4 in the reference's order (an, pn for k = 1..10;
 * Init.jl:155-159), NULL otherwise.  The reference's error() cases (a state_type
 * invalid for N, a goal that contradicts state_type 7/8, N = 2 with a goal other
 * than g/s) return VSAV_E_INVALID, and so do the cases where it raises UndefVarError
 * (N > 3; 3D state_type 7). */
#define VSAV_GOAL_G 'g'
#define VSAV_GOAL_S 's'
int vsav_generate_initial_condition(vsav_handle* h, int32_t state_type, int32_t goal, const double* blob_u);

/* Seeded shape initial conditions computed on the device (2D; no counterpart in
 * the reference, whose generate_initial_condition builds hard-coded shapes on
 * the host, Init.jl:74-216): one shape per vesicle field (V), boundary radius
 * R(theta) = a b / sqrt((b cos theta)^2 + (a sin theta)^2)
 *            + sum_k amp[k] cos(m[k] theta + phase[k])
 * in the frame rotated by rot about (cx, cy) on the grid x_i = -Lx/2 + Lx i/Nx,
 * phi = tanh((R - r) / (sqrt(2) epsilon)) (Init.jl:113),
 * psi = psi_in (1 + phi)/2 + psi_out (1 - phi)/2, u = p = 0; then
 * vsav_init_state(h, 0). */
typedef struct vsav_shape2d {
  double cx, cy, a, b, rot, psi_in, psi_out;
  int32_t nmodes;               /* 0..8 */
  int32_t m[8];
  double amp[8], phase[8];
} vsav_shape2d;
int vsav_init_shapes2d(vsav_handle* h, const vsav_shape2d* shapes);

/* solve_step1..7 (Solvers.jl:14,144,242,267,344,431,459); n is the step index
 * of simulation.jl:71 (n == 1 -> BDF1, else BDF2).  Results stay on the device
 * (Step1Cache and the step intermediates); read them with vsav_get_work. */
int vsav_step1(vsav_handle* h, int32_t n, vsav_status* st);
int vsav_step2(vsav_handle* h, int32_t n);
int vsav_step3(vsav_handle* h);
int vsav_step4(vsav_handle* h, int32_t n);
int vsav_step5(vsav_handle* h, int32_t n);
int vsav_step6(vsav_handle* h);
int vsav_step7(vsav_handle* h, int32_t n);
/* update_state!(old, present) + new present from Steps 6/7 + 6 irffts (simulation.jl:88-110) */
int vsav_update_state(vsav_handle* h);
/* nsteps full time steps (simulation.jl:71-110) starting at step index n0 with
 * dt[k*R + r] for step k, run r (NULL: keep the current dt).  If energy /
 * area_ratio are non-NULL the monitor of simulation.jl:146-148 runs after every
 * step and writes [nsteps][R]. */
int vsav_run(vsav_handle* h, int32_t n0, int32_t nsteps, const double* dt, double* energy,
             double* area_ratio, vsav_status* st);
/* vsav_run bracketed by CUDA events on the handle's stream: device time in ms */
int vsav_time_run(vsav_handle* h, int32_t n0, int32_t nsteps, const double* dt, int32_t monitor,
                  double* device_ms);
/* per-kernel-class timing (CUDA events around each launch of the class, plus
 * the algorithmic bytes of the launch: inputs read once, outputs written once).
 * enable: 1 on, 0 off, 2 reset counters.  kclass: 0 FFT column pass, 1 x-pass
 * r2c, 2 x-pass c2r, 3 x-pass c2c, 4 fused psi x-pass (inverse, x M_psi,
 * forward), 5 psi operator combine, 6 pointwise, 7 learned-preconditioner network,
 * 8 FFT column pass of FP32 data (class 0 then counts the FP64 ones).
 * out3 = (launches, total ms, total bytes). */
int vsav_profile(vsav_handle* h, int32_t enable);
/* kernels launched by this library so far (all handles) */
int64_t vsav_launch_count(void);
int vsav_profile_read(vsav_handle* h, int32_t kclass, double* out3);
/* The FFT kernel variant (elements per thread E, threads per CTA NT) of each
 * pass family that this handle uses, and where the choice came from
 * ("measured" at creation, "process": an earlier handle of the same shape,
 * "file": the JSON file named by the environment variable VSAV_TUNE_FILE,
 * "forced": VSAV_TUNE), as a NUL-terminated JSON object written to buf
 * (capacity cap bytes; *needed receives the size with the NUL, buf may be
 * NULL to query it).  Replaces FFTW's plan-time measurement (the MEASURE
 * planning of src/SpectralUtils.jl:61-71), whose wisdom the reference does not
 * persist either. */
int vsav_get_tuning(vsav_handle* h, char* buf, int64_t cap, int64_t* needed);
/* compute_modified_energy(present, old) and the area ratio (simulation.jl:146-147), per run */
int vsav_monitor(vsav_handle* h, double* energy, double* area_ratio);

/* intermediates: what 0 Step1Cache field (idx 0..15 in the order phi11 phi12
 * phi13 phi14 phi21 psi11 psi12 psi21 mu11 mu12 mu13 mu14 mu21 nu11 nu12 nu21),
 * 1 Step 3 field (phi1 psi1 phi2 psi2 mu1 nu1 mu2 nu2), 2 u_tilde_hat (idx 0/1,
 * [R][nd][..][nkx]), 3 u_tilde physical (idx 0/1), 4 H1,H2,H3,MG physical. */
int vsav_get_work(vsav_handle* h, int32_t what, int32_t idx, double* out);
/* scalar intermediates: 0 Step 2 R values [R][6] (R11 R21 R31 R12 R22 R32),
 * 1 Q [R], 2 theta_1/theta_2 [R][2], 3 area [V], 4 M_max [R],
 * 5 psi BiCGSTAB per system [3R][4] (iters, solved, status, rnorm/eps),
 * 6 measured true relative residual ||b - A x|| / ||b|| per system [3R] of the
 * last psi solves (vsav_options.psi_check; zeros otherwise) */
int vsav_get_scalar_work(vsav_handle* h, int32_t what, double* out);

/* to_spectral! / to_physical! (SpectralUtils.jl:132-148) on nf fields:
 * kind 0 rfft, 1 irfft, 10+m irfft of multiplier m * input
 * (m: 1 D1x, 2 D1y, 3 D1z, 4 Laplacian, 5 Biharmonic).  nf <= 3 V. */
int vsav_transform(vsav_handle* h, int32_t kind, int32_t nf, const double* in, double* out);

/* ---- learned psi preconditioner (no counterpart in the reference, whose
 * Step-1 psi solve uses the diagonal spectral preconditioner only,
 * Solvers.jl:53-75).  A network of five 3x3 convolutions, 2 -> 16 -> 16 -> 16
 * -> 16 -> 1 channels with ReLU after the first four; parameters theta[7409]
 * layer by layer W[o][i][ky][kx] then b[o]; convolution weights used
 * BF16-rounded (nearest even), biases FP32, FP32 accumulation.  Inputs
 * [B][2][H][W] float32, outputs [B][1][H'][W'] float32; periodic convolutions
 * keep the size, valid ones shrink it by 10 (5 layers).  Host or device
 * pointers are accepted. */
typedef struct vsav_net vsav_net;
/* cap_pixels: largest B*H*W of an input batch */
int vsav_net_create(int64_t cap_pixels, int32_t device, vsav_net** out);
int vsav_net_destroy(vsav_net* net);
/* error text of the last failed call (net NULL: of the last failed vsav_net_create) */
const char* vsav_net_last_error(const vsav_net* net);
int vsav_net_nparams(void);
/* sets the FP32 master parameters and resets the Adam state */
int vsav_net_set_params(vsav_net* net, const double* theta);
/* rounded != 0: the weights as used (BF16-rounded) */
int vsav_net_get_params(vsav_net* net, double* theta, int32_t rounded);
/* impl 0: FP32 per-layer kernels (periodic or valid); impl 1: the fused
 * tensor-core kernel of the preconditioner (periodic; H, W powers of two,
 * multiples of 32; BF16 activations) */
int vsav_net_forward(vsav_net* net, const float* x, int32_t B, int32_t H, int32_t W, int32_t periodic,
                     int32_t impl, float* out);
/* loss_kind 0: loss = 1/2 sum (out - t)^2; 1: the residual-norm loss of
 * vsav_net_train (square valid crops, unit weights); and dloss/dtheta
 * (host [7409]), FP32 kernels */
int vsav_net_grad(vsav_net* net, const float* x, const float* t, int32_t B, int32_t H, int32_t W,
                  int32_t periodic, int32_t loss_kind, double op_c0, double* loss, double* grad);
/* nsteps Adam steps (betas 0.9/0.999, eps 1e-8, learning rate lr) on
 * minibatches of `batch` crops drawn with replacement (seeded) from the crop
 * sets x [ncrops][2][S][S] and t [ncrops][1][S-10][S-10] (device pointers,
 * valid convolutions), minimising sum_b w_b sum (out - t)^2 / sum_b w_b sum t^2
 * over the batch, w [ncrops] per-crop weights (device, NULL: all 1).  flip != 0
 * multiplies input channel 0 and the target of each drawn crop by a random
 * sign.  loss_kind 1 replaces out - t by the residual it leaves, L(out - t)
 * with L u = op_c0 u - div_h(M grad_h u) in grid units (5-point conservative
 * stencil, M = 0.075 + 0.025 * input channel 1), at interior output points.
 * The loss per step is written to losses[nsteps] (host, may be NULL). */
int vsav_net_train(vsav_net* net, const float* x, const float* t, const float* w, int64_t ncrops, int32_t S,
                   int32_t batch, int32_t nsteps, double lr, uint64_t seed, int32_t flip, int32_t loss_kind,
                   double op_c0, double* losses);
/* the same weighted loss over a whole crop set, in chunks of `batch` */
int vsav_net_eval(vsav_net* net, const float* x, const float* t, const float* w, int64_t ncrops, int32_t S,
                  int32_t batch, int32_t loss_kind, double op_c0, double* loss);

/* Network parameters (theta[7409], layout above) of the learned psi
 * preconditioner of a handle created with psi_precond = 2 (precision FP32 or
 * MIXED, FULL psi form, 2D, Nx and Ny >= 32).  Must be set before the first
 * Step 1.  (No counterpart in the reference.) */
int vsav_set_psi_net(vsav_handle* h, const double* theta);
/* Training-data harvest (no counterpart in the reference): with
 * max_snapshots > 0 every later psi solve of the handle (FP64, FULL,
 * psi_precond 0) keeps, in device memory, the physical real parts (FP32) of
 * its BiCGSTAB iterates x_k and preconditioned residuals M^-1 (b - A x_k) for
 * k = 0..max_snapshots-1, its final solution and M_psi; 0 turns it off.
 * vsav_psi_harvest_read copies those of the last solve to out (host or device):
 * [nsnap][2][3V][Ny][Nx] (x_k, r_k), then x* [3V][Ny][Nx], then M_psi
 * [V][Ny][Nx]; out == NULL only reports nsnap and the float count needed. */
int vsav_psi_harvest(vsav_handle* h, int32_t max_snapshots);
int vsav_psi_harvest_read(vsav_handle* h, float* out, int64_t capacity, int32_t* nsnap, int64_t* nfloats);

/* No counterpart in the reference (an addition of this library).
 * Inverse 2D real FFT in FP32 that allocates nothing, for callers that cannot
 * call cudaMalloc -- code embedded in a host application that owns all GPU
 * memory (a pool or arena), or that runs where a device allocation would
 * block or is forbidden.  spec: device [nf][Ny][Nx/2+1] complex float
 * (interleaved), out: device [nf][Ny][Nx] float; mult as in vsav_transform
 * (0 none, 1 d/dx, 2 d/dy, 4 Laplacian, 5 biharmonic) with wavenumbers from
 * Lx, Ly; stream: a cudaStream_t or NULL.  The one intermediate buffer lives
 * in a fixed file-scope device array of 8 MiB (1 Mi complex floats) that every
 * GPU holds from library load until process exit: nf * Ny * (Nx/2+1) above
 * that limit is rejected with VSAV_E_INVALID (split the batch), as are Nx or
 * Ny that are not powers of two up to 2048.  The first call on a device
 * resolves that array's device address and uploads the twiddle table
 * (synchronously), so make it before any stream capture.  All calls share the
 * array: calls that can overlap on the GPU (different streams, devices'
 * threads racing on one device) race; serialise them.  vsav_noalloc_error()
 * returns the error text of this thread's last call (empty after a success).
 * The return code covers this call's own launches only: an error that earlier
 * CUDA work left pending on the calling thread is neither reported nor
 * cleared.  Device ordinals up to 63 are supported. */
int vsav_irfft2d_f32_noalloc(const float* spec, float* out, int32_t nf, int32_t Nx, int32_t Ny, double Lx,
                             double Ly, int32_t mult, void* stream);
const char* vsav_noalloc_error(void);

#ifdef __cplusplus
}
#endif
#endif
