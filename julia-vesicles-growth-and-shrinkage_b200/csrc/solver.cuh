// Host orchestration of one SAV time step on the device: the analogue of
// Operators (src/Types.jl:298-342) + solve_step1..7 (src/Solvers.jl) + the
// loop body of run_simulation (src/simulation.jl:71-148).
//
// All state lives on the device.  Two time levels (present, old) are swapped
// by pointer at the end of a step, which is what update_state!
// (src/Types.jl:243-265) achieves by copying.
#pragma once
#include <vector>
#include <cstring>
#include <string>
#include <memory>
#include <algorithm>
#include <type_traits>
#include <cstdlib>
#include <map>
#include <cstdio>
#include <mutex>
#include "psi.cuh"
#include "cols_tma.cuh"
#include "c2r_bulk.cuh"
#include "net_apply.cuh"
#include "net_tc.cuh"

namespace vsav {

enum FieldId : int { F_PHI = 0, F_PHI_HAT, F_PSI, F_PSI_HAT, F_U, F_U_HAT, F_P, F_P_HAT, F_MU, F_MU_HAT, F_NU, F_NU_HAT };

struct Options {
  int precision = 0;       // 0 FP64, 1 FP32 bulk
  int psi_form = 0;        // 0 FULL (reference form), 1 HALF
  int psi_precond = 0;     // 0 diagonal on the left (Krylov.jl form), 1 flexible right-preconditioned
                          // BiCGSTAB with the diagonal, 2 the same with diagonal + learned correction
  int psi_itmax = 20;
  double psi_rtol = 1e-12, psi_atol = 1e-14;
  int check_every_iter = 1;  // read back convergence flags each BiCGSTAB iteration
  int psi_mixed = 0;         // FP64 fields with the psi BiCGSTAB in FP32 + FP64 iterative refinement
  int psi_refine_min = 1;    // least refinement sweeps of the mixed mode
  double psi_inner_rtol = 1e-6;   // tightest relative tolerance of one FP32 sweep
  int graph = 1;             // vsav_run replays each time step as a CUDA graph
  int psi3d_var = 0;         // 3D: variable psi mobility + BiCGSTAB (the 2D scheme) instead of the constant-M0 division
  int psi_stop = 0;          // 0: Krylov.jl's stop on ||M^-1 r|| (the reference); 1: on the true residual ||b - A x||
  int psi_check = 0;         // 1: measure ||b - A x|| / ||b|| of every psi system after each solve
};

struct StepStatus {
  int err_flags = 0;        // 1,2,4: W_i + C_i < 0
  int psi_systems = 0;
  int psi_max_iters = 0;
  int psi_not_converged = 0;
  double psi_max_rnorm_rel = 0.0;
};

class SolverBase {
 public:
  virtual ~SolverBase() {}
  virtual void set_field(int level, int fid, const void* host, int is_device) = 0;
  virtual void get_field(int level, int fid, void* host) = 0;
  // float32 frames for headless visualisation (what: 0 phi sum per run, 1 speed per run, 100 + field id)
  virtual void export_f32(int level, int what, float* host) = 0;
  virtual void set_scalars(int level, const double* q4 /* [R][4] Q,R1,R2,R3 */) = 0;
  virtual void get_scalars(int level, double* q4) = 0;
  virtual void set_dt(const double* dt) = 0;
  virtual void get_dt(double* dt) = 0;
  virtual void set_A0(const double* a0) = 0;
  virtual void get_A0(double* a0) = 0;
  virtual void init_state(int hats_given) = 0;
  // seeded-shape initial phi/psi on the device (2D), u = p = 0, then init_state
  virtual void init_shapes2d(const struct Shape2D* shapes) = 0;
  virtual void init_reference_shapes(int state_type, int goal, const double* blob_u) = 0;
  virtual void step1(int n) = 0;
  virtual void step2(int n) = 0;
  virtual void step3() = 0;
  virtual void step4(int n) = 0;
  virtual void step5(int n) = 0;
  virtual void step6() = 0;
  virtual void step7(int n) = 0;
  virtual void update_state() = 0;
  virtual void monitor(double* energy, double* aratio) = 0;
  // one whole time step (Steps 1-7, update, optional monitor) replayed from a CUDA graph
  // captured on first use; false if this handle runs steps eagerly
  virtual bool step_graph(int n, double* energy, double* aratio) = 0;
  virtual void get_work(int what, int idx, void* host) = 0;
  virtual void get_scalar_work(int what, double* out) = 0;
  virtual void transform(int kind, int nf, const double* in, double* out) = 0;
  virtual StepStatus status() = 0;
  virtual void sync() = 0;
  virtual void profile(int enable) = 0;
  virtual void profile_read(int cls, double* out3) = 0;
  virtual cudaStream_t stream() = 0;
  // learned psi preconditioner: packed mma fragments + biases (net_pack) and
  // the tcgen05 kernel's B-operand image (net_pack_tc)
  virtual void set_psi_net(const uint32_t* frags, const float* bias, const uint16_t* timg) = 0;
  // snapshots of the psi BiCGSTAB iterates (training data of the network)
  virtual void harvest(int cap) = 0;
  virtual long long harvest_read(float* out, long long cap, int* nsnap) = 0;
  // the FFT kernel variants this handle uses (JSON text)
  virtual std::string tuning() = 0;
};

struct Dims {
  int nd, Nx, Ny, Nz, V, R;
  double Lx, Ly, Lz;
};

static __global__ void k_copy_mmax(const double* sch, double* mm, int R) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < R) mm[r] = sch[r * 8 + 3];
  }

static __global__ void k_set_adt(const double* dt, double a, double* adt, int R) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < R) adt[r] = a / dt[r];
  }

static __global__ void k_area0(const double* asum, double cell, double* A0, int V) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < V) A0[v] = asum[v] * cell;
  }

static __global__ void k_init_scalars(const double* sch, double* s, int R) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < R) { s[r * 4 + 0] = 1.0; s[r * 4 + 1] = sch[r * 8 + 0]; s[r * 4 + 2] = sch[r * 8 + 1]; s[r * 4 + 3] = sch[r * 8 + 2]; }
  }

// Condition of a Krylov WHILE node of a captured time step: 1 while any
// system is active.  Bounded: after itmax + 1 evaluations the loop stops
// whatever the flags say (and flags the overrun in *err, bit 3).
static __global__ void k_loop_cond(cudaGraphConditionalHandle hnd, const BiState* st_, int S, unsigned* trips, int limit,
                            int* err) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int any = 0;
  for (int s = 0; s < S; ++s) any |= st_[s].active;
  const unsigned t = ++(*trips);
  if (any && (int)t > limit) { any = 0; atomicOr(err, 8); }
  cudaGraphSetConditional(hnd, any ? 1u : 0u);
}

static __global__ void k_bi_flags(const BiState* st_, int* upd, int S) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < S) upd[s] = st_[s].active;
  }

template <typename T>
__global__ void k_import_real(const double* src, T* dst, int Fo, int Fi, long long P, int dir) {
    long long tot = (long long)Fo * Fi * P;
    K_LOOP(tot, i) {
      long long p = i % P, f = i / P;
      int o = (int)(f / Fi), in = (int)(f % Fi);
      long long d = ((long long)in * Fo + o) * P + p;
      if (dir == 0) dst[d] = (T)src[i]; else ((double*)src)[i] = (double)dst[d];
    }
  }

template <typename T>
__global__ void k_import_hat(const double* src, cplx<T>* dst, int Fo, int Fi, long long rows, int nkx, int kp, int dir) {
    long long tot = (long long)Fo * Fi * rows * nkx;
    K_LOOP(tot, i) {
      int kx = (int)(i % nkx);
      long long rr = i / nkx;
      long long row = rr % rows, f = rr / rows;
      int o = (int)(f / Fi), in = (int)(f % Fi);
      long long d = (((long long)in * Fo + o) * rows + row) * kp + kx;
      if (dir == 0) { cplx<T> z; z.x = (T)src[2 * i]; z.y = (T)src[2 * i + 1]; dst[d] = z; }
      else { ((double*)src)[2 * i] = (double)dst[d].x; ((double*)src)[2 * i + 1] = (double)dst[d].y; }
    }
  }


// ---------------------------------------------------------------------------
// per-kernel-class timing: CUDA events around every launch of the class on the
// handle's stream, plus the algorithmic bytes of each launch (inputs read once
// + outputs written once).  Off unless enabled.
// ---------------------------------------------------------------------------
enum KClass : int { KC_COLS = 0, KC_ROWS_R2C, KC_ROWS_C2R, KC_ROWS_C2C, KC_ROWS_MUL, KC_PSI_VEC, KC_POINTWISE, KC_NET,
                    KC_COLS_F32, KC_N };

struct Prof {
  bool on = false;
  std::vector<cudaEvent_t> ev;
  std::vector<std::pair<int, double>> rec;   // (class, bytes) per event pair
  double ms[KC_N] = {0}, bytes[KC_N] = {0};
  long long launches[KC_N] = {0};
  void enable(bool e) {
    on = e;
    if (e && ev.empty()) {
      ev.resize(2 * 16384);
      for (auto& x : ev) VSAV_CUDA(cudaEventCreate(&x));
    }
  }
  void begin(cudaStream_t st) {
    if (!on) return;
    if (2 * rec.size() + 2 > ev.size()) throw std::runtime_error("profiler event pool exhausted; collect more often");
    VSAV_CUDA(cudaEventRecord(ev[2 * rec.size()], st));
  }
  void end(cudaStream_t st, int cls, double b) {
    if (!on) return;
    VSAV_CUDA(cudaEventRecord(ev[2 * rec.size() + 1], st));
    rec.push_back({cls, b});
  }
  void collect() {
    for (size_t i = 0; i < rec.size(); ++i) {
      VSAV_CUDA(cudaEventSynchronize(ev[2 * i + 1]));
      float t = 0;
      VSAV_CUDA(cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]));
      ms[rec[i].first] += t; bytes[rec[i].first] += rec[i].second; launches[rec[i].first] += 1;
    }
    rec.clear();
  }
  void reset() { collect(); for (int k = 0; k < KC_N; ++k) { ms[k] = 0; bytes[k] = 0; launches[k] = 0; } }
  ~Prof() { for (auto& x : ev) cudaEventDestroy(x); }
};

template <typename B> __device__ __forceinline__ B conv_to(double a) { return (B)a; }
template <typename B> __device__ __forceinline__ B conv_to(float a) { return (B)a; }
template <typename B> __device__ __forceinline__ B conv_to(double2 a);
template <typename B> __device__ __forceinline__ B conv_to(float2 a);
template <> __device__ __forceinline__ float2 conv_to<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> __device__ __forceinline__ double2 conv_to<double2>(float2 a) { return make_double2(a.x, a.y); }
template <typename A, typename B>
__global__ void k_cast(const A* __restrict__ x, B* __restrict__ y, long long n) {
  K_LOOP(n, i) y[i] = conv_to<B>(x[i]);
}
// y += x   (x in the other precision)
template <typename A, typename B>
__global__ void k_add_cast(const A* __restrict__ x, B* __restrict__ y, long long n) {
  K_LOOP(n, i) y[i] = y[i] + conv_to<B>(x[i]);
}
// r = b - y
template <typename T>
__global__ void k_sub(const T* __restrict__ b, const T* __restrict__ y, T* __restrict__ r, long long n) {
  K_LOOP(n, i) r[i] = b[i] - y[i];
}

template <typename T> class Solver;

// A 2D vesicle shape: boundary radius R(theta) = a b / sqrt((b cos)^2 + (a sin)^2)
// + sum_k amp_k cos(m_k theta + phase_k) in the frame rotated by rot about
// (cx, cy); phi = tanh((R - r) / (sqrt(2) eps)), psi = psi_in (1+phi)/2 + psi_out (1-phi)/2
// (the tanh profile of Init.jl:113).
struct Shape2D {
  double cx, cy, a, b, rot, psi_in, psi_out;
  int nmodes;
  int m[8];
  double amp[8], phase[8];
};

template <typename T>
__global__ void k_shapes2d(T* __restrict__ phi, T* __restrict__ psi, const Shape2D* __restrict__ sh, int V, int Nx, int Ny,
                           double Lx, double Ly, double eps) {
  const long long P = (long long)Nx * Ny, tot = (long long)V * P;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot; k += (long long)gridDim.x * blockDim.x) {
    const int v = (int)(k / P);
    const long long q = k - (long long)v * P;
    const int j = (int)(q / Nx), i = (int)(q - (long long)j * Nx);
    const Shape2D s = sh[v];
    const double x = -0.5 * Lx + Lx * i / Nx - s.cx, y = -0.5 * Ly + Ly * j / Ny - s.cy;
    const double cr = cos(s.rot), sr = sin(s.rot);
    const double xr = cr * x + sr * y, yr = -sr * x + cr * y;
    const double th = atan2(yr, xr), r = hypot(xr, yr);
    const double bc = s.b * cos(th), as = s.a * sin(th);
    double R = s.a * s.b / sqrt(bc * bc + as * as);
    for (int k2 = 0; k2 < s.nmodes; ++k2) R += s.amp[k2] * cos(s.m[k2] * th + s.phase[k2]);
    const double p = tanh((R - r) / (1.4142135623730951 * eps));
    phi[k] = (T)p;
    psi[k] = (T)(s.psi_in * (1 + p) / 2 + s.psi_out * (1 - p) / 2);
  }
}

// Frames for headless visualisation, as float32 (the arrays the reference's plots
// draw, scripts/visualize.jl): per run r, phi_plot = sum of the run's vesicle
// fields + N_r - 1 (simulation.jl:124, Main.jl:119), or the speed |u|
// (visualize.jl:71-73).  out: [R][P].
template <typename T>
__global__ void k_export_run(const T* __restrict__ phi, const T* __restrict__ u, const int* __restrict__ vbeg, int what,
                             int R, int nd, long long P, float* __restrict__ out) {
  const long long tot = (long long)R * P;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot; k += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(k / P);
    const long long q = k - (long long)r * P;
    double s = 0.0;
    if (what == 0) {
      const int v0 = vbeg[r], v1 = vbeg[r + 1];
      for (int v = v0; v < v1; ++v) s += (double)phi[(long long)v * P + q];
      s += (double)(v1 - v0) - 1.0;
    } else {
      for (int d = 0; d < nd; ++d) { const double c = (double)u[((long long)d * R + r) * P + q]; s += c * c; }
      s = sqrt(s);
    }
    out[k] = (float)s;
  }
}
template <typename T>
__global__ void k_to_f32(const T* __restrict__ in, float* __restrict__ out, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    out[k] = (float)in[k];
}

// One vesicle field of the reference's generate_initial_condition (Init.jl:74-197,
// Init_3d.jl:67-137), resolved on the host from (state_type, goal, N of the run):
// the shape kind, its centre and constants, psi = alpha phi + beta (Init.jl:191-197).
enum { RS_ZERO = 0, RS_ELLIPSE, RS_TRIANGLE, RS_STAR, RS_BLOB, RS_ELLIPSOID };
struct RefShape {
  int kind;
  double cx, cy, cz;
  double R0, amp;                    // ELLIPSE/ELLIPSOID: R; TRIANGLE: radius; STAR/BLOB: R0, amplitude
  double alpha, beta;
  double an[10], pn[10];             // BLOB: R(theta) = R0 + sum_k an_k R0 cos(k theta + pn_k)
};

// The grid is x_i = i dx from 0 (range(0, Lx - dx, length=Nx), Init.jl:80-83);
// angles are Julia's atan(X - cx, Y - cy) = atan2(dx, dy), measured from the y axis.
template <typename T>
__global__ void k_ref_shapes(T* __restrict__ phi, T* __restrict__ psi, const RefShape* __restrict__ sh, int V, int Nx,
                             int Ny, int Nz, double dx, double dy, double dz, double eps) {
  const long long NxNy = (long long)Nx * Ny, P = NxNy * Nz, tot = (long long)V * P;
  const double den = 1.4142135623730951 * eps;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot; k += (long long)gridDim.x * blockDim.x) {
    const int v = (int)(k / P);
    const long long q = k - (long long)v * P;
    const int l = (int)(q / NxNy);
    const long long q2 = q - (long long)l * NxNy;
    const int j = (int)(q2 / Nx), i = (int)(q2 - (long long)j * Nx);
    const RefShape& s = sh[v];
    const double X = i * dx - s.cx, Y = j * dy - s.cy;
    double p = 0.0;
    switch (s.kind) {
      case RS_ELLIPSE: {                         // Init.jl:107-110
        const double dist = sqrt(X * X / 2 + Y * Y);
        p = tanh((s.R0 - dist) / den);
        break;
      }
      case RS_TRIANGLE: {                        // Init.jl:112-127: smoothed max of three half-planes
        const double ks = sqrt(3.0) / 2, kc = 0.5, sm = 40.0;
        const double d1 = -Y, d2 = ks * X + kc * Y, d3 = -ks * X + kc * Y;
        const double mx = fmax(d1, fmax(d2, d3));
        const double ds = mx + (1 / sm) * log(exp(sm * (d1 - mx)) + exp(sm * (d2 - mx)) + exp(sm * (d3 - mx)));
        p = -tanh((ds - s.R0 / 3) / den);
        break;
      }
      case RS_STAR: {                            // Init.jl:128-139, 167-185
        const double r = sqrt(X * X + Y * Y), th = atan2(X, Y);
        p = tanh((s.R0 + s.amp * cos(10 * th) - r) / den);
        break;
      }
      case RS_BLOB: {                            // Init.jl:140-160
        const double r = sqrt(X * X + Y * Y), th = atan2(X, Y);
        double R = s.R0;
        for (int m = 0; m < 10; ++m) R += s.an[m] * s.R0 * cos((m + 1) * th + s.pn[m]);
        p = tanh((R - r) / den);
        break;
      }
      case RS_ELLIPSOID: {                       // Init_3d.jl:103-106
        const double Z = l * dz - s.cz;
        const double dist = sqrt(X * X / 2 + Y * Y / 2 + Z * Z);
        p = tanh((s.R0 - dist) / den);
        break;
      }
      default: break;
    }
    phi[k] = (T)p;
    psi[k] = (T)(s.alpha * p + s.beta);
  }
}

// Book-keeping of one step-graph capture: the kernels captured outside the
// Krylov loops, and per loop (a WHILE node) the kernels of its body and the
// device counter of its evaluated conditions (1 + iterations).
struct CaptureCtx {
  long long fixed = 0;
  std::vector<long long> body;
  unsigned* d_trips = nullptr;     // [kMaxLoops]
  cudaStream_t side = nullptr;     // stream the loop bodies are captured on
  int* err = nullptr;              // error flags of the handle that owns the capture
  static constexpr int kMaxLoops = 16;
};
inline CaptureCtx*& capture_ctx() { static thread_local CaptureCtx* c = nullptr; return c; }

template <typename T>
class Solver : public SolverBase {
 public:
  using C = cplx<T>;
  Geom g{};
  Phys ph{};
  Options opt;
  Dims dm;
  cudaStream_t st = nullptr;
  std::vector<void*> allocs;
  // device bookkeeping
  int *d_run_of = nullptr, *d_vbeg = nullptr;
  double *d_psi_in = nullptr, *d_psi_out = nullptr;
  std::vector<int> h_run_sizes;
  Runs rn{};
  C* tab = nullptr;
  // state levels
  T* phys4[2]; C* hat4[2]; T* uphys[2]; C* uhat[2]; double* sc[2];
  double *d_dt, *d_A0, *d_adt;
  // step-1 work
  T *phis, *psis, *Mpsi, *ustar, *d4, *omega, *lapomega, *H4, *gG, *gstar, *adv;
  C *tmpH, *tmpH2, *Hh, *flh, *advh, *cache, *rhs, *s3, *uth;
  T *cphys, *mn, *gu, *gmu, *gnu, *conv, *coupl, *rhs2, *utp, *tmpP, *mon_lap, *mon_g4, *mon_ga, *mon_gp;
  double *scH, *factor, *area, *mmax_v, *mmax_r, *fd, *fd2, *r2, *qv, *theta, *energy, *aratio, *asum;
  double2* part;
  int* d_err;
  // psi solver
  C *vb = nullptr, *vx = nullptr, *vr = nullptr, *vp = nullptr, *vv = nullptr, *vs = nullptr, *vt = nullptr, *vt12 = nullptr;
  C *vph = nullptr, *vsh = nullptr;          // preconditioned directions (flexible BiCGSTAB)
  uint32_t* nfrag = nullptr;                 // learned preconditioner weights (mma fragments)
  float *nbias = nullptr, *inv_s = nullptr;
  bool net_ok = false;
  uint4* ntimg = nullptr;                    // the same weights as tcgen05 B operands
  int net_sms = 1;                           // SMs of the device: the persistent tcgen05 grid
  int net_impl = 1;                          // network kernel: 1 k_net_apply (mma.sync), 2 k_net_apply_tc (tcgen05)
  float* hv = nullptr;                       // harvested iterates
  int hv_cap = 0, hv_count = 0;
  BiState* bst = nullptr; int *bupd = nullptr, *d_any = nullptr;
  double* d_true_res = nullptr;     // [3R] measured ||b - A x|| / ||b|| of the last psi solves (psi_check)
  int* h_pinned_any = nullptr;
  StepStatus last;
  double* stage = nullptr;   // host-format staging
  size_t stage_bytes = 0;
  double cur_a = 1, cur_b = -1, cur_c = 0;
  Prof prof;
  bool own_stream = true;
  // run on another solver's stream (the mixed-precision psi helper)
  void adopt_stream(cudaStream_t s2) {
    VSAV_CUDA(cudaStreamSynchronize(st));
    if (own_stream) VSAV_CUDA(cudaStreamDestroy(st));
    st = s2; own_stream = false;
  }

  template <typename X> X* dalloc(size_t n) {
    void* p = nullptr;
    VSAV_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(X)));
    VSAV_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(X), st));
    allocs.push_back(p);
    return (X*)p;
  }

  static int ilog2(int n) { int l = 0; while ((1 << l) < n) ++l; return l; }

  Solver(const Dims& d, const Phys& p, const Options& o, const int* run_sizes, const double* psi_in, const double* psi_out)
      : ph(p), opt(o), dm(d) {
    VSAV_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (const char* env = getenv("VSAV_PSI_FUSED")) fused_ops = atoi(env) != 0;
    if (const char* env = getenv("VSAV_PSI_CHUNK_MB")) psi_chunk_mb = atoll(env);
    // VSAV_GRAPH=0 runs every step eagerly (kernel-level profilers see each launch)
    if (const char* env = getenv("VSAV_GRAPH")) if (atoi(env) == 0) opt.graph = 0;
    g.nd = d.nd; g.Nx = d.Nx; g.Ny = d.Ny; g.Nz = (d.nd == 3) ? d.Nz : 1;
    g.nkx = d.Nx / 2 + 1;
    g.kp = (g.nkx + 15) / 16 * 16;
    g.P = (long long)g.Nz * g.Ny * g.Nx;
    g.H = (long long)g.Nz * g.Ny * g.kp;
    g.Pfull = (long long)g.Nz * g.Ny * g.Nx;
    g.kxs = 2 * M_PI / d.Lx; g.kys = 2 * M_PI / d.Ly; g.kzs = (d.nd == 3) ? 2 * M_PI / d.Lz : 0.0;
    const int V = d.V, R = d.R, nd = d.nd;
    // runs
    std::vector<int> run_of(V), vbeg(R + 1);
    int v = 0;
    for (int r = 0; r < R; ++r) { vbeg[r] = v; for (int k = 0; k < run_sizes[r]; ++k) run_of[v++] = r; }
    vbeg[R] = v;
    if (v != V) throw std::runtime_error("run sizes do not add up to the number of vesicle fields");
    h_run_sizes.assign(run_sizes, run_sizes + R);
    d_run_of = dalloc<int>(V); d_vbeg = dalloc<int>(R + 1);
    d_psi_in = dalloc<double>(V); d_psi_out = dalloc<double>(V);
    VSAV_CUDA(cudaMemcpyAsync(d_run_of, run_of.data(), V * sizeof(int), cudaMemcpyHostToDevice, st));
    VSAV_CUDA(cudaMemcpyAsync(d_vbeg, vbeg.data(), (R + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
    VSAV_CUDA(cudaMemcpyAsync(d_psi_in, psi_in, V * sizeof(double), cudaMemcpyHostToDevice, st));
    VSAV_CUDA(cudaMemcpyAsync(d_psi_out, psi_out, V * sizeof(double), cudaMemcpyHostToDevice, st));
    rn.V = V; rn.R = R; rn.run_of = d_run_of; rn.vbeg = d_vbeg; rn.psi_in = d_psi_in; rn.psi_out = d_psi_out;
    // twiddles: tab[n + m] = exp(-2 pi i m / n), n = 1..2^k
    int nmax = std::max(g.Nx, std::max(g.Ny, g.Nz));
    std::vector<C> ht(2 * nmax);
    for (int n = 1; n <= nmax; n <<= 1)
      for (int m = 0; m < n; ++m) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
        // exact values at the quarter points
        long double cr = cosl(a), ci = sinl(a);
        if (4 * m % n == 0) { int q = 4 * m / n; cr = (q == 0) ? 1 : (q == 2 ? -1 : 0); ci = (q == 1) ? -1 : (q == 3 ? 1 : 0); }
        ht[n + m] = mk<C>((double)cr, (double)ci);
      }
    tab = dalloc<C>(2 * nmax);
    VSAV_CUDA(cudaMemcpyAsync(tab, ht.data(), ht.size() * sizeof(C), cudaMemcpyHostToDevice, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
    const long long VP = (long long)V * g.P, VH = (long long)V * g.H, RP = (long long)R * g.P, RH = (long long)R * g.H;
    (void)VH;
    for (int l = 0; l < 2; ++l) {
      phys4[l] = dalloc<T>(4 * VP); hat4[l] = dalloc<C>(4 * VH);
      uphys[l] = dalloc<T>((nd + 1) * RP); uhat[l] = dalloc<C>((nd + 1) * RH);
      sc[l] = dalloc<double>(4 * R);
    }
    d_dt = dalloc<double>(R); d_A0 = dalloc<double>(V); d_adt = dalloc<double>(R);
    phis = dalloc<T>(VP); psis = dalloc<T>(VP); Mpsi = dalloc<T>(VP); ustar = dalloc<T>(nd * RP);
    d4 = dalloc<T>(4 * VP); omega = dalloc<T>(VP); lapomega = dalloc<T>(VP); H4 = dalloc<T>(4 * VP);
    gG = dalloc<T>(3 * VP); gstar = dalloc<T>(2 * nd * VP); adv = dalloc<T>(2 * VP);
    long long tmpf = std::max<long long>(8 * V, 9 * R);
    tmpH = dalloc<C>(tmpf * g.H); tmpH2 = dalloc<C>(V * g.H); Hh = dalloc<C>(4 * VH); flh = dalloc<C>(3 * VH);
    advh = dalloc<C>(2 * VH); cache = dalloc<C>(16 * VH); rhs = dalloc<C>(3 * VH); s3 = dalloc<C>(8 * VH);
    uth = dalloc<C>(2 * nd * RH);
    cphys = dalloc<T>(8 * VP); mn = dalloc<T>(4 * VP); gu = dalloc<T>(nd * nd * RP); gmu = dalloc<T>(nd * VP);
    gnu = dalloc<T>(nd * VP); conv = dalloc<T>(nd * RP); coupl = dalloc<T>(nd * RP); rhs2 = dalloc<T>(nd * RP);
    utp = dalloc<T>(2 * nd * RP); tmpP = dalloc<T>(3 * VP);
    mon_lap = dalloc<T>(2 * VP); mon_g4 = dalloc<T>(4 * VP); mon_ga = dalloc<T>(2 * VP); mon_gp = dalloc<T>(2 * RP);
    scH = dalloc<double>(8 * R); factor = dalloc<double>(V); area = dalloc<double>(V); asum = dalloc<double>(V);
    mmax_v = dalloc<double>(V); mmax_r = dalloc<double>(R);
    fd = dalloc<double>(3 * V * 32 + R * 32); fd2 = dalloc<double>(3 * V * 32 + R * 32);
    r2 = dalloc<double>(6 * R); qv = dalloc<double>(R); theta = dalloc<double>(2 * R);
    energy = dalloc<double>(R); aratio = dalloc<double>(R);
    long long nmaxe = std::max<long long>(g.Pfull, g.H);
    long long bpf = (nmaxe + 2047) / 2048;
    part = dalloc<double2>(bpf * std::max(3 * V, R) * 32);
    d_err = dalloc<int>(1);
    if (nd == 2 || opt.psi3d_var) {
      long long n = psi_n();
      if (nd == 3 && (!psi_full() || opt.psi_precond != 0))
        throw std::runtime_error("the 3D variable-mobility psi solve is the full-spectrum, diagonal-preconditioned form");
      vb = dalloc<C>(3 * V * n); vr = dalloc<C>(3 * V * n); vp = dalloc<C>(3 * V * n);
      vv = dalloc<C>(3 * V * n); vs = dalloc<C>(3 * V * n); vt = dalloc<C>(3 * V * n);
      vt12 = dalloc<C>((nd == 3 ? 9 : 6) * V * n);
      vx = psi_full() ? dalloc<C>(3 * V * n) : nullptr;
      bst = dalloc<BiState>(3 * R); bupd = dalloc<int>(3 * R); d_any = dalloc<int>(1);
      d_true_res = dalloc<double>(3 * R);
      VSAV_CUDA(cudaMemsetAsync(d_true_res, 0, 3 * R * sizeof(double), st));
      VSAV_CUDA(cudaMallocHost(&h_pinned_any, sizeof(int)));
      if (opt.psi_precond < 0 || opt.psi_precond > 2) throw std::runtime_error("psi_precond must be 0, 1 or 2");
      if (opt.psi_precond >= 1 && !opt.psi_mixed) {
        vph = dalloc<C>(3 * V * n); vsh = dalloc<C>(3 * V * n);
      }
      if (opt.psi_precond == 2 && !opt.psi_mixed) {
        if (!std::is_same<T, float>::value)
          throw std::runtime_error("the learned psi preconditioner runs in the FP32 psi solve (precision fp32 or mixed)");
        if (!psi_full()) throw std::runtime_error("the learned psi preconditioner needs the full-spectrum psi form");
        if (g.Nx < NA_T || g.Ny < NA_T) throw std::runtime_error("the learned psi preconditioner needs Nx, Ny >= 32");
        nfrag = dalloc<uint32_t>(NF_WORDS); nbias = dalloc<float>(NF_BIAS); inv_s = dalloc<float>(3 * V);
        ntimg = dalloc<uint4>(NT_WBYTES / 16);
        VSAV_CUDA(cudaFuncSetAttribute(k_net_apply<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, NA_SMEM));
        VSAV_CUDA(net_tc_attributes<1>());
        // VSAV_NET_TC=1 selects the tcgen05 kernel (read once, for this handle's life); the
        // mma.sync kernel is the default: at 16 channels a tcgen05.mma (M 128, N 16, K 16)
        // is issue-bound, so the warp-level MMAs of eight warps finish the layer sooner
        if (const char* env = getenv("VSAV_NET_TC")) net_impl = atoi(env) != 0 ? 2 : 1;
        int dev = 0;
        VSAV_CUDA(cudaGetDevice(&dev));
        VSAV_CUDA(cudaDeviceGetAttribute(&net_sms, cudaDevAttrMultiProcessorCount, dev));
      }
    }
    long long nh = std::max<long long>(3LL * V, 2LL * R * nd) * std::max<long long>(g.P, (long long)g.Nz * g.Ny * g.nkx * 2);
    stage_bytes = nh * sizeof(double);
    stage = dalloc<double>(nh);
    VSAV_CUDA(cudaStreamSynchronize(st));
    autotune();
    // VSAV_PSI_SPLIT=0/1 overrides the autotuner's choice between the fused and the split
    // forward pass + combine; read once here, so it holds for this handle's whole life
    // (graph replays included) and is what the tuning record reports
    if (const char* env = getenv("VSAV_PSI_SPLIT")) split_comb = atoi(env) != 0;
    // VSAV_COLS_TMA overrides the choice of the TMA-fed field column pass (where eligible):
    // 0 off, 1 on (the tuned block shape, else the first usable one), 2 + v block shape v
    if (const char* env = getenv("VSAV_COLS_TMA")) {
      const int b = atoi(env);
      if (b >= 2) { cols_tma_var = b - 2; cols_tma = cols_tma_var_ok(cols_tma_var); }
      else {
        cols_tma = b != 0 && cols_tma_eligible();
        for (int v = CT_NV - 1; cols_tma && v >= 0; --v)
          if (!cols_tma_var_ok(cols_tma_var)) cols_tma_var = v;
      }
      if (!cols_tma) cols_tma_var = 0;
    }
    // VSAV_C2R_BULK=0/1 overrides the choice of the bulk-copy-fed c2r x pass (where eligible)
    if (const char* env = getenv("VSAV_C2R_BULK")) c2r_bulk = atoi(env) != 0 && c2r_bulk_shape();
    // VSAV_PSI_TMA=0/1 overrides the choice of the TMA-fed psi column passes (where eligible)
    if (const char* env = getenv("VSAV_PSI_TMA")) {
      tma_cols = atoi(env) != 0 && tma_eligible();
      for (int v = TMA_NV - 1; tma_cols && v >= 0; --v) {  // a usable variant where none was tuned
        if (!tma_var_ok(tma_var_inv2)) tma_var_inv2 = v;
        if (!tma_var_ok(tma_var_comb)) tma_var_comb = v;
      }
    }
    // VSAV_PSI_BULK overrides the choice of the bulk-copy-fed psi x pass (where eligible):
    // 0 off, 1 on (the tuned block shape, else the first usable one), 2 + v block shape v
    if (const char* env = getenv("VSAV_PSI_BULK")) {
      const int b = atoi(env);
      bulk_rows = b != 0 && bulk_eligible();
      if (b >= 2) bulk_var = b - 2;
      if (bulk_rows && !bulk_var_ok(bulk_var))
        for (int v = BR_NV - 1; v >= 0; --v)
          if (bulk_var_ok(v)) bulk_var = v;
      if (!bulk_rows) bulk_var = 0;
    }
    if constexpr (std::is_same<T, double>::value) {
      if (opt.psi_mixed && (nd == 2 || opt.psi3d_var)) {
        Options o2 = opt;
        o2.psi_mixed = 0;
        o2.psi_check = 0;            // the parent measures the FP64 residual after the sweeps
        std::vector<int> rs(dm.R);
        std::vector<double> pin(dm.V), pout(dm.V);
        VSAV_CUDA(cudaMemcpy(pin.data(), d_psi_in, dm.V * sizeof(double), cudaMemcpyDeviceToHost));
        VSAV_CUDA(cudaMemcpy(pout.data(), d_psi_out, dm.V * sizeof(double), cudaMemcpyDeviceToHost));
        for (int r = 0; r < dm.R; ++r) rs[r] = 0;
        for (int v2 = 0; v2 < dm.V; ++v2) rs[run_of[v2]]++;
        psi32 = new Solver<float>(dm, ph, o2, rs.data(), pin.data(), pout.data());
        psi32->adopt_stream(st);
      }
    }
  }

  ~Solver() override {
    cudaStreamSynchronize(st);
    if (hv) cudaFree(hv);
    for (auto& row : sgraph)
      for (auto& sg : row) {
        if (sg.exec) cudaGraphExecDestroy(sg.exec);
        if (sg.graph) cudaGraphDestroy(sg.graph);
      }
    if (side_st) cudaStreamDestroy(side_st);
    if (h_trips) cudaFreeHost(h_trips);
    if (psi32) { delete psi32; psi32 = nullptr; }
    if (own_stream == false) st = nullptr;
    for (void* p : allocs) cudaFree(p);
    if (h_pinned_any) cudaFreeHost(h_pinned_any);
    if (own_stream) cudaStreamDestroy(st);
  }

  bool psi_full() const { return opt.psi_form == 0; }
  long long psi_n() const { return psi_full() ? g.Pfull : g.H; }

  // ------------------------------------------------------------------ launch helpers
  EW ew(long long n) const {
    EW e; e.n = n; e.chunk = std::min<long long>(2048, n); e.bpf = (int)((n + e.chunk - 1) / e.chunk); return e;
  }
  // the Krylov vector passes of the psi solve (F fields of n slots): about eight
  // 256-thread blocks per SM in all, each streaming a long contiguous range of one
  // field (chunks of at least 2048 slots, a multiple of 1024), so the per-block
  // reduction of the dot partials is amortised over many elements
  EW ewv(long long n, int F) const {
    const long long want = std::max<long long>(1, (148LL * 8 + F - 1) / std::max(F, 1));
    long long chunk = (n + want - 1) / want;
    chunk = std::max<long long>(2048, (chunk + 1023) / 1024 * 1024);
    EW e; e.n = n; e.chunk = std::min<long long>(chunk, n); e.bpf = (int)((n + e.chunk - 1) / e.chunk); return e;
  }
  int gridfor(long long n, int bs = 256) const { long long b = (n + bs - 1) / bs; return (int)std::min<long long>(b, 148 * 16); }
  void fin(int K, int F, const EW& e, double* out) {
    k_fin_fields<<<F, 256, 0, st>>>(part, e.bpf, K, out); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }

  // ---- FFT kernel variants: (E elements per thread, NT threads per CTA) ----
  // The autotuner picks one variant per pass family at handle creation.
  // FAM_COLS: column passes of half spectra; FAM_COLS_PSI: of the full-spectrum
  // psi vectors (2D, 3V or 6V fields), tuned separately
  // FAM_PSI_INV2 / FAM_PSI_COMB: the fused column passes of the FULL psi operator
  // FAM_PSI_FWD2: the forward pass of the split alternative to FAM_PSI_COMB (with k_psi_combz)
  enum Fam { FAM_R2C = 0, FAM_C2R, FAM_C2C, FAM_MUL, FAM_COLS, FAM_COLS_PSI, FAM_PSI_INV2, FAM_PSI_COMB, FAM_PSI_FWD2,
             FAM_N };
  static constexpr int NVAR = 7;
  static constexpr int VE[2][NVAR] = {{8, 8, 16, 32, 8, 16, 32}, {4, 4, 8, 16, 4, 8, 16}};      // [T==double][variant]
  static constexpr int VNT[NVAR] = {256, 512, 256, 256, 1024, 512, 128};
  int choice[FAM_N] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  int split_comb = 0;            // 1: forward pass + combine as k_psi_cols_fwd2 + k_psi_combz (autotuned)
  bool tuned_from_cache = false;
  double tune_ms[FAM_N][NVAR] = {};
  static constexpr int DIX = std::is_same<T, double>::value ? 1 : 0;
  int vE(int v) const { return VE[DIX][v]; }

  void area_sums(const T* phi, const T* gx, const T* gy, const EW& e) {
    k_area<T><<<dim3(e.bpf, dm.V), 256, 0, st>>>(phi, gx, gy, ph, e, part); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    fin(1, dm.V, e, asum);
  }

  int rows_lognl(int L, int E, int NT, long long nrows, int cap_rows = 0) const {
    int nl = std::max(1, E * NT / L);
    while (nl > 1 && nl / 2 >= nrows) nl /= 2;
    if (cap_rows) while (nl > cap_rows) nl /= 2;
    return ilog2(nl);
  }
  size_t rows_smem(int L, int nl) const { return (size_t)(2 * nl * line_pitch(L) + nl) * sizeof(C); }

#define VSAV_DISPATCH(fam, ...)                                                          \
  switch (choice[fam]) {                                                                 \
    case 0: { constexpr int E_ = VE[DIX][0], NT_ = VNT[0]; __VA_ARGS__; } break;         \
    case 1: { constexpr int E_ = VE[DIX][1], NT_ = VNT[1]; __VA_ARGS__; } break;         \
    case 2: { constexpr int E_ = VE[DIX][2], NT_ = VNT[2]; __VA_ARGS__; } break;         \
    case 3: { constexpr int E_ = VE[DIX][3], NT_ = VNT[3]; __VA_ARGS__; } break;         \
    case 4: { constexpr int E_ = VE[DIX][4], NT_ = VNT[4]; __VA_ARGS__; } break;         \
    case 5: { constexpr int E_ = VE[DIX][5], NT_ = VNT[5]; __VA_ARGS__; } break;         \
    default: { constexpr int E_ = VE[DIX][6], NT_ = VNT[6]; __VA_ARGS__; } break;        \
  }

  template <int E_, int NT_>
  void set_smem_attr(const void* fn, size_t sm) {
    if (sm > 48 * 1024) VSAV_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  }

  void rows_r2c(const T* in0, const T* in1, double a0, double a1, C* out, long long nrows) {
    int L = g.Nx / 2, logL = ilog2(L);
    VSAV_DISPATCH(FAM_R2C, {
      int lognl = rows_lognl(L, E_, NT_, nrows);
      int nl = 1 << lognl;
      int thr = std::max(1, nl * L / E_);
      long long grid = (nrows + nl - 1) / nl;
      size_t sm = rows_smem(L, nl);
      set_smem_attr<E_, NT_>((const void*)k_rows_r2c<T, E_, NT_>, sm);
      prof.begin(st);
      k_rows_r2c<T, E_, NT_><<<(unsigned)grid, thr, sm, st>>>(in0, in1, (T)a0, (T)a1, out, logL, lognl, nrows, g.kp, tab); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      prof.end(st, KC_ROWS_R2C, (double)nrows * (g.Nx * sizeof(T) * (in1 ? 2 : 1) + g.nkx * sizeof(C)));
    })
  }
  void rows_c2r(const C* in, T* out, double scale, long long nrows) {
    if (c2r_bulk && c2r_bulk_ok(nrows)) { rows_c2r_bulk(in, out, scale, nrows); return; }
    int L = g.Nx / 2, logL = ilog2(L);
    VSAV_DISPATCH(FAM_C2R, {
      int lognl = rows_lognl(L, E_, NT_, nrows);
      int nl = 1 << lognl;
      int thr = std::max(1, nl * L / E_);
      long long grid = (nrows + nl - 1) / nl;
      size_t sm = rows_smem(L, nl);
      set_smem_attr<E_, NT_>((const void*)k_rows_c2r<T, E_, NT_>, sm);
      prof.begin(st);
      k_rows_c2r<T, E_, NT_><<<(unsigned)grid, thr, sm, st>>>(in, out, (T)scale, logL, lognl, nrows, g.kp, tab); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      prof.end(st, KC_ROWS_C2R, (double)nrows * (g.Nx * sizeof(T) + g.nkx * sizeof(C)));
    })
  }
  // ---- the bulk-copy-fed c2r x pass (k_rows_c2r_bulk, c2r_bulk.cuh): E 8 / 256 threads,
  // half-length rows L = Nx/2 = 256 .. 1024; autotuned against k_rows_c2r (FAM_C2R)
  static constexpr int CB_E = 8, CB_NT = 256;
  int c2r_bulk = 0;
  double c2r_bulk_ms = 0.0;
  int c2r_bulk_ctas = 0;
  bool c2r_bulk_shape() const {
    const int L = g.Nx / 2;
    return L >= 256 && L <= 1024 && L >= CB_E * CB_E && CB_E * CB_NT / L >= 1;
  }
  bool c2r_bulk_ok(long long nrows) const { return c2r_bulk_shape() && nrows % (CB_E * CB_NT / (g.Nx / 2)) == 0; }
  template <int LOGL>
  void launch_c2r_bulk(const C* in, T* out, double scale, long long nrows) {
    constexpr int L = 1 << LOGL, NL = CB_E * CB_NT / L;
    const long long nb = nrows / NL;
    const size_t smem = c2r_bulk_smem<T, CB_E, CB_NT, LOGL>(g.kp);
    const void* fn = (const void*)k_rows_c2r_bulk<T, CB_E, CB_NT, LOGL>;
    const int grid = (int)std::min<long long>(nb, tma_grid(fn, CB_NT, smem, c2r_bulk_ctas));
    prof.begin(st);
    k_rows_c2r_bulk<T, CB_E, CB_NT, LOGL><<<grid, CB_NT, smem, st>>>(in, out, (T)scale, nb, g.kp, tab, d_err);
    VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    prof.end(st, KC_ROWS_C2R, (double)nrows * (g.Nx * sizeof(T) + g.nkx * sizeof(C)));
  }
  void rows_c2r_bulk(const C* in, T* out, double scale, long long nrows) {
    if (!c2r_bulk_ok(nrows)) throw std::runtime_error("bulk c2r pass: unusable row count or length");
    switch (ilog2(g.Nx / 2)) {
      case 8: launch_c2r_bulk<8>(in, out, scale, nrows); break;
      case 9: launch_c2r_bulk<9>(in, out, scale, nrows); break;
      case 10: launch_c2r_bulk<10>(in, out, scale, nrows); break;
      default: throw std::runtime_error("bulk c2r pass: unsupported row length");
    }
  }
  template <bool INV>
  void rows_c2c(const C* in, const T* in_real, C* out, double scale, long long nrows) {
    int L = g.Nx, logL = ilog2(L);
    VSAV_DISPATCH(FAM_C2C, {
      int lognl = rows_lognl(L, E_, NT_, nrows);
      int nl = 1 << lognl;
      int thr = std::max(1, nl * L / E_);
      long long grid = (nrows + nl - 1) / nl;
      size_t sm = rows_smem(L, nl);
      set_smem_attr<E_, NT_>((const void*)k_rows_c2c<T, E_, NT_, INV>, sm);
      prof.begin(st);
      k_rows_c2c<T, E_, NT_, INV><<<(unsigned)grid, thr, sm, st>>>(in, in_real, out, (T)scale, logL, lognl, nrows, tab); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      prof.end(st, KC_ROWS_C2C, (double)nrows * g.Nx * ((in_real ? sizeof(T) : sizeof(C)) + sizeof(C)));
    })
  }
  // geo: 0 2D y (half), 1 3D z (half), 2 3D y (half), 3 2D y (full), 4 3D z (full), 5 3D y (full)
  ColArgs colargs(int geo, long long& nouter, int E, int NT) const {
    ColArgs a{};
    a.geo = geo; a.Nx = g.Nx; a.Ny = g.Ny; a.Nz = g.Nz; a.kp = g.kp;
    a.kxs = g.kxs; a.kys = g.kys; a.kzs = g.kzs;
    a.fkxs = (float)g.kxs; a.fkys = (float)g.kys; a.fkzs = (float)g.kzs;
    int L;
    if (geo == 0) { L = g.Ny; a.S = g.kp; a.W = g.kp; a.O = (long long)g.Ny * g.kp; a.kpv = g.kp; a.nkv = g.nkx; }
    else if (geo == 1) { L = g.Nz; a.S = g.Ny * g.kp; a.W = g.Ny * g.kp; a.O = g.H; a.kpv = g.kp; a.nkv = g.nkx; }
    else if (geo == 2) { L = g.Ny; a.S = g.kp; a.W = g.kp; a.O = (long long)g.Ny * g.kp; a.kpv = g.kp; a.nkv = g.nkx; nouter *= g.Nz; }
    else if (geo == 4) { L = g.Nz; a.S = g.Ny * g.Nx; a.W = g.Ny * g.Nx; a.O = g.Pfull; a.kpv = g.Nx; a.nkv = g.Nx; }
    else if (geo == 5) { L = g.Ny; a.S = g.Nx; a.W = g.Nx; a.O = (long long)g.Ny * g.Nx; a.kpv = g.Nx; a.nkv = g.Nx; nouter *= g.Nz; }
    else { L = g.Ny; a.S = g.Nx; a.W = g.Nx; a.O = (long long)g.Ny * g.Nx; a.kpv = g.Nx; a.nkv = g.Nx; }
    a.logL = ilog2(L);
    int TW = std::max(1, E * NT / L);
    while (TW > 1 && TW / 2 >= a.W) TW /= 2;
    a.TW = TW;
    a.logTW = ilog2(TW);
    a.tiles = (a.W + TW - 1) / TW;
    return a;
  }
  void cols(bool inv, int geo, long long nf, const C* in0, const C* in1, double a0, double a1, int mult, double ms,
            C* out, double oscale) {
    if (cols_tma && geo == 0 && g.nd == 2) {
      cols_tma_run(inv, nf, in0, in1, a0, a1, mult, ms, out, oscale, cols_tma_var);
      return;
    }
    VSAV_DISPATCH(geo == 3 ? FAM_COLS_PSI : FAM_COLS, {
      long long nouter = nf;
      ColArgs a = colargs(geo, nouter, E_, NT_);
      int L = 1 << a.logL;
      int thr = std::max(a.TW, a.TW * L / E_);
      size_t sm = 2 * (size_t)col_tile_elems(L, a.TW, ilog2(E_)) * sizeof(C);
      long long grid = (long long)a.tiles * nouter;
      long long valid_lines = (geo == 3 || geo == 5) ? (long long)g.Nx
                              : (geo == 4 ? (long long)g.Ny * g.Nx : (long long)g.nkx * (geo == 1 ? g.Ny : 1));
      double cb = (double)nouter * valid_lines * L * sizeof(C) * ((in1 ? 2 : 1) + 1);
      prof.begin(st);
      if (inv) {
        set_smem_attr<E_, NT_>((const void*)k_cols<T, E_, NT_, true>, sm);
        k_cols<T, E_, NT_, true><<<(unsigned)grid, thr, sm, st>>>(in0, in1, (T)a0, (T)a1, mult, ms, out, (T)oscale, a, tab);
      } else {
        set_smem_attr<E_, NT_>((const void*)k_cols<T, E_, NT_, false>, sm);
        k_cols<T, E_, NT_, false><<<(unsigned)grid, thr, sm, st>>>(in0, in1, (T)a0, (T)a1, mult, ms, out, (T)oscale, a, tab);
      }
      VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      prof.end(st, std::is_same<T, float>::value ? KC_COLS_F32 : KC_COLS, cb);
    })
  }
  void rows_mul(C* t, long long nrows, bool full, int f0 = 0, int fc = 0) {
    const int rpf = g.Nz * g.Ny;                          // rows of one field
    if (fc == 0) fc = (int)(nrows / (2 * rpf));
    if (full && bulk_rows && g.nd == 2 && nrows == 2LL * fc * g.Ny) { rows_mul_bulk(t, f0, fc); return; }
    int L = full ? g.Nx : g.Nx / 2, logL = ilog2(L);
    SysMap sm{dm.V, dm.R, d_run_of};
    int rowlen = full ? g.Nx : g.kp;
    VSAV_DISPATCH(FAM_MUL, {
      int lognl = rows_lognl(L, E_, NT_, nrows, g.Ny);
      int nl = 1 << lognl;
      int thr = std::max(1, nl * L / E_);
      long long grid = (nrows + nl - 1) / nl;
      size_t smb = rows_smem(L, nl);
      prof.begin(st);
      if (full) {
        set_smem_attr<E_, NT_>((const void*)k_rows_mul<T, E_, NT_, true>, smb);
        k_rows_mul<T, E_, NT_, true><<<(unsigned)grid, thr, smb, st>>>(t, Mpsi, (T)0, (T)(1.0 / g.P), logL, lognl, nrows,
                                                                       rowlen, rpf, sm, bupd, f0, fc, tab);
      } else {
        set_smem_attr<E_, NT_>((const void*)k_rows_mul<T, E_, NT_, false>, smb);
        k_rows_mul<T, E_, NT_, false><<<(unsigned)grid, thr, smb, st>>>(t, Mpsi, (T)0, (T)(1.0 / g.P), logL, lognl, nrows,
                                                                        rowlen, rpf, sm, bupd, f0, fc, tab);
      }
      VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      // reads + writes t1|t2 rows and reads M once per row
      prof.end(st, KC_ROWS_MUL, (double)nrows * ((full ? g.Nx : g.nkx) * 2.0 * sizeof(C) + g.Nx * sizeof(T)));
    })
  }

  // The bulk-copy-fed persistent form of the FULL x pass (k_rows_mul_bulk, FP32), in
  // three block shapes (E, threads, ring slots); the autotuner times them against the
  // classic kernel.  Row lengths 256 .. 2048 are compiled.
  static constexpr int BR_NV = 3;
  static constexpr int BR_E[BR_NV] = {16, 32, 32}, BR_NT[BR_NV] = {256, 128, 128}, BR_S[BR_NV] = {2, 2, 3};
  int bulk_rows = 0;              // 1: the psi x pass runs as k_rows_mul_bulk (autotuned)
  int bulk_var = 0;
  int bulk_ctas[BR_NV] = {0, 0, 0};
  bool bulk_var_ok(int v) const {
    const int L = g.Nx, E = BR_E[v], NL = BR_NT[v] * E / L;
    return v >= 0 && v < BR_NV && L >= 256 && L <= 2048 && L >= E * E && NL >= 1 && NL <= g.Ny;
  }
  bool bulk_eligible() const {
    if constexpr (!std::is_same<T, float>::value) return false;
    else {
      if (g.nd != 2 || !psi_full() || vt12 == nullptr) return false;
      for (int v = 0; v < BR_NV; ++v)
        if (bulk_var_ok(v)) return true;
      return false;
    }
  }
  template <int E_, int NT_, int S_, int LOGL>
  void launch_rows_bulk(C* t, int f0, int fc, int var) {
    if constexpr (std::is_same<T, float>::value) {
      using G = BulkRows<E_, NT_, LOGL, S_>;
      SysMap sm{dm.V, dm.R, d_run_of};
      const long long ntiles = 2LL * fc * (g.Ny / G::NL);
      const int grid = (int)std::min<long long>(ntiles, tma_grid((const void*)k_rows_mul_bulk<E_, NT_, LOGL, S_>, NT_,
                                                                  G::smem, bulk_ctas[var]));
      prof.begin(st);
      k_rows_mul_bulk<E_, NT_, LOGL, S_><<<grid, NT_, G::smem, st>>>(t, Mpsi, (float)(1.0 / g.P), g.Ny, fc, f0, ntiles, sm,
                                                                     bupd, tab, d_err);
      VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      prof.end(st, KC_ROWS_MUL, (double)2 * fc * g.Ny * (g.Nx * 2.0 * sizeof(C) + g.Nx * sizeof(T)));
    }
  }
  template <int LOGL>
  void rows_bulk_L(C* t, int f0, int fc, int var) {
    if constexpr (BulkRows<BR_E[0], BR_NT[0], LOGL, BR_S[0]>::ok)
      if (var == 0) { launch_rows_bulk<BR_E[0], BR_NT[0], BR_S[0], LOGL>(t, f0, fc, 0); return; }
    if constexpr (BulkRows<BR_E[1], BR_NT[1], LOGL, BR_S[1]>::ok)
      if (var == 1) { launch_rows_bulk<BR_E[1], BR_NT[1], BR_S[1], LOGL>(t, f0, fc, 1); return; }
    if constexpr (BulkRows<BR_E[2], BR_NT[2], LOGL, BR_S[2]>::ok)
      if (var == 2) { launch_rows_bulk<BR_E[2], BR_NT[2], BR_S[2], LOGL>(t, f0, fc, 2); return; }
    throw std::runtime_error("bulk x pass: block shape not compiled for this row length");
  }
  void rows_mul_bulk(C* t, int f0, int fc, int var = -1) {
    if (var < 0) var = bulk_var;
    if (!bulk_var_ok(var)) throw std::runtime_error("bulk x pass: block shape unusable at this size");
    switch (ilog2(g.Nx)) {
      case 8: rows_bulk_L<8>(t, f0, fc, var); break;
      case 9: rows_bulk_L<9>(t, f0, fc, var); break;
      case 10: rows_bulk_L<10>(t, f0, fc, var); break;
      case 11: rows_bulk_L<11>(t, f0, fc, var); break;
      default: throw std::runtime_error("bulk x pass: unsupported row length");
    }
  }

  // fused FULL-form operator column passes (fields f0 .. f0+fc-1; t1/t2 chunk-local)
  void psi_cols_inv2(const C* x, C* t1, C* t2, int f0, int fc, bool use_active = true) {
    SysMap sm{dm.V, dm.R, d_run_of};
    VSAV_DISPATCH(FAM_PSI_INV2, {
      long long nouter = fc;
      ColArgs a = colargs(3, nouter, E_, NT_);
      int L = 1 << a.logL;
      int thr = std::max(a.TW, a.TW * L / E_);
      size_t sm_b = 2 * (size_t)col_tile_elems(L, a.TW, ilog2(E_)) * sizeof(C);
      long long grid = (long long)a.tiles * fc;
      set_smem_attr<E_, NT_>((const void*)k_psi_cols_inv2<T, E_, NT_>, sm_b);
      prof.begin(st);
      k_psi_cols_inv2<T, E_, NT_><<<(unsigned)grid, thr, sm_b, st>>>(x, t1, t2, ph.S4, a, sm, use_active ? bupd : nullptr, f0, tab);
      VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      prof.end(st, std::is_same<T, float>::value ? KC_COLS_F32 : KC_COLS, (double)fc * g.Pfull * 3.0 * sizeof(C));
    })
  }
  void psi_cols_fwd2(C* t1, const C* t2, int f0, int fc, bool use_active = true) {
    SysMap sm{dm.V, dm.R, d_run_of};
    VSAV_DISPATCH(FAM_PSI_FWD2, {
      long long nouter = fc;
      ColArgs a = colargs(3, nouter, E_, NT_);
      int L = 1 << a.logL;
      int thr = std::max(a.TW, a.TW * L / E_);
      size_t sm_b = (2 * (size_t)col_tile_elems(L, a.TW, ilog2(E_)) + (size_t)L * a.TW) * sizeof(C);
      long long grid = (long long)a.tiles * fc;
      set_smem_attr<E_, NT_>((const void*)k_psi_cols_fwd2<T, E_, NT_>, sm_b);
      prof.begin(st);
      k_psi_cols_fwd2<T, E_, NT_><<<(unsigned)grid, thr, sm_b, st>>>(t1, t2, a, sm, use_active ? bupd : nullptr, f0, tab);
      VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      prof.end(st, KC_PSI_VEC, (double)fc * g.Pfull * 3.0 * sizeof(C));
    })
  }
  void psi_combz(const C* x, const C* z, C* y, int mode, const C* svec, const double* pre, int f0, int fc, const EW& e,
                 bool use_active = true) {
    SysMap sm{dm.V, dm.R, d_run_of};
    prof.begin(st);
    k_psi_combz<T><<<dim3(e.bpf, (unsigned)fc), 256, 0, st>>>(x, z, y, vb, svec, mode, d_adt, pre, ph.S4, vgeom(), sm,
                                                               use_active ? bupd : nullptr, f0, e, part); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    prof.end(st, KC_PSI_VEC, (double)fc * g.Pfull * 4.0 * sizeof(C));
  }
  // returns the number of dot partials per field (column tiles)
  int psi_cols_comb(const C* t1, const C* t2, const C* x, C* y, int mode, const C* svec, const double* pre, int f0, int fc,
                    bool use_active = true) {
    SysMap sm{dm.V, dm.R, d_run_of};
    int tiles = 0;
    VSAV_DISPATCH(FAM_PSI_COMB, {
      long long nouter = fc;
      ColArgs a = colargs(3, nouter, E_, NT_);
      int L = 1 << a.logL;
      int thr = std::max(a.TW, a.TW * L / E_);
      size_t sm_b = (2 * (size_t)col_tile_elems(L, a.TW, ilog2(E_)) + (size_t)L * a.TW) * sizeof(C);
      long long grid = (long long)a.tiles * fc;
      tiles = a.tiles;
      set_smem_attr<E_, NT_>((const void*)k_psi_cols_comb<T, E_, NT_>, sm_b);
      prof.begin(st);
      k_psi_cols_comb<T, E_, NT_><<<(unsigned)grid, thr, sm_b, st>>>(t1, t2, x, y, vb, svec, mode, d_adt, pre, ph.S4, a, sm,
                                                                      use_active ? bupd : nullptr, f0, tab, part);
      VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      prof.end(st, KC_PSI_VEC, (double)fc * g.Pfull * 5.0 * sizeof(C));
    })
    return tiles;
  }

  // ---- TMA-fed persistent column passes of the FULL psi operator (FP32) ----
  // One tile: TW = E * NT / (2 L) columns, t1 and t2 (or both directions) as 2 TW lines.
  // Two block shapes: variant 0 E 16 / NT 512 (tiles of 8192 elements: 4 columns at
  // L = 1024, one block per SM for the combine), variant 1 E 8 / NT 512 (tiles of 4096:
  // 2 columns, two blocks per SM); the autotuner picks one per pass.  Column lengths
  // L = 256 .. 2048 are compiled (tma_var_ok).
  // ---- the TMA-fed persistent y pass of the 2D half-spectrum field transforms
  // (k_cols_tma, cols_tma.cuh): two block shapes, both with 2-column tiles at
  // L = 1024 (E 16 / NT 128: three blocks per SM in FP64; E 8 / NT 256), column
  // lengths L = 256 .. 2048; autotuned against k_cols (the classic family FAM_COLS)
  static constexpr int CT_NV = 2;
  static constexpr int CT_E[CT_NV] = {16, 8}, CT_NT[CT_NV] = {128, 256};
  int cols_tma = 0, cols_tma_var = 0;
  double cols_tma_ms[CT_NV] = {0.0, 0.0};
  int cols_tma_ctas[2][2][CT_NV] = {};           // [inverse][inputs - 1][variant] resident blocks
  bool cols_tma_var_ok(int v) const {
    if (v < 0 || v >= CT_NV) return false;
    const int L = g.Ny, E = CT_E[v], TW = CT_E[v] * CT_NT[v] / L;
    return g.nd == 2 && L >= 256 && L <= 2048 && L >= E * E && TW >= 2 && TW <= 16 && g.kp % TW == 0;
  }
  bool cols_tma_eligible() const {
    for (int v = 0; v < CT_NV; ++v)
      if (cols_tma_var_ok(v)) return true;
    return false;
  }
  template <int E_, int NT_, int LOGL>
  static constexpr bool cols_tma_shape_ok() {
    constexpr int L = 1 << LOGL, TW = E_ * NT_ / L;
    return TW >= 2 && TW <= 16 && L >= E_ * E_;
  }
  // tensor map of nouter * Ny half-spectrum rows of kp complex values
  const CUtensorMap* tmap_half(const C* base, long long rows, int TW, int BH) {
    auto key = std::make_pair((const void*)base, -(rows * 4096 + TW * 512 + BH));
    auto it = tmaps.find(key);
    if (it == tmaps.end()) it = tmaps.emplace(key, make_tile_map(base, (int)sizeof(C), rows, g.kp, TW, BH)).first;
    return &it->second;
  }
  template <int E_, int NT_, int LOGL, bool INV, int NIN>
  void launch_cols_tma(long long nouter, const C* in0, const C* in1, double a0, double a1, int mult, double ms, C* out,
                       double oscale, int var) {
    constexpr int L = 1 << LOGL, TW = E_ * NT_ / L, BH = L < 256 ? L : 256;
    long long no = nouter;
    ColArgs a = colargs(0, no, E_, NT_);
    if (a.TW != TW) throw std::runtime_error("TMA field column pass: tile width mismatch");
    ColsTmaTiles tt;
    tt.per_field = (g.nkx + TW - 1) / TW;
    tt.total = (int)(tt.per_field * nouter);
    const size_t smem = cols_tma_smem<T, E_, NT_, LOGL, NIN>();
    const CUtensorMap* m0 = tmap_half(in0, nouter * g.Ny, TW, BH);
    const CUtensorMap* m1 = NIN == 2 ? tmap_half(in1, nouter * g.Ny, TW, BH) : m0;
    const void* fn = (const void*)k_cols_tma<T, E_, NT_, LOGL, INV, NIN>;
    const int grid = std::min(tt.total, tma_grid(fn, NT_, smem, cols_tma_ctas[INV ? 1 : 0][NIN - 1][var]));
    prof.begin(st);
    k_cols_tma<T, E_, NT_, LOGL, INV, NIN><<<grid, NT_, smem, st>>>(*m0, *m1, (T)a0, (T)a1, mult, ms, out, (T)oscale, a, tt,
                                                                    tab, d_err);
    VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    prof.end(st, std::is_same<T, float>::value ? KC_COLS_F32 : KC_COLS,
             (double)nouter * g.nkx * L * sizeof(C) * (NIN + 1));
  }
  template <int LOGL, bool INV, int NIN>
  void cols_tma_L(long long nf, const C* in0, const C* in1, double a0, double a1, int mult, double ms, C* out,
                  double oscale, int var) {
    if constexpr (cols_tma_shape_ok<CT_E[0], CT_NT[0], LOGL>())
      if (var == 0) { launch_cols_tma<CT_E[0], CT_NT[0], LOGL, INV, NIN>(nf, in0, in1, a0, a1, mult, ms, out, oscale, 0); return; }
    if constexpr (cols_tma_shape_ok<CT_E[1], CT_NT[1], LOGL>())
      if (var == 1) { launch_cols_tma<CT_E[1], CT_NT[1], LOGL, INV, NIN>(nf, in0, in1, a0, a1, mult, ms, out, oscale, 1); return; }
    throw std::runtime_error("TMA field column pass: block shape not compiled for this column length");
  }
  template <int LOGL>
  void cols_tma_I(bool inv, long long nf, const C* in0, const C* in1, double a0, double a1, int mult, double ms, C* out,
                  double oscale, int var) {
    if (inv) {
      if (in1) cols_tma_L<LOGL, true, 2>(nf, in0, in1, a0, a1, mult, ms, out, oscale, var);
      else cols_tma_L<LOGL, true, 1>(nf, in0, in1, a0, a1, mult, ms, out, oscale, var);
    } else {
      if (in1) cols_tma_L<LOGL, false, 2>(nf, in0, in1, a0, a1, mult, ms, out, oscale, var);
      else cols_tma_L<LOGL, false, 1>(nf, in0, in1, a0, a1, mult, ms, out, oscale, var);
    }
  }
  void cols_tma_run(bool inv, long long nf, const C* in0, const C* in1, double a0, double a1, int mult, double ms, C* out,
                    double oscale, int var) {
    if (!cols_tma_var_ok(var)) throw std::runtime_error("TMA field column pass: block shape unusable at this size");
    switch (ilog2(g.Ny)) {
      case 8: cols_tma_I<8>(inv, nf, in0, in1, a0, a1, mult, ms, out, oscale, var); break;
      case 9: cols_tma_I<9>(inv, nf, in0, in1, a0, a1, mult, ms, out, oscale, var); break;
      case 10: cols_tma_I<10>(inv, nf, in0, in1, a0, a1, mult, ms, out, oscale, var); break;
      case 11: cols_tma_I<11>(inv, nf, in0, in1, a0, a1, mult, ms, out, oscale, var); break;
      default: throw std::runtime_error("TMA field column pass: unsupported column length");
    }
  }

  static constexpr int TMA_NV = 2;
  static constexpr int TMA_VE[TMA_NV] = {16, 8}, TMA_VNT[TMA_NV] = {512, 512};
  int tma_cols = 0;               // 1: the psi column passes run as the TMA-fed kernels (autotuned)
  int tma_var_inv2 = 0, tma_var_comb = 0;
  int tma_ctas[2][TMA_NV] = {{0, 0}, {0, 0}};   // [pass][variant] resident blocks (persistent grid)
  std::map<std::pair<const void*, long long>, CUtensorMap> tmaps;
  // variant v usable at this size: the single-buffer FFT needs L >= E^2, a tile of
  // 2 <= TW <= 16 columns (16-byte TMA rows, lanes TW apart within a warp)
  bool tma_var_ok(int v) const {
    const int L = g.Ny, E = TMA_VE[v], TW = TMA_VE[v] * TMA_VNT[v] / (2 * L);
    return L >= E * E && L >= 256 && L <= 2048 && TW >= 2 && TW <= 16 && g.Nx % TW == 0;
  }
  bool tma_eligible() const {
    if constexpr (!std::is_same<T, float>::value) return false;
    else {
      if (g.nd != 2 || !psi_full() || vt12 == nullptr) return false;
      for (int v = 0; v < TMA_NV; ++v)
        if (tma_var_ok(v)) return true;
      return false;
    }
  }
  TmaTiles tma_tiles(int fc, int v) const {
    TmaTiles tt{};
    const int L = g.Ny;
    tt.TW = TMA_VE[v] * TMA_VNT[v] / (2 * L);
    tt.logTW = ilog2(tt.TW);
    tt.tiles = g.Nx / tt.TW;
    tt.total = fc * tt.tiles;
    tt.BH = std::min(L, 256);
    tt.nbox = L / tt.BH;
    return tt;
  }
  const CUtensorMap* tmap(const C* base, long long rows, int TW, int BH) {
    auto key = std::make_pair((const void*)base, rows * 4096 + TW * 512 + BH);
    auto it = tmaps.find(key);
    if (it == tmaps.end()) it = tmaps.emplace(key, make_tile_map(base, (int)sizeof(C), rows, g.Nx, TW, BH)).first;
    return &it->second;
  }
  int tma_grid(const void* fn, int nt, size_t smem, int& cache) {
    if (!cache) {
      VSAV_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      int per = 0, dev = 0, nsm = 0;
      VSAV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, nt, smem));
      VSAV_CUDA(cudaGetDevice(&dev));
      VSAV_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
      if (per < 1) throw std::runtime_error("TMA column pass does not fit on an SM");
      cache = per * nsm;
    }
    return cache;
  }
  template <int E_, int NT_, int LOGL>
  void launch_inv2_tma(const C* x, C* t1, C* t2, int f0, int fc, bool use_active, int var) {
    if constexpr (std::is_same<T, float>::value) {
      SysMap sm{dm.V, dm.R, d_run_of};
      long long nouter = fc;
      ColArgs a = colargs(3, nouter, E_, NT_);
      TmaTiles tt = tma_tiles(fc, var);
      const size_t smem = tma_col_smem(g.Ny, tt.TW, E_, 1);
      const CUtensorMap* mx = tmap(x, 3LL * dm.V * g.Ny, tt.TW, tt.BH);
      const int grid = std::min(tt.total, tma_grid((const void*)k_psi_cols_inv2_tma<E_, NT_, LOGL>, NT_, smem, tma_ctas[0][var]));
      prof.begin(st);
      k_psi_cols_inv2_tma<E_, NT_, LOGL><<<grid, NT_, smem, st>>>(*mx, t1, t2, ph.S4, a, tt, sm, use_active ? bupd : nullptr, f0,
                                                             tab, d_err);
      VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      prof.end(st, KC_COLS_F32, (double)fc * g.Pfull * 3.0 * sizeof(C));
    }
  }
  template <int E_, int NT_, int LOGL>
  int launch_comb_tma(const C* t1, const C* t2, const C* x, C* y, int mode, const C* svec, const double* pre, int f0,
                      int fc, bool use_active, int var) {
    if constexpr (std::is_same<T, float>::value) {
      SysMap sm{dm.V, dm.R, d_run_of};
      long long nouter = fc;
      ColArgs a = colargs(3, nouter, E_, NT_);
      TmaTiles tt = tma_tiles(fc, var);
      const size_t smem = tma_col_smem(g.Ny, tt.TW, E_, 4);
      const long long rows_g = 3LL * dm.V * g.Ny, rows_c = (long long)fc * g.Ny;
      const CUtensorMap* m1 = tmap(t1, rows_c, tt.TW, tt.BH);
      const CUtensorMap* m2 = tmap(t2, rows_c, tt.TW, tt.BH);
      const CUtensorMap* mx = tmap(x, rows_g, tt.TW, tt.BH);
      const CUtensorMap* mc = tmap(mode == 0 ? vb : svec, rows_g, tt.TW, tt.BH);
      const int grid = std::min(tt.total, tma_grid((const void*)k_psi_cols_comb_tma<E_, NT_, LOGL>, NT_, smem, tma_ctas[1][var]));
      prof.begin(st);
      k_psi_cols_comb_tma<E_, NT_, LOGL><<<grid, NT_, smem, st>>>(*m1, *m2, *mx, *mc, y, mode, d_adt, pre, ph.S4, a, tt, sm,
                                                             use_active ? bupd : nullptr, f0, tab, part, d_err);
      VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      prof.end(st, KC_PSI_VEC, (double)fc * g.Pfull * 5.0 * sizeof(C));
      return tt.tiles;
    }
    return 0;
  }
  // dispatch over the compiled column lengths and block shapes (only the shapes whose
  // tile is valid at that length are instantiated; tma_var_ok keeps the others unused)
  template <int E_, int NT_, int LOGL>
  static constexpr bool tma_shape_ok() {
    constexpr int L = 1 << LOGL, TW = E_ * NT_ / (2 * L);
    return TW >= 2 && TW <= 16 && L >= E_ * E_;
  }
  template <int LOGL>
  void inv2_tma_L(const C* x, C* t1, C* t2, int f0, int fc, bool use_active, int var) {
    if constexpr (tma_shape_ok<TMA_VE[0], TMA_VNT[0], LOGL>())
      if (var == 0) { launch_inv2_tma<TMA_VE[0], TMA_VNT[0], LOGL>(x, t1, t2, f0, fc, use_active, 0); return; }
    if constexpr (tma_shape_ok<TMA_VE[1], TMA_VNT[1], LOGL>())
      if (var == 1) { launch_inv2_tma<TMA_VE[1], TMA_VNT[1], LOGL>(x, t1, t2, f0, fc, use_active, 1); return; }
    throw std::runtime_error("TMA column pass: block shape not compiled for this column length");
  }
  template <int LOGL>
  int comb_tma_L(const C* t1, const C* t2, const C* x, C* y, int mode, const C* svec, const double* pre, int f0, int fc,
                 bool use_active, int var) {
    if constexpr (tma_shape_ok<TMA_VE[0], TMA_VNT[0], LOGL>())
      if (var == 0) return launch_comb_tma<TMA_VE[0], TMA_VNT[0], LOGL>(t1, t2, x, y, mode, svec, pre, f0, fc, use_active, 0);
    if constexpr (tma_shape_ok<TMA_VE[1], TMA_VNT[1], LOGL>())
      if (var == 1) return launch_comb_tma<TMA_VE[1], TMA_VNT[1], LOGL>(t1, t2, x, y, mode, svec, pre, f0, fc, use_active, 1);
    throw std::runtime_error("TMA column pass: block shape not compiled for this column length");
  }
  void psi_cols_inv2_tma(const C* x, C* t1, C* t2, int f0, int fc, bool use_active, int var = -1) {
    if (var < 0) var = tma_var_inv2;
    switch (ilog2(g.Ny)) {
      case 8: inv2_tma_L<8>(x, t1, t2, f0, fc, use_active, var); break;
      case 9: inv2_tma_L<9>(x, t1, t2, f0, fc, use_active, var); break;
      case 10: inv2_tma_L<10>(x, t1, t2, f0, fc, use_active, var); break;
      case 11: inv2_tma_L<11>(x, t1, t2, f0, fc, use_active, var); break;
      default: throw std::runtime_error("TMA column pass: unsupported column length");
    }
  }
  int psi_cols_comb_tma(const C* t1, const C* t2, const C* x, C* y, int mode, const C* svec, const double* pre, int f0,
                        int fc, bool use_active, int var = -1) {
    if (var < 0) var = tma_var_comb;
    switch (ilog2(g.Ny)) {
      case 8: return comb_tma_L<8>(t1, t2, x, y, mode, svec, pre, f0, fc, use_active, var);
      case 9: return comb_tma_L<9>(t1, t2, x, y, mode, svec, pre, f0, fc, use_active, var);
      case 10: return comb_tma_L<10>(t1, t2, x, y, mode, svec, pre, f0, fc, use_active, var);
      case 11: return comb_tma_L<11>(t1, t2, x, y, mode, svec, pre, f0, fc, use_active, var);
      default: throw std::runtime_error("TMA column pass: unsupported column length");
    }
  }

  // time every variant of every pass family on scratch buffers; keep the fastest
  // process-wide tuning cache: handles of the same shape reuse the first choice
  static std::map<std::string, std::vector<int>>& tune_cache() { static std::map<std::string, std::vector<int>> m; return m; }
  std::string tune_key() const {
    return std::to_string(sizeof(T)) + ":" + std::to_string(g.Nx) + "x" + std::to_string(g.Ny) + "x" + std::to_string(g.Nz) +
           ":V" + std::to_string(dm.V) + ":R" + std::to_string(dm.R) + ":f" + std::to_string(opt.psi_form);
  }
  bool variant_ok(int fam, int v) const {
    int Lr = (fam == FAM_C2C || (fam == FAM_MUL && psi_full())) ? g.Nx : g.Nx / 2;
    int Lc = (g.nd == 3) ? std::min(g.Ny, g.Nz) : g.Ny;
    int L = (fam == FAM_COLS || fam == FAM_COLS_PSI || fam == FAM_PSI_INV2 || fam == FAM_PSI_COMB || fam == FAM_PSI_FWD2)
                ? Lc : Lr;
    return vE(v) <= L && vE(v) * VNT[v] / L >= 1;
  }
  // Where this handle's variants came from: "forced" (VSAV_TUNE), "measured", "process" (the
  // in-memory cache of an earlier handle of the same shape) or "file" (VSAV_TUNE_FILE)
  const char* tune_source = "measured";
  // VSAV_TUNE_FILE: a JSON object {key: [variant per family..., split]} that persists the
  // choices across processes.  A key found there is used as is; a key measured here is
  // added to the file (rewritten whole, under the process-wide tuning lock).
  static bool tune_file_read(const char* path, std::map<std::string, std::vector<int>>& out) {
    FILE* f = fopen(path, "r");
    if (!f) return false;
    std::string txt;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) txt.append(buf, n);
    fclose(f);
    size_t i = 0;
    while ((i = txt.find('"', i)) != std::string::npos) {
      size_t j = txt.find('"', i + 1);
      if (j == std::string::npos) break;
      std::string key = txt.substr(i + 1, j - i - 1);
      size_t a = txt.find('[', j), b = txt.find(']', j);
      if (a == std::string::npos || b == std::string::npos || b < a) break;
      std::vector<int> v;
      const char* q = txt.c_str() + a + 1;
      const char* end = txt.c_str() + b;
      while (q < end) {
        char* nx = nullptr;
        long x = strtol(q, &nx, 10);
        if (nx == q) { ++q; continue; }
        v.push_back((int)x);
        q = nx;
      }
      if ((int)v.size() == FAM_N + 2) out[key] = v;
      i = b + 1;
    }
    return true;
  }
  static void tune_file_write(const char* path, const std::map<std::string, std::vector<int>>& m) {
    std::string tmp = std::string(path) + ".tmp";
    FILE* f = fopen(tmp.c_str(), "w");
    if (!f) return;
    fprintf(f, "{\n");
    size_t k = 0;
    for (const auto& kv : m) {
      fprintf(f, "  \"%s\": [", kv.first.c_str());
      for (size_t i = 0; i < kv.second.size(); ++i) fprintf(f, "%s%d", i ? ", " : "", kv.second[i]);
      fprintf(f, "]%s\n", ++k < m.size() ? "," : "");
    }
    fprintf(f, "}\n");
    fclose(f);
    rename(tmp.c_str(), path);
  }
  void autotune() {
    if (const char* forced = getenv("VSAV_TUNE")) {      // one digit per family: the variant index
      int k = 0;
      for (const char* q = forced; *q && k < FAM_N; ++q)
        if (*q >= '0' && *q <= '9') { int v = *q - '0'; if (v < NVAR && variant_ok(k, v)) choice[k] = v; ++k; }
      tune_source = "forced";
      return;
    }
    const char* tfile = getenv("VSAV_TUNE_FILE");
    {
      // a tuning file that names this shape wins over the in-process cache
      std::lock_guard<std::mutex> lk(tune_mutex());
      auto it = tune_cache().find(tune_key());
      auto from_process = [&]() {
        for (int f = 0; f < FAM_N; ++f) choice[f] = it->second[f];
        split_comb = it->second[FAM_N];
        tma_from_code(it->second[FAM_N + 1]);
        tuned_from_cache = true;
        tune_source = "process";
      };
      if (!(tfile && *tfile) && it != tune_cache().end()) { from_process(); return; }
      if (tfile && *tfile) {
        std::map<std::string, std::vector<int>> fm;
        tune_file_read(tfile, fm);
        auto jt = fm.find(tune_key());
        bool ok = jt != fm.end();
        if (ok)
          for (int f = 0; f < FAM_N; ++f)
            if (jt->second[f] < 0 || jt->second[f] >= NVAR || !variant_ok(f, jt->second[f])) ok = false;
        if (ok) {
          for (int f = 0; f < FAM_N; ++f) choice[f] = jt->second[f];
          split_comb = jt->second[FAM_N] != 0;
          tma_from_code(jt->second[FAM_N + 1]);
          tune_cache()[tune_key()] = jt->second;
          tuned_from_cache = true;
          tune_source = "file";
          return;
        }
      }
      if (it != tune_cache().end()) { from_process(); return; }
    }
    autotune_measure();
    std::lock_guard<std::mutex> lk(tune_mutex());
    std::vector<int> c(choice, choice + FAM_N);
    c.push_back(split_comb);
    c.push_back(tma_cols | tma_var_inv2 << 1 | tma_var_comb << 3 | bulk_rows << 5 | bulk_var << 6 | cols_tma << 8 |
                cols_tma_var << 9 | c2r_bulk << 10);
    tune_cache()[tune_key()] = c;
    if (tfile && *tfile) {
      std::map<std::string, std::vector<int>> fm;
      tune_file_read(tfile, fm);
      fm[tune_key()] = c;
      tune_file_write(tfile, fm);
    }
  }
  void tma_from_code(int code) {
    tma_var_inv2 = (code >> 1) & 3;
    tma_var_comb = (code >> 3) & 3;
    if (tma_var_inv2 >= TMA_NV || tma_var_comb >= TMA_NV) tma_var_inv2 = tma_var_comb = 0;
    tma_cols = (code & 1) && tma_eligible() && tma_var_ok(tma_var_inv2) && tma_var_ok(tma_var_comb);
    bulk_var = (code >> 6) & 3;
    bulk_rows = ((code >> 5) & 1) && bulk_eligible() && bulk_var_ok(bulk_var);
    if (!bulk_rows) bulk_var = 0;
    cols_tma_var = (code >> 9) & 1;
    cols_tma = ((code >> 8) & 1) && cols_tma_var_ok(cols_tma_var);
    if (!cols_tma) cols_tma_var = 0;
    c2r_bulk = ((code >> 10) & 1) && c2r_bulk_shape();
  }
  // the variants in use, as JSON: {"key", "source", "split", families: "E<e>/NT<nt>"}
  std::string tuning_json() const {
    static const char* nm[FAM_N] = {"rows_r2c", "rows_c2r", "rows_c2c", "rows_mul", "cols", "cols_psi", "psi_inv2",
                                    "psi_comb", "psi_fwd2"};
    std::string o = "{\"key\": \"" + tune_key() + "\", \"source\": \"" + tune_source + "\", \"psi_forward_combine\": \"" +
                    (split_comb ? "split" : "fused") + "\", \"psi_column_passes\": \"" +
                    (tma_cols ? "tma" : "classic") + "\", \"field_column_pass\": \"" +
                    (cols_tma ? "tma E" + std::to_string(CT_E[cols_tma_var]) + "/NT" + std::to_string(CT_NT[cols_tma_var])
                              : std::string("classic")) + "\", \"field_c2r_pass\": \"" +
                    (c2r_bulk ? "bulk E" + std::to_string(CB_E) + "/NT" + std::to_string(CB_NT) : std::string("classic")) +
                    "\", \"variants\": {";
    o += std::string("\"psi_rows\": \"") +
         (bulk_rows ? "bulk E" + std::to_string(BR_E[bulk_var]) + "/NT" + std::to_string(BR_NT[bulk_var]) + "/S" +
                          std::to_string(BR_S[bulk_var])
                    : std::string("classic")) + "\", ";
    if (tma_cols)
      o += "\"psi_inv2_tma\": \"E" + std::to_string(TMA_VE[tma_var_inv2]) + "/NT" + std::to_string(TMA_VNT[tma_var_inv2]) +
           "\", \"psi_comb_tma\": \"E" + std::to_string(TMA_VE[tma_var_comb]) + "/NT" +
           std::to_string(TMA_VNT[tma_var_comb]) + "\", ";
    for (int f = 0; f < FAM_N; ++f)
      o += std::string(f ? ", " : "") + "\"" + nm[f] + "\": \"E" + std::to_string(vE(choice[f])) + "/NT" +
           std::to_string(VNT[choice[f]]) + "\"";
    o += "}";
    if (ntimg) o += std::string(", \"psi_net_kernel\": \"") + (net_impl == 2 ? "k_net_apply_tc (tcgen05)" : "k_net_apply (mma.sync)") + "\"";
    if (psi32) o += ", \"psi_fp32\": " + psi32->tuning_json();
    return o + "}";
  }
  std::string tuning() override { return tuning_json(); }
  static std::mutex& tune_mutex() { static std::mutex m; return m; }
  void autotune_measure() {
    cudaEvent_t e0, e1;
    VSAV_CUDA(cudaEventCreate(&e0));
    VSAV_CUDA(cudaEventCreate(&e1));
    const int V = dm.V;
    const long long nrows = (long long)V * g.Nz * g.Ny;
    bool was = prof.on;
    prof.on = false;
    bool have_mul = (g.nd == 2) && vt12 != nullptr;
    // the fused x pass skips inactive systems: time it with every system active
    if (have_mul) VSAV_CUDA(cudaMemsetAsync(bupd, 0xff, 3 * dm.R * sizeof(int), st));
    cols_tma = 0;
    c2r_bulk = 0;
    for (int fam = 0; fam < FAM_N; ++fam) {
      if (fam == FAM_MUL && !have_mul) continue;
      if ((fam == FAM_C2C || fam == FAM_COLS_PSI || fam == FAM_PSI_INV2 || fam == FAM_PSI_COMB || fam == FAM_PSI_FWD2) &&
          !(g.nd == 2 && psi_full()))
        continue;
      double best = 1e30;
      int bestv = 0;
      while (!variant_ok(fam, bestv) && bestv + 1 < NVAR) ++bestv;
      for (int v = 0; v < NVAR; ++v) {
        if (!variant_ok(fam, v)) continue;
        choice[fam] = v;
        auto run = [&]() {
          switch (fam) {
            case FAM_R2C: rows_r2c(tmpP, nullptr, 1, 0, tmpH, nrows); break;
            case FAM_C2R: rows_c2r(tmpH, tmpP, 1.0, nrows); break;
            case FAM_C2C: rows_c2c<false>(vb, nullptr, vt, 1.0, 3LL * V * g.Ny); break;
            case FAM_MUL: rows_mul(vt12, 2LL * psi_chunk() * g.Ny, psi_full(), 0, psi_chunk()); break;
            case FAM_COLS_PSI: cols(true, 3, 3LL * V, vb, nullptr, 1, 0, M_ONE, 1, vt, 1); break;
            case FAM_PSI_INV2: psi_cols_inv2(vb, vt12, vt12 + 3LL * V * psi_n(), 0, 3 * V, false); break;
            case FAM_PSI_COMB: psi_cols_comb(vt12, vt12 + 3LL * V * psi_n(), vb, vt, 0, nullptr, nullptr, 0, 3 * V, false); break;
            case FAM_PSI_FWD2: psi_cols_fwd2(vt12, vt12 + 3LL * V * psi_n(), 0, 3 * V, false); break;
            default: cols(false, g.nd == 2 ? 0 : 1, V, tmpH, nullptr, 1, 0, M_ONE, 1, tmpH, 1); break;
          }
        };
        run();
        VSAV_CUDA(cudaEventRecord(e0, st));
        for (int k = 0; k < 3; ++k) run();
        VSAV_CUDA(cudaEventRecord(e1, st));
        VSAV_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        VSAV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        tune_ms[fam][v] = ms / 3;
        if (ms < best) { best = ms; bestv = v; }
      }
      choice[fam] = bestv;
    }
    // the bulk-copy-fed c2r x pass against the classic one (as chosen above), on the same call
    if (c2r_bulk_ok(nrows)) {
      auto fn = [&]() { rows_c2r_bulk(tmpH, tmpP, 1.0, nrows); };
      fn();
      VSAV_CUDA(cudaEventRecord(e0, st));
      for (int k = 0; k < 3; ++k) fn();
      VSAV_CUDA(cudaEventRecord(e1, st));
      VSAV_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      VSAV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      c2r_bulk_ms = ms / 3;
      c2r_bulk = c2r_bulk_ms < tune_ms[FAM_C2R][choice[FAM_C2R]];
    }
    // the TMA-fed field column pass against the classic one (as chosen above), on the same call
    if (cols_tma_eligible()) {
      double best = 1e30;
      int bv = -1;
      for (int v = 0; v < CT_NV; ++v) {
        if (!cols_tma_var_ok(v)) continue;
        auto fn = [&]() { cols_tma_run(false, V, tmpH, nullptr, 1, 0, M_ONE, 1, tmpH, 1, v); };
        fn();
        VSAV_CUDA(cudaEventRecord(e0, st));
        for (int k = 0; k < 3; ++k) fn();
        VSAV_CUDA(cudaEventRecord(e1, st));
        VSAV_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        VSAV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cols_tma_ms[v] = ms / 3;
        if (cols_tma_ms[v] < best) { best = cols_tma_ms[v]; bv = v; }
      }
      if (bv >= 0 && best < tune_ms[FAM_COLS][choice[FAM_COLS]]) { cols_tma = 1; cols_tma_var = bv; }
    }
    // split or fused forward pass + combine: the split pair's streaming combine timed on the same fields
    split_comb = 0;
    if (g.nd == 2 && psi_full() && vt12 != nullptr) {
      const long long n = psi_n();
      EW e = ew(n);
      auto combz = [&]() { psi_combz(vb, vt12, vt, 0, nullptr, nullptr, 0, 3 * V, e, false); };
      combz();
      VSAV_CUDA(cudaEventRecord(e0, st));
      for (int k = 0; k < 3; ++k) combz();
      VSAV_CUDA(cudaEventRecord(e1, st));
      VSAV_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      VSAV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      split_ms = tune_ms[FAM_PSI_FWD2][choice[FAM_PSI_FWD2]] + ms / 3;
      // the fused form (fewer bytes) unless the split pair is clearly faster
      split_comb = split_ms < 0.95 * tune_ms[FAM_PSI_COMB][choice[FAM_PSI_COMB]];
    }
    // the TMA-fed pair of psi column passes against the classic pair (as chosen above)
    tma_cols = 0;
    if (tma_eligible()) {
      const long long n = psi_n();
      const int F3 = 3 * V;
      C* t1 = vt12;
      C* t2 = vt12 + (long long)F3 * n;
      auto timed = [&](auto&& fn) {
        fn();
        VSAV_CUDA(cudaEventRecord(e0, st));
        for (int k = 0; k < 3; ++k) fn();
        VSAV_CUDA(cudaEventRecord(e1, st));
        VSAV_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        VSAV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms / 3;
      };
      double ti[TMA_NV], tc[TMA_NV];
      tma_var_inv2 = tma_var_comb = -1;
      for (int v = 0; v < TMA_NV; ++v) {
        if (!tma_var_ok(v)) continue;
        ti[v] = timed([&]() { psi_cols_inv2_tma(vb, t1, t2, 0, F3, false, v); });
        tc[v] = timed([&]() { psi_cols_comb_tma(t1, t2, vb, vt, 0, nullptr, nullptr, 0, F3, false, v); });
        if (tma_var_inv2 < 0 || ti[v] < ti[tma_var_inv2]) tma_var_inv2 = v;
        if (tma_var_comb < 0 || tc[v] < tc[tma_var_comb]) tma_var_comb = v;
      }
      tma_ms = ti[tma_var_inv2] + tc[tma_var_comb];
      const double classic = tune_ms[FAM_PSI_INV2][choice[FAM_PSI_INV2]] +
                             (split_comb ? split_ms : tune_ms[FAM_PSI_COMB][choice[FAM_PSI_COMB]]);
      tma_cols = tma_ms < classic;
    }
    // the bulk-copy-fed x pass against the classic one (as chosen above)
    bulk_rows = 0;
    bulk_var = 0;
    if (bulk_eligible()) {
      const int Fc = psi_chunk();                        // the classic pass was timed on one chunk too
      double best = 1e30;
      int bv = -1;
      for (int v = 0; v < BR_NV; ++v) {
        if (!bulk_var_ok(v)) continue;
        auto fn = [&]() { rows_mul_bulk(vt12, 0, Fc, v); };
        fn();
        VSAV_CUDA(cudaEventRecord(e0, st));
        for (int k = 0; k < 3; ++k) fn();
        VSAV_CUDA(cudaEventRecord(e1, st));
        VSAV_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        VSAV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        bulk_ms[v] = ms / 3;
        if (bulk_ms[v] < best) { best = bulk_ms[v]; bv = v; }
      }
      if (bv >= 0 && best < tune_ms[FAM_MUL][choice[FAM_MUL]]) { bulk_rows = 1; bulk_var = bv; }
    }
    prof.on = was;
    if (getenv("VSAV_VERBOSE")) {
      const char* nm[FAM_N] = {"rows_r2c", "rows_c2r", "rows_c2c", "rows_mul", "cols", "cols_psi", "psi_inv2", "psi_comb",
                               "psi_fwd2"};
      for (int f = 0; f < FAM_N; ++f) for (int v = 0; v < NVAR; ++v) if (!variant_ok(f, v)) tune_ms[f][v] = -1;
      for (int f = 0; f < FAM_N; ++f) {
        fprintf(stderr, "[vsav autotune %s] %-9s", std::is_same<T, double>::value ? "fp64" : "fp32", nm[f]);
        for (int v = 0; v < NVAR; ++v) fprintf(stderr, "  E%d/NT%d %.3f ms", vE(v), VNT[v], tune_ms[f][v]);
        fprintf(stderr, "  -> %d\n", choice[f]);
      }
      fprintf(stderr, "[vsav autotune %s] forward pass + combine: %s (split %.3f ms); TMA column passes: %s (%.3f ms)\n",
              std::is_same<T, double>::value ? "fp64" : "fp32", split_comb ? "split" : "fused", split_ms,
              tma_cols ? "on" : "off", tma_ms);
      fprintf(stderr, "[vsav autotune %s] bulk x pass: %s (%.3f / %.3f / %.3f ms)\n",
              std::is_same<T, double>::value ? "fp64" : "fp32", bulk_rows ? "on" : "off", bulk_ms[0], bulk_ms[1], bulk_ms[2]);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // the scratch buffers carry garbage now: clear what later code expects zeroed
    VSAV_CUDA(cudaMemsetAsync(tmpH, 0, std::max<long long>(8 * dm.V, 9 * dm.R) * g.H * sizeof(C), st));
    if (have_mul) VSAV_CUDA(cudaMemsetAsync(bupd, 0, 3 * dm.R * sizeof(int), st));
    VSAV_CUDA(cudaStreamSynchronize(st));
  }

  // rfft over the nd spatial axes of nf real fields  (in = a0 in0 + a1 in1)
  void rfft(const T* in0, long long nf, C* out, const T* in1 = nullptr, double a0 = 1, double a1 = 0) {
    rows_r2c(in0, in1, a0, a1, out, nf * g.Nz * g.Ny);
    if (g.nd == 2) cols(false, 0, nf, out, nullptr, 1, 0, M_ONE, 1, out, 1);
    else { cols(false, 2, nf, out, nullptr, 1, 0, M_ONE, 1, out, 1); cols(false, 1, nf, out, nullptr, 1, 0, M_ONE, 1, out, 1); }
  }
  // irfft of mult * (a0 in0 + a1 in1), normalised (the reference's ifft plans)
  void irfft(const C* in0, long long nf, T* out, int mult = M_ONE, double ms = 1.0, const C* in1 = nullptr, double a0 = 1,
             double a1 = 0) {
    if (nf * g.H > std::max<long long>(8 * dm.V, 9 * dm.R) * g.H) throw std::runtime_error("irfft batch too large");
    if (g.nd == 2) cols(true, 0, nf, in0, in1, a0, a1, mult, ms, tmpH, 1);
    else { cols(true, 1, nf, in0, in1, a0, a1, mult, ms, tmpH, 1); cols(true, 2, nf, tmpH, nullptr, 1, 0, M_ONE, 1, tmpH, 1); }
    rows_c2r(tmpH, out, 1.0 / (double)g.P, nf * g.Nz * g.Ny);
  }

  // ------------------------------------------------------------------ pieces
  void set_bdf(int n) {
    if (n == 1) { cur_a = 1.0; cur_b = -1.0; cur_c = 0.0; } else { cur_a = 1.5; cur_b = -2.0; cur_c = 0.5; }
  }

  // H1, H2, H3, MG at (phi, psi)  (+ W3 integrands, M_psi when phio given) -> H4, Hh, scH
  void compute_H(const T* phi_in, const T* phio, const T* psi_in, const T* psio, bool star) {
    const int V = dm.V;
    const long long VP = (long long)V * g.P;
    EW e = ew(g.P);
    dim3 gv(e.bpf, V);
    const T *phi = phi_in, *psi = psi_in;
    if (star) {
      k_star<T><<<gv, 256, 0, st>>>(phi_in, phio, psi_in, psio, phis, psis, Mpsi, ph, rn, e, part); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      phi = phis; psi = psis;
    } else {
      k_star<T><<<gv, 256, 0, st>>>(phi_in, nullptr, psi_in, nullptr, nullptr, nullptr, nullptr, ph, rn, e, part); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
    }
    fin(3, V, e, fd2);                                   // fd2[v*3+1..2] = f_osm, psi^2
    if (star) { k_fin_max<<<V, 32, 0, st>>>(part, e.bpf, 3, 0, mmax_v); VSAV_COUNT_LAUNCH(); VSAV_LAUNCH_CHECK(); }
    rfft(phi, V, tmpH2);
    irfft(tmpH2, V, d4, M_DX);
    irfft(tmpH2, V, d4 + VP, M_DY);
    irfft(tmpH2, V, d4 + 2 * VP, M_LAP);
    irfft(tmpH2, V, d4 + 3 * VP, M_BIH);
    area_sums(phi, d4, d4 + VP, e);              // fd2 slot 0 of each vesicle <- f_surf sum
    k_surf<T><<<gv, 256, 0, st>>>(phi, d4, d4 + VP, d4 + 2 * VP, omega, ph, e, part); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    fin(3, V, e, fd);                                    // fd[v*3+0..2] = surf, bend, E2
    k_fin_H<<<(dm.R + 63) / 64, 64, 0, st>>>(asum, fd, fd2, star ? mmax_v : nullptr, d_A0, ph, rn, scH, factor, area, d_err); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    if (star) { k_copy_mmax<<<(dm.R + 63) / 64, 64, 0, st>>>(scH, mmax_r, dm.R); VSAV_COUNT_LAUNCH(); VSAV_LAUNCH_CHECK(); }
    rfft(omega, V, tmpH2);
    irfft(tmpH2, V, lapomega, M_LAP);
    k_H<T><<<gv, 256, 0, st>>>(phi, psi, omega, lapomega, d4 + 2 * VP, d4 + 3 * VP, scH, factor, H4, VP, ph, rn, e); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    rfft(H4, 4LL * V, Hh);
  }


  // ------------------------------------------------------------------ steps
  void step1(int n) override {
    set_bdf(n);
    const int V = dm.V, R = dm.R, nd = g.nd;
    const long long VP = (long long)V * g.P, VH = (long long)V * g.H, RP = (long long)R * g.P;
    compute_H(phys4[0], phys4[1], phys4[0] + VP, phys4[1] + VP, true);
    k_axpby<T><<<gridfor(nd * RP), 256, 0, st>>>(uphys[0], uphys[1], ustar, 2.0, -1.0, nd * RP); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    // psi 12 flux: D1_d . rfft(M dG/dx_d)
    const C* Gh = Hh + 3 * VH;
    for (int d = 0; d < nd; ++d) irfft(Gh, V, gG + d * VP, M_DX + d);
    const bool psi_krylov_step = nd == 2 || opt.psi3d_var;
    if (psi_krylov_step) {
      k_mul_field<T><<<gridfor((long long)nd * VP), 256, 0, st>>>(gG, Mpsi, 1.0, gG, VP, nd); VSAV_COUNT_LAUNCH();
    } else {
      k_mul_field<T><<<gridfor(3 * VP), 256, 0, st>>>(gG, nullptr, ph.M0_psi, gG, 3 * VP, 1); VSAV_COUNT_LAUNCH();
    }
    VSAV_LAUNCH_CHECK();
    rfft(gG, (long long)nd * V, flh);
    // advection of the stored spectra: u* . grad(phi*), u* . grad(psi*)
    for (int q = 0; q < 2; ++q)
      for (int d = 0; d < nd; ++d)
        irfft(hat4[0] + q * VH, V, gstar + (q * nd + d) * VP, M_DX + d, 1.0, hat4[1] + q * VH, 2.0, -1.0);
    k_advect<T><<<gridfor(2 * VP), 256, 0, st>>>(gstar, ustar, adv, 2, nd, rn, g.P); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    rfft(adv, 2LL * V, advh);
    k_set_adt<<<(R + 63) / 64, 64, 0, st>>>(d_dt, cur_a, d_adt, R); VSAV_COUNT_LAUNCH();
    k_step1_k<T><<<gridfor(VH), 256, 0, st>>>(hat4[0], hat4[1], Hh, flh, nd, advh, cache, rhs, d_dt, cur_a, cur_b, cur_c,
                                              ph, rn, g, psi_krylov_step ? 0 : 1); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    if (psi_krylov_step) {
      psi_solve();
      k_nu<T><<<gridfor(VH), 256, 0, st>>>(cache, Gh, ph.S4, VH, g); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
    }
  }

  void step2(int n) override {
    set_bdf(n);
    const int V = dm.V;
    const long long VP = (long long)V * g.P;
    irfft(cache, 8LL * V, cphys);
    EW e = ew(g.P);
    k_dot2<T><<<dim3(e.bpf, V), 256, 0, st>>>(H4, phys4[0], phys4[1], phys4[0] + VP, phys4[1] + VP, cphys, cur_b, cur_c, VP, e, part); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    fin(22, V, e, fd);
    k_fin_step2<<<(dm.R + 63) / 64, 64, 0, st>>>(fd, sc[0], sc[1], cur_a, cur_b, cur_c, ph, rn, r2); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }

  void step3() override {
    const long long VH = (long long)dm.V * g.H;
    k_step3<T><<<gridfor(VH), 256, 0, st>>>(cache, r2, s3, rn, g); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }

  void step4(int n) override {
    set_bdf(n);
    const int V = dm.V, R = dm.R, nd = g.nd;
    const long long VP = (long long)V * g.P, VH = (long long)V * g.H, RP = (long long)R * g.P, RH = (long long)R * g.H;
    for (int c = 0; c < nd; ++c)
      for (int d = 0; d < nd; ++d)
        irfft(uhat[0] + c * RH, R, gu + (c * nd + d) * RP, M_DX + d, 1.0, uhat[1] + c * RH, 2.0, -1.0);
    for (int d = 0; d < nd; ++d) {
      irfft(hat4[0] + 2 * VH, V, gmu + d * VP, M_DX + d, 1.0, hat4[1] + 2 * VH, 2.0, -1.0);
      irfft(hat4[0] + 3 * VH, V, gnu + d * VP, M_DX + d, 1.0, hat4[1] + 3 * VH, 2.0, -1.0);
    }
    k_conv_coupl<T><<<gridfor(RP), 256, 0, st>>>(ustar, gu, phis, psis, gmu, gnu, conv, coupl, rhs2, ph.lamda, nd, rn, g.P); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    rfft(rhs2, (long long)nd * R, uth + nd * RH);
    k_step4_k<T><<<gridfor(RH), 256, 0, st>>>(uhat[0], uhat[1], uth, d_dt, cur_a, cur_b, cur_c, ph, R, g); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    irfft(uth, 2LL * nd * R, utp);
  }

  void step5(int n) override {
    set_bdf(n);
    const int V = dm.V, R = dm.R;
    const long long VP = (long long)V * g.P, VH = (long long)V * g.H, RP = (long long)R * g.P;
    irfft(s3 + 4 * VH, 4LL * V, mn);
    EW e = ew(g.P);
    k_dot5v<T><<<dim3(e.bpf, V), 256, 0, st>>>(adv, mn, VP, e, part); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    fin(4, V, e, fd);
    k_dot5r<T><<<dim3(e.bpf, R), 256, 0, st>>>(coupl, conv, utp, g.nd, RP, e, part); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    fin(4, R, e, fd2);
    k_fin_step5<<<(R + 63) / 64, 64, 0, st>>>(fd, fd2, sc[0], sc[1], d_dt, g.nd == 3, cur_a, cur_b, cur_c, ph, rn, qv, theta); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }

  void step6() override {
    const long long VH = (long long)dm.V * g.H;
    k_step6<T><<<gridfor(VH), 256, 0, st>>>(s3, qv, hat4[1], rn, g); VSAV_COUNT_LAUNCH();
    k_step6_scalars<<<(dm.R + 63) / 64, 64, 0, st>>>(r2, qv, sc[1], dm.R); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }

  void step7(int n) override {
    set_bdf(n);
    const long long RH = (long long)dm.R * g.H;
    k_step67<T><<<gridfor(RH), 256, 0, st>>>(uth, qv, uhat[0], uhat[1], d_dt, cur_a, ph, dm.R, g); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }

  // old <- present ; present <- new (written into old's storage by steps 6/7) ; physical fields by irfft
  void swap_levels() {
    std::swap(phys4[0], phys4[1]); std::swap(hat4[0], hat4[1]);
    std::swap(uphys[0], uphys[1]); std::swap(uhat[0], uhat[1]);
    std::swap(sc[0], sc[1]);
    parity ^= 1;
  }
  void update_state() override {
    swap_levels();
    ++steps_done;
    irfft(hat4[0], 4LL * dm.V, phys4[0]);
    irfft(uhat[0], (long long)(g.nd + 1) * dm.R, uphys[0]);
  }

  void monitor(double* h_energy, double* h_aratio) override {
    monitor_kernels();
    const int R = dm.R;
    if (h_energy) VSAV_CUDA(cudaMemcpyAsync(h_energy, energy, R * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (h_aratio) VSAV_CUDA(cudaMemcpyAsync(h_aratio, aratio, R * sizeof(double), cudaMemcpyDeviceToHost, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
  }
  void monitor_kernels() {
    const int V = dm.V, R = dm.R;
    const long long VP = (long long)V * g.P, VH = (long long)V * g.H, RP = (long long)R * g.P, RH = (long long)R * g.H;
    const C* ph_p = uhat[0] + g.nd * RH;
    irfft(ph_p, R, mon_gp, M_DX);
    irfft(ph_p, R, mon_gp + RP, M_DY);
    irfft(hat4[0], V, mon_lap, M_LAP);
    irfft(hat4[0], V, mon_lap + VP, M_LAP, 1.0, hat4[1], 2.0, -1.0);
    bool s2 = ph.S2 != 0.0;
    if (s2) {
      irfft(hat4[0], V, mon_g4, M_DX);
      irfft(hat4[0], V, mon_g4 + VP, M_DY);
      irfft(hat4[0], V, mon_g4 + 2 * VP, M_DX, 1.0, hat4[1], 2.0, -1.0);
      irfft(hat4[0], V, mon_g4 + 3 * VP, M_DY, 1.0, hat4[1], 2.0, -1.0);
    }
    rfft(phys4[0], V, tmpH2);
    irfft(tmpH2, V, mon_ga, M_DX);
    irfft(tmpH2, V, mon_ga + VP, M_DY);
    EW e = ew(g.P);
    k_mon_v<T><<<dim3(e.bpf, V), 256, 0, st>>>(phys4[0], phys4[1], phys4[0] + VP, phys4[1] + VP, mon_lap, mon_lap + VP,
                                               s2 ? mon_g4 : nullptr, mon_ga, VP, ph, e, part); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    fin(9, V, e, fd);
    k_mon_r<T><<<dim3(e.bpf, R), 256, 0, st>>>(uphys[0], uphys[1], mon_gp, g.nd, RP, e, part); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    fin(3, R, e, fd2);
    k_fin_mon<<<(R + 63) / 64, 64, 0, st>>>(fd, fd2, sc[0], sc[1], d_dt, d_A0, ph, rn, energy, aratio, area); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }

  // ------------------------------------------------------------------ step graphs
  // A BDF2 time step (Steps 1-7, update, optional monitor) is captured once per
  // (level parity, monitor) -- the two time levels swap by pointer each step,
  // so even and odd steps bake in different addresses -- and replayed with one
  // cudaGraphLaunch; its Krylov loops are conditional WHILE nodes, so a step
  // needs no host round trip.  The first (BDF1) step runs eagerly, which also
  // sets every kernel's attributes before any capture.
  struct StepGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CaptureCtx cx;
  };
  StepGraph sgraph[2][2];         // [level parity][monitor]
  int parity = 0;
  unsigned* d_trips_all = nullptr;
  unsigned* h_trips = nullptr;
  cudaStream_t side_st = nullptr;
  long long steps_done = 0;

  void capture_step(StepGraph& sg, int n, int mon, unsigned* trips) {
    sg.cx = CaptureCtx{};
    sg.cx.d_trips = trips;
    sg.cx.side = side_st;
    sg.cx.err = d_err;
    capture_ctx() = &sg.cx;
    const long long c0 = launch_counter().load();
    VSAV_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      step1(n); step2(n); step3(); step4(n); step5(n); step6(); step7(n);
      update_state();
      if (mon) monitor_kernels();
    } catch (...) {
      cudaGraph_t tmp = nullptr;
      cudaStreamEndCapture(st, &tmp);
      if (tmp) cudaGraphDestroy(tmp);
      capture_ctx() = nullptr;
      throw;
    }
    capture_ctx() = nullptr;
    VSAV_CUDA(cudaStreamEndCapture(st, &sg.graph));
    long long total = launch_counter().load() - c0, bodies = 0;
    for (long long b : sg.cx.body) bodies += b;
    sg.cx.fixed = total - bodies;
    launch_counter().fetch_sub(total);      // captured, not launched
    VSAV_CUDA(cudaGraphInstantiate(&sg.exec, sg.graph, 0));
  }

  bool step_graph(int n, double* h_energy, double* h_aratio) override {
    if (!opt.graph || n < 2 || steps_done < 1 || prof.on || hv_cap || (psi32 && psi32->prof.on)) return false;
    const int mon = (h_energy || h_aratio) ? 1 : 0;
    if (!d_trips_all) {
      d_trips_all = dalloc<unsigned>(4 * CaptureCtx::kMaxLoops);
      VSAV_CUDA(cudaMallocHost(&h_trips, CaptureCtx::kMaxLoops * sizeof(unsigned)));
      VSAV_CUDA(cudaStreamCreateWithFlags(&side_st, cudaStreamNonBlocking));
    }
    StepGraph& sg = sgraph[parity][mon];
    const bool fresh = sg.exec == nullptr;
    if (fresh) {
      set_bdf(n);
      capture_step(sg, n, mon, d_trips_all + (parity * 2 + mon) * CaptureCtx::kMaxLoops);
    }
    set_bdf(n);
    VSAV_CUDA(cudaGraphLaunch(sg.exec, st));
    if (!fresh) { swap_levels(); ++steps_done; }   // the capture itself ran update_state once
    const size_t nl = sg.cx.body.size();
    if (nl) VSAV_CUDA(cudaMemcpyAsync(h_trips, sg.cx.d_trips, nl * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    if (h_energy) VSAV_CUDA(cudaMemcpyAsync(h_energy, energy, dm.R * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (h_aratio) VSAV_CUDA(cudaMemcpyAsync(h_aratio, aratio, dm.R * sizeof(double), cudaMemcpyDeviceToHost, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
    long long launched = sg.cx.fixed;
    for (size_t l = 0; l < nl; ++l) launched += sg.cx.body[l] * (long long)(h_trips[l] > 0 ? h_trips[l] - 1 : 0);
    launch_counter().fetch_add(launched);
    return true;
  }

  // simulation.jl:22-53
  void init_shapes2d(const Shape2D* shapes) override {
    if (g.nd != 2) throw std::runtime_error("shape initial conditions are 2D");
    const int V = dm.V, R = dm.R;
    const long long VP = (long long)V * g.P;
    for (int v = 0; v < V; ++v)
      if (shapes[v].nmodes < 0 || shapes[v].nmodes > 8 || !(shapes[v].a > 0) || !(shapes[v].b > 0))
        throw std::runtime_error("bad shape " + std::to_string(v) + ": need a, b > 0 and 0..8 modes");
    if ((size_t)V * sizeof(Shape2D) > stage_bytes) throw std::runtime_error("too many vesicle fields for the staging buffer");
    VSAV_CUDA(cudaMemcpyAsync(stage, shapes, V * sizeof(Shape2D), cudaMemcpyHostToDevice, st));
    k_shapes2d<T><<<gridfor(VP), 256, 0, st>>>(phys4[0], phys4[0] + VP, reinterpret_cast<const Shape2D*>(stage), V, g.Nx,
                                               g.Ny, dm.Lx, dm.Ly, ph.eps); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    VSAV_CUDA(cudaMemsetAsync(uphys[0], 0, (g.nd + 1) * (long long)R * g.P * sizeof(T), st));
    init_state(0);
  }

  // generate_initial_condition(conf, ops, state_type) (Init.jl:74-216, Init_3d.jl:67-152)
  // for every run of the handle, each with its own N; blob_u: [R][20] uniform draws
  // of state_type 4 (the reference's rand() calls, Init.jl:156-157), in draw order.
  void init_reference_shapes(int state_type, int goal, const double* blob_u) override {
    const int V = dm.V, R = dm.R;
    const bool is3 = g.nd == 3, gs = goal == 's', gg = goal == 'g';
    auto fail = [&](int r, const std::string& m) {
      throw std::runtime_error("generate_initial_condition" + (R > 1 ? " (run " + std::to_string(r) + ")" : std::string()) +
                               ": " + m);
    };
    std::vector<RefShape> sh(V);
    std::memset(sh.data(), 0, V * sizeof(RefShape));
    int v0 = 0;
    for (int r = 0; r < R; ++r) {
      const int N = h_run_sizes[r];
      double cx[3], cy[3], cz[3];
      if (N == 1) {
        cx[0] = dm.Lx / 2; cy[0] = dm.Ly / 2; cz[0] = dm.Lz / 2;
      } else if (N == 2) {
        if (is3) { cx[0] = 0.73; cx[1] = 1.27; }                      // Init_3d.jl:89
        else if (gg) { cx[0] = 0.75; cx[1] = 1.25; }                  // Init.jl:90-95
        else if (gs) { cx[0] = 0.65; cx[1] = 1.35; }
        else fail(r, "what's the goal? (N = 2 needs goal g or s)");
        cy[0] = cy[1] = dm.Ly / 2; cz[0] = cz[1] = dm.Lz / 2;
      } else if (N == 3) {
        for (int n = 0; n < 3; ++n) { cx[n] = (n + 1) * dm.Lx / 4; cy[n] = dm.Ly / 2; cz[n] = dm.Lz / 2; }
      } else {
        fail(r, "N = " + std::to_string(N) + " has no vesicle centres (N <= 3)");
      }
      const std::string st = "state_type " + std::to_string(state_type);
      if (N == 1 && state_type > 6) fail(r, st + " is invalid for N = 1");
      if (N >= 2 && state_type <= 6 && !(is3 && N == 3)) fail(r, st + " is invalid for N = " + std::to_string(N));
      for (int n = 0; n < N; ++n) {
        RefShape& s = sh[v0 + n];
        s.cx = cx[n]; s.cy = cy[n]; s.cz = cz[n];
        s.alpha = gs ? -0.1 : -0.35;
        s.beta = gs ? 0.7 : 0.45;
        if (is3) {
          if (N == 1 && state_type == 1) { s.kind = RS_ELLIPSOID; s.R0 = 0.2 * dm.Lx; }
          if (N == 2 && state_type == 7) {
            if (gs) fail(r, "state_type 7 needs goal g");
            fail(r, "state_type 7 is not defined in 3D (the reference's branch uses the 2D grids X, Y)");
          }
          continue;
        }
        if (N == 1) {
          if (state_type == 1) { s.kind = RS_ELLIPSE; s.R0 = 0.2 * dm.Lx; }
          else if (state_type == 2) { s.kind = RS_TRIANGLE; s.R0 = 0.65 * dm.Lx; }
          else if (state_type == 3) { s.kind = RS_STAR; s.R0 = gs ? 0.3 : 0.18; s.amp = gs ? 0.01 : 0.02; }
          else if (state_type == 4) {
            if (!blob_u) fail(r, "state_type 4 needs its 20 uniform draws per run");
            s.kind = RS_BLOB; s.R0 = gs ? 0.3 : 0.2; s.amp = gs ? 0.15 : 0.25;
            const double* u = blob_u + 20LL * r;
            for (int m = 0; m < 10; ++m) {
              s.an[m] = (u[2 * m] * 2 - 1) * s.amp / (m + 1);
              s.pn[m] = u[2 * m + 1] * 2 * M_PI;
            }
          }
        } else if (state_type == 7) {
          if (gs) fail(r, "state_type 7 needs goal g");
          s.kind = RS_STAR; s.R0 = 0.2; s.amp = 0.02;
        } else if (state_type == 8) {
          if (gg) fail(r, "state_type 8 needs goal s");
          s.kind = RS_STAR; s.R0 = 0.3; s.amp = 0.01;
        }
      }
      v0 += N;
    }
    if ((size_t)V * sizeof(RefShape) > stage_bytes) throw std::runtime_error("too many vesicle fields for the staging buffer");
    const long long VP = (long long)V * g.P;
    VSAV_CUDA(cudaMemcpyAsync(stage, sh.data(), V * sizeof(RefShape), cudaMemcpyHostToDevice, st));
    k_ref_shapes<T><<<gridfor(VP), 256, 0, st>>>(phys4[0], phys4[0] + VP, reinterpret_cast<const RefShape*>(stage), V,
                                                 g.Nx, g.Ny, g.Nz, dm.Lx / g.Nx, dm.Ly / g.Ny,
                                                 is3 ? dm.Lz / g.Nz : 1.0, ph.eps); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    VSAV_CUDA(cudaMemsetAsync(uphys[0], 0, (g.nd + 1) * (long long)R * g.P * sizeof(T), st));
    init_state(0);
  }

  void init_state(int hats_given) override {
    const int V = dm.V, R = dm.R;
    const long long VP = (long long)V * g.P, VH = (long long)V * g.H;
    if (!hats_given) {
      rfft(phys4[0], V, hat4[0]);
      rfft(phys4[0] + VP, V, hat4[0] + VH);
      rfft(uphys[0], (long long)(g.nd + 1) * R, uhat[0]);
    }
    // A0 = calculate_area(phi)
    EW e = ew(g.P);
    rfft(phys4[0], V, tmpH2);
    irfft(tmpH2, V, mon_ga, M_DX);
    irfft(tmpH2, V, mon_ga + VP, M_DY);
    area_sums(phys4[0], mon_ga, mon_ga + VP, e);
    k_area0<<<(V + 63) / 64, 64, 0, st>>>(asum, ph.cell, d_A0, V); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    compute_H(phys4[0], nullptr, phys4[0] + VP, nullptr, false);
    k_init_scalars<<<(R + 63) / 64, 64, 0, st>>>(scH, sc[0], R); VSAV_COUNT_LAUNCH();
    k_init_munu<T><<<gridfor(VH), 256, 0, st>>>(hat4[0], Hh, sc[0], ph, rn, g); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    irfft(hat4[0] + 2 * VH, 2LL * V, phys4[0] + 2 * VP);
    // old = deepcopy(present)
    VSAV_CUDA(cudaMemcpyAsync(phys4[1], phys4[0], 4 * VP * sizeof(T), cudaMemcpyDeviceToDevice, st));
    VSAV_CUDA(cudaMemcpyAsync(hat4[1], hat4[0], 4 * VH * sizeof(C), cudaMemcpyDeviceToDevice, st));
    VSAV_CUDA(cudaMemcpyAsync(uphys[1], uphys[0], (g.nd + 1) * (long long)R * g.P * sizeof(T), cudaMemcpyDeviceToDevice, st));
    VSAV_CUDA(cudaMemcpyAsync(uhat[1], uhat[0], (g.nd + 1) * (long long)R * g.H * sizeof(C), cudaMemcpyDeviceToDevice, st));
    VSAV_CUDA(cudaMemcpyAsync(sc[1], sc[0], 4 * R * sizeof(double), cudaMemcpyDeviceToDevice, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
  }

  // ------------------------------------------------------------------ psi BiCGSTAB (2D)
  // fields per chunk of the psi operator: the chunk's two intermediates stay in L2
  // (chunking is off by default: VSAV_PSI_CHUNK_MB sets the L2 budget of a chunk)
  long long psi_chunk_mb = 0;  // VSAV_PSI_CHUNK_MB, read when the handle is created (0: no chunking)
  int psi_chunk() const {
    if (psi_chunk_mb <= 0) return 3 * dm.V;
    const long long per = 2LL * psi_n() * (long long)sizeof(C);
    long long fc = std::max<long long>(1, (psi_chunk_mb << 20) / per);
    return (int)std::min<long long>(fc, 3LL * dm.V);
  }

  // y = P^-1 A in (+ dots), chunk by chunk: y-inverse (2 multipliers), fused
  // x pass (inverse, x M_psi, forward), y-forward, combine
  EW dot_ew{};                 // partial layout of the dots of the last matvec
  double split_ms = 0.0, tma_ms = 0.0, bulk_ms[3] = {0.0, 0.0, 0.0};
  bool use_split() const { return split_comb != 0; }
  bool fused_ops = true;       // FULL form: fused column passes (VSAV_PSI_FUSED=0: separate kernels)
  void matvec(const C* in, C* out, int mode, const C* svec, bool precond = true) {
    if (g.nd == 3) { matvec3(in, out, mode, svec, precond); return; }
    const int V = dm.V;
    const long long F = 3LL * V, n = psi_n();
    const bool full = psi_full();
    const int geo = full ? 3 : 0;
    const int Fc = psi_chunk();
    EW e = ew(n);
    VGeom vg{full ? 1 : 0, g.Nx, g.Ny, g.kp, g.nkx, ilog2(g.Nx), n, g.kxs, g.kys};
    SysMap sm{V, dm.R, d_run_of};
    const double* pre = precond ? mmax_r : nullptr;
    dot_ew = e;
    for (int f0 = 0; f0 < F; f0 += Fc) {
      const int fc = (int)std::min<long long>(Fc, F - f0);
      C* t1 = vt12;
      C* t2 = vt12 + (long long)fc * n;
      if (full && fused_ops && tma_cols) {
        // the TMA-fed persistent forms of the two column passes
        psi_cols_inv2_tma(in, t1, t2, f0, fc, true);
        rows_mul(t1, 2LL * fc * g.Ny, full, f0, fc);
        dot_ew.bpf = psi_cols_comb_tma(t1, t2, in, out, mode, svec, pre, f0, fc, true);
        continue;
      }
      if (full && fused_ops) {
        // one read of x for both inverse passes; the forward pass carries the combine
        psi_cols_inv2(in, t1, t2, f0, fc);
        rows_mul(t1, 2LL * fc * g.Ny, full, f0, fc);
        if (use_split()) {
          psi_cols_fwd2(t1, t2, f0, fc);
          psi_combz(in, t1, out, mode, svec, pre, f0, fc, e);
        } else {
          const int tiles = psi_cols_comb(t1, t2, in, out, mode, svec, pre, f0, fc);
          dot_ew.bpf = tiles;
        }
        continue;
      }
      cols(true, geo, fc, in + f0 * n, nullptr, 1, 0, full ? M_DX0 : M_DXZ, ph.S4, t1, 1);
      cols(true, geo, fc, in + f0 * n, nullptr, 1, 0, M_DY, ph.S4, t2, 1);
      rows_mul(t1, 2LL * fc * g.Ny, full, f0, fc);
      cols(false, geo, 2LL * fc, t1, nullptr, 1, 0, M_ONE, 1, t1, 1);
      prof.begin(st);
      k_psi_combine<T><<<dim3(e.bpf, (unsigned)fc), 256, 0, st>>>(in, t1, t2, out, vb, svec, mode, d_adt, pre, ph.S4, vg,
                                                                   sm, bupd, f0, e, part); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      prof.end(st, KC_PSI_VEC, (double)fc * (full ? g.Pfull : (long long)g.Ny * g.nkx) * 5.0 * sizeof(C));
    }
  }

  // 3D full-spectrum operator (variable mobility): per direction d the inverse
  // z and y passes of i k_d S4 x, then one x pass (inverse, * M_psi / P,
  // forward) and the forward y and z passes over all three, then the combine.
  void matvec3(const C* in, C* out, int mode, const C* svec, bool precond) {
    const int V = dm.V;
    const long long F = 3LL * V, n = psi_n();
    EW e = ew(n);
    SysMap sm{V, dm.R, d_run_of};
    const double* pre = precond ? mmax_r : nullptr;
    dot_ew = e;
    C* t = vt12;                                          // [3][F][n]
    const int mults[3] = {M_DX0, M_DY, M_DZ};
    for (int d = 0; d < 3; ++d) {
      cols(true, 4, F, in, nullptr, 1, 0, mults[d], ph.S4, t + d * F * n, 1);
      cols(true, 5, F, t + d * F * n, nullptr, 1, 0, M_ONE, 1, t + d * F * n, 1);
    }
    rows_mul(t, 3 * F * g.Nz * g.Ny, true, 0, (int)F);
    cols(false, 5, 3 * F, t, nullptr, 1, 0, M_ONE, 1, t, 1);
    cols(false, 4, 3 * F, t, nullptr, 1, 0, M_ONE, 1, t, 1);
    prof.begin(st);
    k_psi_combine3<T><<<dim3(e.bpf, (unsigned)F), 256, 0, st>>>(in, t, t + F * n, t + 2 * F * n, out, vb, svec, mode, d_adt,
                                                                pre, ph.S4, vgeom(), sm, bupd, e, part); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    prof.end(st, KC_PSI_VEC, (double)F * n * 6.0 * sizeof(C));
  }

  // b = fft(irfft(rhs)) (FULL) / rfft(irfft(rhs)) (HALF)   (Solvers.jl:70-71)
  void psi_prepare_b() {
    const long long F = 3LL * dm.V;
    irfft(rhs, F, tmpP);
    if (g.nd == 3) {
      rows_c2c<false>(nullptr, tmpP, vb, 1.0, F * g.Nz * g.Ny);
      cols(false, 5, F, vb, nullptr, 1, 0, M_ONE, 1, vb, 1);
      cols(false, 4, F, vb, nullptr, 1, 0, M_ONE, 1, vb, 1);
      return;
    }
    if (psi_full()) {
      rows_c2c<false>(nullptr, tmpP, vb, 1.0, F * g.Ny);
      cols(false, 3, F, vb, nullptr, 1, 0, M_ONE, 1, vb, 1);
    } else {
      rfft(tmpP, F, vb);
    }
  }
  C* psi_x() { return psi_full() ? vx : cache + 5LL * dm.V * g.H; }
  void psi_finish() {
    const long long F = 3LL * dm.V, VH = (long long)dm.V * g.H;
    if (psi_full()) {
      const int rows = g.Nz * g.Ny;
      k_trunc<T><<<gridfor(F * rows * g.kp), 256, 0, st>>>(vx, cache + 5 * VH, g.Nx, rows, g.kp, g.nkx, (int)F); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
    }
  }
  void psi_solve() {
    if (opt.psi_mixed) { psi_solve_mixed(); return; }
    psi_prepare_b();
    psi_krylov(psi_x(), opt.psi_rtol, opt.psi_itmax);
    if (opt.psi_check) psi_check_residual(psi_x());
    psi_finish();
  }

  // psi_check: ||b - A x|| / ||b|| per system of the solve just finished, in this
  // handle's arithmetic (FP64 for FP64 and mixed handles), into d_true_res
  void psi_check_residual(const C* x) {
    const int V = dm.V, R = dm.R, S = 3 * R;
    const long long F = 3LL * V, n = psi_n();
    EW e = ewv(n, (int)F);
    SysMap sm{V, R, d_run_of};
    VSAV_CUDA(cudaMemsetAsync(bupd, 0xff, S * sizeof(int), st));     // every system active in A x
    matvec(x, vt, 0, nullptr, false);
    k_psi_resnorm<T><<<dim3(e.bpf, (unsigned)F), 256, 0, st>>>(vb, vt, vgeom(), e, part); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    fin(4, (int)F, e, fd);
    k_psi_true_res<<<(S + 63) / 64, 64, 0, st>>>(fd, d_true_res, sm, S, (int)F); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }

  // ---- mixed precision: FP32 BiCGSTAB on FP64 residuals (iterative refinement)
  Solver<float>* psi32 = nullptr;
  void psi_solve_mixed();

  // Runs iter() -- one BiCGSTAB iteration ending in k_bi_beta, which leaves the
  // activity of every system in bst and d_any -- until no system is active
  // (at most itmax times: k_bi_beta retires a system at itmax).  Eagerly: a
  // host loop reading d_any after each iteration.  Under stream capture (a
  // time-step graph): a conditional WHILE node whose body is one iteration
  // followed by the condition kernel, bounded by itmax + 1 iterations.
  template <typename F> void krylov_loop(int itmax, F&& iter) {
    const int S = 3 * dm.R;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    VSAV_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusActive) {
      for (int it = 0; it < itmax; ++it) {
        iter();
        if (opt.check_every_iter) {
          VSAV_CUDA(cudaMemcpyAsync(h_pinned_any, d_any, sizeof(int), cudaMemcpyDeviceToHost, st));
          VSAV_CUDA(cudaStreamSynchronize(st));
          if (!*h_pinned_any) break;
        }
        // refresh the activity flags for the operator kernels of the next iteration
        k_bi_flags<<<(S + 63) / 64, 64, 0, st>>>(bst, bupd, S); VSAV_COUNT_LAUNCH();
      }
      return;
    }
    CaptureCtx* cx = capture_ctx();
    if (!cx || (int)cx->body.size() >= CaptureCtx::kMaxLoops)
      throw std::runtime_error("Krylov loop captured outside a time-step capture");
    unsigned* trips = cx->d_trips + cx->body.size();
    int* err = cx->err ? cx->err : d_err;
    cudaGraph_t gr = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndep = 0;
    VSAV_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &gr, &deps, &ndep));
    cudaGraphConditionalHandle hnd;
    VSAV_CUDA(cudaGraphConditionalHandleCreate(&hnd, gr, 0, cudaGraphCondAssignDefault));
    VSAV_CUDA(cudaMemsetAsync(trips, 0, sizeof(unsigned), st));
    k_loop_cond<<<1, 32, 0, st>>>(hnd, bst, S, trips, itmax + 1, err); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    VSAV_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &gr, &deps, &ndep));
    std::vector<cudaGraphNode_t> dv(deps, deps + ndep);
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = hnd;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    VSAV_CUDA(cudaGraphAddNode(&node, gr, dv.data(), dv.size(), &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    VSAV_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    cudaStream_t outer = st;
    st = cx->side;
    const long long c0 = launch_counter().load();
    VSAV_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
      iter();
      k_bi_flags<<<(S + 63) / 64, 64, 0, st>>>(bst, bupd, S); VSAV_COUNT_LAUNCH();
      k_loop_cond<<<1, 32, 0, st>>>(hnd, bst, S, trips, itmax + 1, err); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
    } catch (...) {
      cudaGraph_t tmp = nullptr;
      cudaStreamEndCapture(st, &tmp);
      st = outer;
      throw;
    }
    cudaGraph_t done = nullptr;
    VSAV_CUDA(cudaStreamEndCapture(st, &done));
    st = outer;
    cx->body.push_back(launch_counter().load() - c0);
  }

  // BiCGSTAB (Krylov.jl semantics) on b = vb from x0 = 0, result in x
  void psi_krylov(C* x, double rtol, int itmax) {
    if (opt.psi_precond >= 1) { psi_flex(x, rtol, itmax); return; }
    const int V = dm.V, R = dm.R, S = 3 * R;
    const long long F = 3LL * V, n = psi_n();
    const bool full = psi_full();
    EW e = ewv(n, (int)F);
    VGeom vg = vgeom();
    SysMap sm{V, R, d_run_of};
    k_psi_init<T><<<dim3(e.bpf, (unsigned)F), 256, 0, st>>>(vb, x, vr, vp, d_adt, mmax_r, ph.S4, vg, sm, e, part); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    fin(4, (int)F, e, fd);
    k_bi_init<<<(S + 63) / 64, 64, 0, st>>>(fd, bst, bupd, sm, S, (int)F, opt.psi_atol, rtol, itmax, opt.psi_stop); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    if (hv_cap) { hv_count = 0; harvest_snap(x, vr); }
    krylov_loop(itmax, [&]() {
      matvec(vp, vv, 0, nullptr);                       // v = M^-1 A p ; <c, v>
      fin(4, (int)F, dot_ew, fd);
      k_bi_alpha<<<(S + 63) / 64, 64, 0, st>>>(fd, bst, sm, S, (int)F); VSAV_COUNT_LAUNCH();
      k_psi_s<T><<<dim3(e.bpf, (unsigned)F), 256, 0, st>>>(vr, vv, vs, bst, sm, e); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      matvec(vs, vt, 1, vs);                            // t = M^-1 A s ; <t,s>, <t,t>
      fin(4, (int)F, dot_ew, fd);
      k_bi_omega<<<(S + 63) / 64, 64, 0, st>>>(fd, bst, sm, S, (int)F); VSAV_COUNT_LAUNCH();
      k_psi_update<T><<<dim3(e.bpf, (unsigned)F), 256, 0, st>>>(x, vr, vp, vs, vt, vb, bst, vg, sm, e, part, nullptr, d_adt,
                                                                mmax_r, ph.S4); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      fin(4, (int)F, e, fd);
      VSAV_CUDA(cudaMemsetAsync(d_any, 0, sizeof(int), st));
      k_bi_beta<<<(S + 63) / 64, 64, 0, st>>>(fd, bst, bupd, sm, S, (int)F, itmax, d_any, opt.psi_stop); VSAV_COUNT_LAUNCH();
      k_psi_p<T><<<dim3(e.bpf, (unsigned)F), 256, 0, st>>>(vp, vr, vv, bst, bupd, sm, e); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      if (hv_cap && hv_count < hv_cap) harvest_snap(x, vr);
    });
    if (hv_cap) harvest_final(x);
    (void)full;
  }

  // ---- flexible right-preconditioned BiCGSTAB (an addition; the reference
  // solve is the left-preconditioned psi_krylov above).  x0 = 0, shadow c = b,
  // stop on ||b - A x|| <= atol + rtol ||b|| or itmax.  The preconditioner P
  // may change between applications (learned correction): x is built from the
  // stored preconditioned directions p^ = P p, s^ = P s.
  //   p^ = P p; v = A p^; alpha = rho / <c, v>; s = r - alpha v
  //   s^ = P s; t = A s^; omega = <t, s> / <t, t>
  //   x += alpha p^ + omega s^; r = s - omega t; beta = (rho'/rho)(alpha/omega)
  //   p = r + beta (p - omega v)
  VGeom vgeom() const {
    VGeom v{psi_full() ? 1 : 0, g.Nx, g.Ny, g.kp, g.nkx, ilog2(g.Nx), psi_n(), g.kxs, g.kys};
    if (g.nd == 3) { v.nd3 = 1; v.logNy = ilog2(g.Ny); v.Nz = g.Nz; v.kzs = g.kzs; }
    return v;
  }
  void psi_flex(C* x, double rtol, int itmax) {
    const int V = dm.V, R = dm.R, S = 3 * R;
    const long long F = 3LL * V, n = psi_n();
    EW e = ewv(n, (int)F);
    VGeom vg = vgeom();
    SysMap sm{V, R, d_run_of};
    if (opt.psi_precond == 2 && !net_ok)
      throw std::runtime_error("learned psi preconditioner selected but no network loaded (vsav_set_psi_net)");
    k_psi_init<T><<<dim3(e.bpf, (unsigned)F), 256, 0, st>>>(vb, x, vr, vp, d_adt, nullptr, ph.S4, vg, sm, e, part); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    fin(4, (int)F, e, fd);
    k_bi_init<<<(S + 63) / 64, 64, 0, st>>>(fd, bst, bupd, sm, S, (int)F, opt.psi_atol, rtol, itmax, opt.psi_stop); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    krylov_loop(itmax, [&]() {
      precond_apply(vp, vph);
      matvec(vph, vv, 0, nullptr, false);               // v = A p^ ; <c, v>
      fin(4, (int)F, dot_ew, fd);
      k_bi_alpha<<<(S + 63) / 64, 64, 0, st>>>(fd, bst, sm, S, (int)F); VSAV_COUNT_LAUNCH();
      k_psi_s<T><<<dim3(e.bpf, (unsigned)F), 256, 0, st>>>(vr, vv, vs, bst, sm, e); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      precond_apply(vs, vsh);
      matvec(vsh, vt, 1, vs, false);                    // t = A s^ ; <t, s>, <t, t>
      fin(4, (int)F, dot_ew, fd);
      k_bi_omega<<<(S + 63) / 64, 64, 0, st>>>(fd, bst, sm, S, (int)F); VSAV_COUNT_LAUNCH();
      k_psi_update<T><<<dim3(e.bpf, (unsigned)F), 256, 0, st>>>(x, vr, vph, vs, vt, vb, bst, vg, sm, e, part, vsh, d_adt,
                                                                nullptr, ph.S4); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      fin(4, (int)F, e, fd);
      VSAV_CUDA(cudaMemsetAsync(d_any, 0, sizeof(int), st));
      k_bi_beta<<<(S + 63) / 64, 64, 0, st>>>(fd, bst, bupd, sm, S, (int)F, itmax, d_any, opt.psi_stop); VSAV_COUNT_LAUNCH();
      k_psi_p<T><<<dim3(e.bpf, (unsigned)F), 256, 0, st>>>(vp, vr, vv, bst, bupd, sm, e); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
    });
  }

  // full-spectrum inverse 2D FFT of F = 3V vectors (normalised), in -> out
  void ifft_full(const C* in, C* out) {
    const long long F = 3LL * dm.V;
    cols(true, 3, F, in, nullptr, 1, 0, M_ONE, 1, out, 1);
    rows_c2c<true>(out, nullptr, out, 1.0 / (double)g.P, F * g.Ny);
  }

  // out = P in.  Diagonal: D^-1 in.  Learned: D^-1 in + FFT(s * net(y / s, M~)),
  // y = Re IFFT(D^-1 in) per field, s its RMS, M~ = (M_psi - 0.075) / 0.025.
  void precond_apply(const C* in, C* out) {
    const long long F = 3LL * dm.V, n = psi_n();
    EW e = ewv(n, (int)F);
    SysMap sm{dm.V, dm.R, d_run_of};
    k_psi_diag<T><<<dim3(e.bpf, (unsigned)F), 256, 0, st>>>(in, out, d_adt, mmax_r, ph.S4, vgeom(), sm, e); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    if (opt.psi_precond != 2) return;
    if constexpr (std::is_same<T, float>::value) {
      C* w1 = vt12;
      C* w2 = vt12 + F * n;
      ifft_full(out, w1);
      k_re_sumsq<T><<<dim3(e.bpf, (unsigned)F), 256, 0, st>>>(w1, e, part); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      fin(1, (int)F, e, fd2);
      k_inv_rms<<<(unsigned)((F + 127) / 128), 128, 0, st>>>(fd2, (double)n, inv_s, (int)F); VSAV_COUNT_LAUNCH();
      prof.begin(st);
      if (net_impl == 2) {
        const long long tiles = F * (g.Ny / NT_T) * (g.Nx / NT_T);
        k_net_apply_tc<1><<<(unsigned)std::min<long long>(tiles, net_sms), NT_THREADS, NT_SMEM, st>>>(
            w1, Mpsi, inv_s, w2, g.Ny, g.Nx, dm.V, (int)F, ntimg, nbias, d_err); VSAV_COUNT_LAUNCH();
      } else {
        k_net_apply<1><<<dim3((unsigned)((g.Ny / NA_T) * (g.Nx / NA_T)), (unsigned)F), NA_THREADS, NA_SMEM, st>>>(
            w1, Mpsi, inv_s, w2, g.Ny, g.Nx, dm.V, nfrag, nbias); VSAV_COUNT_LAUNCH();
      }
      VSAV_LAUNCH_CHECK();
      prof.end(st, KC_NET, (double)F * n * (2.0 * sizeof(C)) + (double)dm.V * g.P * sizeof(T));
      rows_c2c<false>(w2, nullptr, w2, 1.0, F * g.Ny);
      cols(false, 3, F, w2, nullptr, 1, 0, M_ONE, 1, out, 1);
    }
  }

  void set_psi_net(const uint32_t* frags, const float* bias, const uint16_t* timg) override {
    if (psi32) { psi32->set_psi_net(frags, bias, timg); return; }
    if (!nfrag) throw std::runtime_error("the handle was not created with the learned psi preconditioner (psi_precond = 2)");
    VSAV_CUDA(cudaMemcpyAsync(nfrag, frags, NF_WORDS * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    VSAV_CUDA(cudaMemcpyAsync(nbias, bias, NF_BIAS * sizeof(float), cudaMemcpyHostToDevice, st));
    VSAV_CUDA(cudaMemcpyAsync(ntimg, timg, NT_WBYTES, cudaMemcpyHostToDevice, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
    net_ok = true;
  }

  // ---- harvest of (x_k, r~_k) pairs of the reference-form BiCGSTAB: physical
  // real parts (FP32) of every iterate of the last psi solve, the final
  // solution and M_psi.  Layout: [cap][2][3V][P] | x* [3V][P] | M [V][P].
  void harvest(int cap) override {
    if (cap < 0) throw std::runtime_error("harvest capacity must be >= 0");
    if (cap > 0 && (g.nd != 2 || !psi_full() || opt.psi_precond != 0 || opt.psi_mixed))
      throw std::runtime_error("harvest needs a 2D handle with the reference-form psi solve (FULL, psi_precond 0, not mixed)");
    if (hv) { VSAV_CUDA(cudaStreamSynchronize(st)); VSAV_CUDA(cudaFree(hv)); hv = nullptr; }
    hv_cap = cap; hv_count = 0;
    if (cap > 0) {
      const long long FP = 3LL * dm.V * g.P;
      VSAV_CUDA(cudaMalloc(&hv, ((2LL * cap + 1) * FP + (long long)dm.V * g.P) * sizeof(float)));
    }
  }
  void harvest_snap(const C* x, const C* r) {
    const long long FP = 3LL * dm.V * g.P;
    float* dst = hv + (long long)hv_count * 2 * FP;
    ifft_full(x, vt12);
    k_take_re<T><<<gridfor(FP), 256, 0, st>>>(vt12, dst, FP); VSAV_COUNT_LAUNCH();
    ifft_full(r, vt12);
    k_take_re<T><<<gridfor(FP), 256, 0, st>>>(vt12, dst + FP, FP); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    ++hv_count;
  }
  void harvest_final(const C* x) {
    const long long FP = 3LL * dm.V * g.P, VP = (long long)dm.V * g.P;
    float* dst = hv + 2LL * hv_cap * FP;
    ifft_full(x, vt12);
    k_take_re<T><<<gridfor(FP), 256, 0, st>>>(vt12, dst, FP); VSAV_COUNT_LAUNCH();
    k_cast<T, float><<<gridfor(VP), 256, 0, st>>>(Mpsi, dst + FP, VP); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }
  long long harvest_read(float* out, long long cap, int* nsnap) override {
    if (!hv) throw std::runtime_error("harvest is not enabled");
    const long long FP = 3LL * dm.V * g.P, VP = (long long)dm.V * g.P;
    const long long need = 2LL * hv_count * FP + FP + VP;
    if (nsnap) *nsnap = hv_count;
    if (!out) return need;
    if (cap < need) throw std::runtime_error("harvest output buffer too small: " + std::to_string(need) + " floats needed");
    VSAV_CUDA(cudaMemcpyAsync(out, hv, 2LL * hv_count * FP * sizeof(float), cudaMemcpyDefault, st));
    VSAV_CUDA(cudaMemcpyAsync(out + 2LL * hv_count * FP, hv + 2LL * hv_cap * FP, (FP + VP) * sizeof(float),
                              cudaMemcpyDefault, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
    return need;
  }

  // ------------------------------------------------------------------ host transfer
  // host layouts (float64): V fields [V][Nz][Ny][Nx]; hats [V][Nz][Ny][nkx] complex;
  // u [R][nd][...]; p [R][...]
  void xfer(int level, int fid, void* host, int dir, int is_device = 0) {
    const int V = dm.V, R = dm.R, nd = g.nd;
    const long long VP = (long long)V * g.P, VH = (long long)V * g.H, RP = (long long)R * g.P, RH = (long long)R * g.H;
    long long rows = (long long)g.Nz * g.Ny;
    bool hat = (fid == F_PHI_HAT || fid == F_PSI_HAT || fid == F_U_HAT || fid == F_P_HAT || fid == F_MU_HAT || fid == F_NU_HAT);
    int Fo, Fi; void* dst;
    switch (fid) {
      case F_PHI: case F_PHI_HAT: Fo = V; Fi = 1; dst = hat ? (void*)hat4[level] : (void*)phys4[level]; break;
      case F_PSI: case F_PSI_HAT: Fo = V; Fi = 1; dst = hat ? (void*)(hat4[level] + VH) : (void*)(phys4[level] + VP); break;
      case F_MU: case F_MU_HAT: Fo = V; Fi = 1; dst = hat ? (void*)(hat4[level] + 2 * VH) : (void*)(phys4[level] + 2 * VP); break;
      case F_NU: case F_NU_HAT: Fo = V; Fi = 1; dst = hat ? (void*)(hat4[level] + 3 * VH) : (void*)(phys4[level] + 3 * VP); break;
      case F_U: case F_U_HAT: Fo = R; Fi = nd; dst = hat ? (void*)uhat[level] : (void*)uphys[level]; break;
      case F_P: case F_P_HAT: Fo = R; Fi = 1; dst = hat ? (void*)(uhat[level] + nd * RH) : (void*)(uphys[level] + nd * RP); break;
      default: throw std::runtime_error("unknown field id");
    }
    size_t nbytes = hat ? (size_t)Fo * Fi * rows * g.nkx * 16 : (size_t)Fo * Fi * g.P * 8;
    if (dir == 0) VSAV_CUDA(cudaMemcpyAsync(stage, host, nbytes, is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    long long tot = hat ? (long long)Fo * Fi * rows * g.nkx : (long long)Fo * Fi * g.P;
    if (hat) { k_import_hat<T><<<gridfor(tot), 256, 0, st>>>(stage, (C*)dst, Fo, Fi, rows, g.nkx, g.kp, dir); VSAV_COUNT_LAUNCH(); }
    else { k_import_real<T><<<gridfor(tot), 256, 0, st>>>(stage, (T*)dst, Fo, Fi, g.P, dir); VSAV_COUNT_LAUNCH(); }
    VSAV_LAUNCH_CHECK();
    if (dir == 1) VSAV_CUDA(cudaMemcpyAsync(host, stage, nbytes, cudaMemcpyDeviceToHost, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
  }
  void set_field(int level, int fid, const void* host, int is_device) override { xfer(level, fid, (void*)host, 0, is_device); }
  void get_field(int level, int fid, void* host) override { xfer(level, fid, host, 1); }
  void export_f32(int level, int what, float* host) override {
    const int V = dm.V, R = dm.R, nd = g.nd;
    const long long VP = (long long)V * g.P, RP = (long long)R * g.P;
    float* out = reinterpret_cast<float*>(stage);
    long long n = RP;
    const T* src = nullptr;
    if (what != 0 && what != 1) {
      switch (what - 100) {
        case F_PHI: src = phys4[level]; n = VP; break;
        case F_PSI: src = phys4[level] + VP; n = VP; break;
        case F_MU: src = phys4[level] + 2 * VP; n = VP; break;
        case F_NU: src = phys4[level] + 3 * VP; n = VP; break;
        case F_U: src = uphys[level]; n = nd * RP; break;          // [nd][R][P] on the device
        case F_P: src = uphys[level] + nd * RP; n = RP; break;
        default: throw std::runtime_error("export: physical-space fields only");
      }
    }
    if ((size_t)n * sizeof(float) > stage_bytes) throw std::runtime_error("export larger than the staging buffer");
    if (src) { k_to_f32<T><<<gridfor(n), 256, 0, st>>>(src, out, n); VSAV_COUNT_LAUNCH(); }
    else { k_export_run<T><<<gridfor(n), 256, 0, st>>>(phys4[level], uphys[level], d_vbeg, what, R, nd, g.P, out); VSAV_COUNT_LAUNCH(); }
    VSAV_LAUNCH_CHECK();
    if (what == 100 + F_U && R > 1) {
      // host order [R][nd][P] (vsav_get_field's), one copy per (run, component)
      for (int r = 0; r < R; ++r)
        for (int d = 0; d < nd; ++d)
          VSAV_CUDA(cudaMemcpyAsync(host + ((long long)r * nd + d) * g.P, out + ((long long)d * R + r) * g.P,
                                    g.P * sizeof(float), cudaMemcpyDeviceToHost, st));
    } else {
      VSAV_CUDA(cudaMemcpyAsync(host, out, n * sizeof(float), cudaMemcpyDeviceToHost, st));
    }
    VSAV_CUDA(cudaStreamSynchronize(st));
  }
  void set_scalars(int level, const double* q4) override {
    VSAV_CUDA(cudaMemcpyAsync(sc[level], q4, 4 * dm.R * sizeof(double), cudaMemcpyHostToDevice, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
  }
  void get_scalars(int level, double* q4) override {
    VSAV_CUDA(cudaMemcpyAsync(q4, sc[level], 4 * dm.R * sizeof(double), cudaMemcpyDeviceToHost, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
  }
  void set_dt(const double* dt) override {
    VSAV_CUDA(cudaMemcpyAsync(d_dt, dt, dm.R * sizeof(double), cudaMemcpyHostToDevice, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
  }
  void get_dt(double* dt) override {
    VSAV_CUDA(cudaMemcpyAsync(dt, d_dt, dm.R * sizeof(double), cudaMemcpyDeviceToHost, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
  }
  void set_A0(const double* a0) override {
    VSAV_CUDA(cudaMemcpyAsync(d_A0, a0, dm.V * sizeof(double), cudaMemcpyHostToDevice, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
  }
  void get_A0(double* a0) override {
    VSAV_CUDA(cudaMemcpyAsync(a0, d_A0, dm.V * sizeof(double), cudaMemcpyDeviceToHost, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
  }

  // intermediate results, for the step-level API and parity tests
  //  what 0: Step1Cache field idx (0..15, cache order), 1: Step3 field idx (s3 order), 2: u_tilde hat (idx 0/1),
  //       3: u_tilde physical (idx 0/1), 4: H fields physical (H1,H2,H3,G)
  void get_work(int what, int idx, void* host) override {
    const int V = dm.V, R = dm.R, nd = g.nd;
    const long long VH = (long long)V * g.H, VP = (long long)V * g.P, RH = (long long)R * g.H, RP = (long long)R * g.P;
    long long rows = (long long)g.Nz * g.Ny;
    if (what == 0 || what == 1 || what == 2) {
      const C* src = what == 0 ? cache + idx * VH : (what == 1 ? s3 + idx * VH : uth + idx * nd * RH);
      int Fo = what == 2 ? R : V, Fi = what == 2 ? nd : 1;
      k_import_hat<T><<<gridfor((long long)Fo * Fi * rows * g.nkx), 256, 0, st>>>(stage, (C*)src, Fo, Fi, rows, g.nkx, g.kp, 1); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      VSAV_CUDA(cudaMemcpyAsync(host, stage, (size_t)Fo * Fi * rows * g.nkx * 16, cudaMemcpyDeviceToHost, st));
    } else {
      const T* src = what == 3 ? utp + idx * nd * RP : H4 + idx * VP;
      int Fo = what == 3 ? R : V, Fi = what == 3 ? nd : 1;
      k_import_real<T><<<gridfor((long long)Fo * Fi * g.P), 256, 0, st>>>(stage, (T*)src, Fo, Fi, g.P, 1); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      VSAV_CUDA(cudaMemcpyAsync(host, stage, (size_t)Fo * Fi * g.P * 8, cudaMemcpyDeviceToHost, st));
    }
    VSAV_CUDA(cudaStreamSynchronize(st));
  }
  //  what 0: step-2 R values [R][6]; 1: Q [R]; 2: theta [R][2]; 3: A (last area) [V]; 4: M_max [R];
  //       5: psi solver stats [3R][4] (iters, solved, status, rnorm/eps)
  void get_scalar_work(int what, double* out) override {
    const int R = dm.R, V = dm.V;
    if (what == 5) {
      if (!bst) throw std::runtime_error("this handle has no psi BiCGSTAB (3D with constant mobility)");
      std::vector<BiState> hb(3 * R);
      VSAV_CUDA(cudaMemcpyAsync(hb.data(), bst, 3 * R * sizeof(BiState), cudaMemcpyDeviceToHost, st));
      VSAV_CUDA(cudaStreamSynchronize(st));
      for (int s = 0; s < 3 * R; ++s) {
        out[4 * s] = hb[s].iters; out[4 * s + 1] = hb[s].solved; out[4 * s + 2] = hb[s].status;
        out[4 * s + 3] = hb[s].rnorm / std::max(hb[s].eps, 1e-300);
      }
      return;
    }
    if (what == 6) {
      if (!d_true_res) throw std::runtime_error("this handle has no psi BiCGSTAB (3D with constant mobility)");
      VSAV_CUDA(cudaMemcpyAsync(out, d_true_res, 3 * R * sizeof(double), cudaMemcpyDeviceToHost, st));
      VSAV_CUDA(cudaStreamSynchronize(st));
      return;
    }
    const double* src = what == 0 ? r2 : (what == 1 ? qv : (what == 2 ? theta : (what == 3 ? area : mmax_r)));
    size_t n = what == 0 ? 6 * R : (what == 2 ? 2 * R : (what == 3 ? V : R));
    VSAV_CUDA(cudaMemcpyAsync(out, src, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
  }

  // standalone transforms on host/device double buffers (for parity tests of the FFT layer)
  //  kind 0: rfft  [nf][Nz][Ny][Nx] -> [nf][Nz][Ny][nkx] complex
  //  kind 1: irfft (inverse of the above, normalised)
  //  kind 10+m: irfft of Mult m * input
  void transform(int kind, int nf, const double* in, double* out) override {
    const long long rows = (long long)g.Nz * g.Ny;
    if ((long long)nf > 3LL * dm.V) throw std::runtime_error("transform batch too large");
    T* rbuf = tmpP;
    C* hbuf = rhs;
    if (kind == 0) {
      VSAV_CUDA(cudaMemcpyAsync(stage, in, (size_t)nf * g.P * 8, cudaMemcpyDefault, st));
      k_import_real<T><<<gridfor(nf * g.P), 256, 0, st>>>(stage, rbuf, nf, 1, g.P, 0); VSAV_COUNT_LAUNCH();
      rfft(rbuf, nf, hbuf);
      k_import_hat<T><<<gridfor(nf * rows * g.nkx), 256, 0, st>>>(stage, hbuf, nf, 1, rows, g.nkx, g.kp, 1); VSAV_COUNT_LAUNCH();
      VSAV_CUDA(cudaMemcpyAsync(out, stage, (size_t)nf * rows * g.nkx * 16, cudaMemcpyDefault, st));
    } else {
      int mult = kind == 1 ? M_ONE : kind - 10;
      VSAV_CUDA(cudaMemcpyAsync(stage, in, (size_t)nf * rows * g.nkx * 16, cudaMemcpyDefault, st));
      VSAV_CUDA(cudaMemsetAsync(hbuf, 0, (size_t)nf * g.H * sizeof(C), st));
      k_import_hat<T><<<gridfor(nf * rows * g.nkx), 256, 0, st>>>(stage, hbuf, nf, 1, rows, g.nkx, g.kp, 0); VSAV_COUNT_LAUNCH();
      irfft(hbuf, nf, rbuf, mult);
      k_import_real<T><<<gridfor(nf * g.P), 256, 0, st>>>(stage, rbuf, nf, 1, g.P, 1); VSAV_COUNT_LAUNCH();
      VSAV_CUDA(cudaMemcpyAsync(out, stage, (size_t)nf * g.P * 8, cudaMemcpyDefault, st));
    }
    VSAV_LAUNCH_CHECK();
    VSAV_CUDA(cudaStreamSynchronize(st));
  }

  StepStatus status() override {
    StepStatus s;
    int e = 0;
    VSAV_CUDA(cudaMemcpyAsync(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
    s.err_flags = e;
    if (psi32) {                                           // the FP32 helper's kernels flag into its own word
      int e2 = 0;
      VSAV_CUDA(cudaMemcpyAsync(&e2, psi32->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
      VSAV_CUDA(cudaStreamSynchronize(st));
      s.err_flags |= e2;
    }
    if (bst) {                                             // a Krylov psi solve exists (2D, or 3D variable mobility)
      int S = 3 * dm.R;
      std::vector<BiState> hb(S);
      VSAV_CUDA(cudaMemcpyAsync(hb.data(), bst, S * sizeof(BiState), cudaMemcpyDeviceToHost, st));
      VSAV_CUDA(cudaStreamSynchronize(st));
      s.psi_systems = S;
      for (auto& b : hb) {
        s.psi_max_iters = std::max(s.psi_max_iters, b.iters);
        if (!b.solved) s.psi_not_converged++;
      }
    }
    return s;
  }
  void sync() override { VSAV_CUDA(cudaStreamSynchronize(st)); }
  // the FP32 psi helper of the mixed mode is profiled with its owner
  void profile(int enable) override {
    VSAV_CUDA(cudaStreamSynchronize(st));
    if (psi32) psi32->profile(enable);
    if (enable == 2) { prof.reset(); return; }
    prof.collect();
    prof.enable(enable != 0);
  }
  void profile_read(int cls, double* out3) override {
    VSAV_CUDA(cudaStreamSynchronize(st));
    prof.collect();
    out3[0] = (double)prof.launches[cls]; out3[1] = prof.ms[cls]; out3[2] = prof.bytes[cls];
    if (psi32) {
      double o[3];
      psi32->profile_read(cls, o);
      out3[0] += o[0]; out3[1] += o[1]; out3[2] += o[2];
    }
  }
  cudaStream_t stream() override { return st; }
};

// Mixed precision (FP64 fields): b (FP64, full spectrum) -> x by sweeps of
//   r = b - A x (FP64 operator, no preconditioner);  A d = r solved by the
//   FP32 helper's BiCGSTAB;  x += d, over enough sweeps that the product of the
//   sweeps' relative tolerances (each >= psi_inner_rtol) reaches psi_rtol.
// The FP32 solve does most of the work; the FP64 residual keeps the result at
// FP64 accuracy after a few sweeps (classical iterative refinement).
template <typename T>
void Solver<T>::psi_solve_mixed() {
  if constexpr (std::is_same<T, double>::value) {
    Solver<float>* H = psi32;
    const int V = dm.V, R = dm.R;
    const long long F = 3LL * V, n = psi_n(), VP = (long long)V * g.P;
    const long long nc = F * n;
    k_cast<double, float><<<gridfor(VP), 256, 0, st>>>(Mpsi, H->Mpsi, VP); VSAV_COUNT_LAUNCH();
    VSAV_CUDA(cudaMemcpyAsync(H->mmax_r, mmax_r, R * sizeof(double), cudaMemcpyDeviceToDevice, st));
    VSAV_CUDA(cudaMemcpyAsync(H->d_adt, d_adt, R * sizeof(double), cudaMemcpyDeviceToDevice, st));
    psi_prepare_b();
    C* x = psi_x();
    VSAV_CUDA(cudaMemsetAsync(x, 0, nc * sizeof(C), st));
    VSAV_CUDA(cudaMemsetAsync(bupd, 0xff, 3 * R * sizeof(int), st));     // every system active in A x
    // the requested relative tolerance is split over the sweeps, each FP32 solve
    // reaching at most 1e-6 (rtol 1e-12: two sweeps at 1e-6; 1e-8: two at 1e-4)
    const double rt = std::min(std::max(opt.psi_rtol, 1e-15), 0.5);
    const int nsw = std::max(std::max(1, (int)std::ceil(std::log(rt) / std::log(opt.psi_inner_rtol) - 1e-9)),
                             opt.psi_refine_min);
    const double inner = std::pow(rt, 1.0 / nsw);
    for (int ref = 0; ref < nsw; ++ref) {
      const C* r = vb;
      if (ref > 0) {
        VSAV_CUDA(cudaMemsetAsync(bupd, 0xff, 3 * R * sizeof(int), st));
        matvec(x, vt, 0, nullptr, false);
        k_sub<C><<<gridfor(nc), 256, 0, st>>>(vb, vt, vs, nc); VSAV_COUNT_LAUNCH();
        r = vs;
      }
      k_cast<double2, float2><<<gridfor(nc), 256, 0, st>>>(r, H->vb, nc); VSAV_COUNT_LAUNCH();
      H->psi_krylov(H->psi_x(), inner, opt.psi_itmax);
      k_add_cast<float2, double2><<<gridfor(nc), 256, 0, st>>>(H->psi_x(), x, nc); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
    }
    VSAV_CUDA(cudaMemcpyAsync(bst, H->bst, 3 * R * sizeof(BiState), cudaMemcpyDeviceToDevice, st));
    if (opt.psi_check) psi_check_residual(x);
    psi_finish();
  }
}

// The two instantiations are compiled in their own translation units
// (solver_f32.cu, solver_f64.cu); the C ABI creates them through these.
SolverBase* make_solver_f32(const Dims& d, const Phys& p, const Options& o, const int* run_sizes, const double* psi_in,
                            const double* psi_out);
SolverBase* make_solver_f64(const Dims& d, const Phys& p, const Options& o, const int* run_sizes, const double* psi_in,
                            const double* psi_out);

}  // namespace vsav
