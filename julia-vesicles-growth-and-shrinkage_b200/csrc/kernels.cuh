// Fused pointwise kernels of the SAV step (physical space and k space), the
// compensated FP64 reductions behind every SAV inner product, the per-run
// scalar solves (R1..R3 3x3 systems, Q equation) and the psi BiCGSTAB vector
// kernels.  Reference formulas are cited next to each kernel.
#pragma once
#include "fft.cuh"

namespace vsav {

constexpr double SQ2 = 1.41421356237309504880;

// physical parameters shared by all runs of a handle (Config, Types.jl:27-74)
struct Phys {
  double eps, M_phi, M0_psi, eta, gamma_surf, gamma_area, gamma_bend;
  double gamma_in, beta_in, gamma_out, beta_out, lamda;
  double S1, S2, S3, S4, C1, C2, C3;
  double cell;      // dx*dy(*dz)
  double conf_dt;   // conf.dt (used by the 3D Step 5, Solvers_3d.jl:386-387)
};

// run / vesicle bookkeeping
struct Runs {
  int V, R;
  const int* run_of;      // [V]
  const int* vbeg;        // [R+1] first vesicle of run r (vesicles of a run are contiguous)
  const double* psi_in;   // [V]
  const double* psi_out;  // [V]
};

// ---------------------------------------------------------------------------
// elementwise launch geometry: grid (bpf, F); block b of field f covers
// elements [b*chunk, (b+1)*chunk) of that field.  Partial sums go to
// part[(f*bpf + b)*K + k].
// ---------------------------------------------------------------------------
struct EW {
  long long n;     // elements per field
  int bpf;         // blocks per field
  long long chunk; // elements per block
};

#define EW_LOOP(ew, f, i)                                                     \
  const int f = blockIdx.y;                                                   \
  const long long i##_beg = (long long)blockIdx.x * (ew).chunk;               \
  const long long i##_end = min((ew).n, i##_beg + (ew).chunk);                \
  for (long long i = i##_beg + threadIdx.x; i < i##_end; i += blockDim.x)

template <int K>
__device__ __forceinline__ void ew_store_partials(KSum (&acc)[K], double2* part, const EW& ew, double* sm) {
  block_reduce_store<K>(acc, part + ((long long)blockIdx.y * ew.bpf + blockIdx.x) * K, sm);
}

// per-field totals: out[f*K + k] = sum over blocks of field f (compensated)
static __global__ void k_fin_fields(const double2* __restrict__ part, int bpf, int K, double* __restrict__ out) {
  const int f = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = warp; k < K; k += nw) {
    KSum a{0.0, 0.0};
    for (int b = lane; b < bpf; b += 32) {
      double2 p = part[((long long)f * bpf + b) * K + k];
      a.merge(p.x, p.y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double s2 = __shfl_down_sync(0xffffffffu, a.s, o);
      double c2 = __shfl_down_sync(0xffffffffu, a.c, o);
      if (lane + o < 32) a.merge(s2, c2);
    }
    if (lane == 0) out[f * K + k] = a.val();
  }
}

// per-field maxima (partials hold max in .x)
static __global__ void k_fin_max(const double2* __restrict__ part, int bpf, int K, int k0, double* __restrict__ out) {
  const int f = blockIdx.x;
  double m = -INFINITY;
  for (int b = threadIdx.x; b < bpf; b += blockDim.x) m = fmax(m, part[((long long)f * bpf + b) * K + k0].x);
  m = warp_max(m);
  if (threadIdx.x == 0) out[f] = m;
}

// ---------------------------------------------------------------------------
// small device helpers for the reference's scalar functions (Utils.jl:8-20)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double g_(double p) { double t = p * p - 1.0; return 0.25 * t * t; }
__device__ __forceinline__ double gp_(double p) { return p * (p * p - 1.0); }
__device__ __forceinline__ double pphi_(double p) { return -0.5 * p * p * p + 1.5 * p; }
__device__ __forceinline__ double pphip_(double p) { return -1.5 * p * p + 1.5; }

// ---------------------------------------------------------------------------
// Step 1 prologue: phi* = 2 phi - phi_old, psi* likewise, M_psi(phi*)
// (Solvers.jl:21-27, Utils.jl:20), and the W3 integrands at (phi*, psi*)
// (Utils.jl:53-60,184-190).  sums: [0] max M, [1] f_osm, [2] psi^2
// When phi_old == nullptr the inputs are used as they are (initialisation).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_star(const T* __restrict__ phi, const T* __restrict__ phio,
                                              const T* __restrict__ psi, const T* __restrict__ psio,
                                              T* __restrict__ phis, T* __restrict__ psis, T* __restrict__ Mpsi,
                                              Phys ph, Runs rn, EW ew, double2* part) {
  __shared__ double sm[2 * 3 * 32];
  KSum acc[3] = {{-INFINITY, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
  double mmax = -INFINITY;
  const int f0 = blockIdx.y;
  const double pin = rn.psi_in[f0], pout = rn.psi_out[f0];
  EW_LOOP(ew, f, i) {
    long long j = (long long)f * ew.n + i;
    double a, s;
    if (phio) { a = 2.0 * (double)phi[j] - (double)phio[j]; s = 2.0 * (double)psi[j] - (double)psio[j]; }
    else { a = phi[j]; s = psi[j]; }
    T aT = (T)a, sT = (T)s;
    if (phis) { phis[j] = aT; psis[j] = sT; }
    double ad = aT, sd = sT;   // what later kernels see
    if (Mpsi) {
      double t = ad * ad - 1.0;
      double m = 0.1 * (1.0 - ph.M0_psi * t * t);
      Mpsi[j] = (T)m;
      mmax = fmax(mmax, (double)(T)m);
    }
    double P = pphi_(ad);
    double fin = 0.5 * ph.gamma_in * (sd - pin) * (sd - pin) + ph.beta_in;
    double fout = 0.5 * ph.gamma_out * (sd - pout) * (sd - pout) + ph.beta_out;
    acc[1].add(((1.0 + P) / 2.0) * fin + ((1.0 - P) / 2.0) * fout);
    acc[2].add(sd * sd);
  }
  // max reduction rides in slot 0 (.s = running max, .c = 0)
  acc[0].s = mmax; acc[0].c = 0.0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double m = warp_max(acc[0].s);
  acc[0].s = 0.0;
  block_reduce_store<3>(acc, part + ((long long)blockIdx.y * ew.bpf + blockIdx.x) * 3, sm);
  __syncthreads();
  if (lane == 0) sm[warp] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = -INFINITY;
    for (int w = 0; w < nw; ++w) mm = fmax(mm, sm[w]);
    part[((long long)blockIdx.y * ew.bpf + blockIdx.x) * 3].x = mm;
    part[((long long)blockIdx.y * ew.bpf + blockIdx.x) * 3].y = 0.0;
  }
}

// u* = 2u - u_old for the velocity components  ([nd][R][P] contiguous)
template <typename T>
__global__ void k_axpby(const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ y, double ca, double cb, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = (T)(ca * (double)a[i] + cb * (double)b[i]);
}

// ---------------------------------------------------------------------------
// surface/bending integrands and omega (Utils.jl:36-50,148-153,166-182)
// sums: [0] f_surf, [1] f_bend, [2] E2 integrand.  out: omega
// (the 3D file uses only the x,y gradients in f_surf and E2: Utils_3d.jl:36-42,175-177)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_surf(const T* __restrict__ phi, const T* __restrict__ gx, const T* __restrict__ gy,
                                              const T* __restrict__ lap, T* __restrict__ omega, Phys ph, EW ew, double2* part) {
  __shared__ double sm[2 * 3 * 32];
  KSum acc[3] = {{0, 0}, {0, 0}, {0, 0}};
  const double e = ph.eps;
  EW_LOOP(ew, f, i) {
    long long j = (long long)f * ew.n + i;
    double p = phi[j], x = gx[j], y = gy[j];
    double fs = (3.0 * SQ2 / 4.0) * (g_(p) / e) + e * (x * x + y * y) / 2.0;
    acc[0].add(fs);
    if (lap) {
      double l = lap[j];
      double t = gp_(p) / e - e * l;
      acc[1].add((3.0 * SQ2 / (16.0 * e)) * t * t);
      acc[2].add(0.5 * ph.S1 * l * l + 0.5 * ph.S2 * (x * x + y * y) + 0.5 * ph.S3 * p * p);
      if (omega) omega[j] = (T)((p * p * p - p) / e - e * l);
    }
  }
  ew_store_partials<3>(acc, part, ew, sm);
}

// per-vesicle sum of the surface energy density f_surf (Utils.jl:36-42): the
// single code path behind every area (A0 at initialisation, A in Steps 1/2),
// so A - A0 is exactly 0 when phi is unchanged, as in the reference
template <typename T>
__global__ void __launch_bounds__(256) k_area(const T* __restrict__ phi, const T* __restrict__ gx, const T* __restrict__ gy,
                                              Phys ph, EW ew, double2* part) {
  __shared__ double sm[2 * 1 * 8];
  KSum acc[1] = {{0, 0}};
  const double e = ph.eps;
  EW_LOOP(ew, f, i) {
    long long j = (long long)f * ew.n + i;
    double p = phi[j], x = gx[j], y = gy[j];
    acc[0].add((3.0 * SQ2 / 4.0) * (g_(p) / e) + e * (x * x + y * y) / 2.0);
  }
  ew_store_partials<1>(acc, part, ew, sm);
}

// per-run SAV normalisers of the H functions (Utils.jl:159-206,228-248):
//  asum[v] = f_surf sums, fs[v*3+1..2] = (f_bend, E2) sums, fo[v*3+1..2] = (f_osm, psi^2) sums,
//  Mmax_v[v] = block maxima.  Writes sc[r*8 + 0..7] = (R1s, R2s, R3s, Mmax, W1, W2, W3, -)
//  and factor[v], area[v].  err |= 1/2/4 when W_i + C_i < 0.
static __global__ void k_fin_H(const double* __restrict__ asum, const double* __restrict__ fs, const double* __restrict__ fo,
                        const double* __restrict__ mmax_v, const double* __restrict__ A0, Phys ph, Runs rn, double* __restrict__ sc,
                        double* __restrict__ factor, double* __restrict__ area, int* __restrict__ err) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rn.R) return;
  double W1 = 0, Ssurf = 0, Sbend = 0, Se2 = 0, Sosm = 0, Spsi = 0, mm = -INFINITY;
  for (int v = rn.vbeg[r]; v < rn.vbeg[r + 1]; ++v) {
    double A = asum[v] * ph.cell;
    area[v] = A;
    double d = A - A0[v];
    W1 += 0.5 * ph.gamma_area * d * d;
    factor[v] = ph.gamma_area * d * (3.0 * SQ2 / 4.0);
    Ssurf += asum[v]; Sbend += fs[v * 3 + 1]; Se2 += fs[v * 3 + 2];
    Sosm += fo[v * 3 + 1]; Spsi += fo[v * 3 + 2];
    if (mmax_v) mm = fmax(mm, mmax_v[v]);
  }
  double W2 = ph.gamma_surf * (Ssurf * ph.cell) + ph.gamma_bend * (Sbend * ph.cell) - Se2 * ph.cell;
  double W3 = Sosm * ph.cell - 0.5 * ph.S4 * (Spsi * ph.cell);
  int e = 0;
  if (W1 + ph.C1 < 0) e |= 1;
  if (W2 + ph.C2 < 0) e |= 2;
  if (W3 + ph.C3 < 0) e |= 4;
  if (e) atomicOr(err, e);
  sc[r * 8 + 0] = sqrt(W1 + ph.C1);
  sc[r * 8 + 1] = sqrt(W2 + ph.C2);
  sc[r * 8 + 2] = sqrt(W3 + ph.C3);
  sc[r * 8 + 3] = mm;
  sc[r * 8 + 4] = W1; sc[r * 8 + 5] = W2; sc[r * 8 + 6] = W3;
}

// H1, H2, H3, MG at (phi, psi)  (Utils.jl:198-248); out: H4 = [H1|H2|H3|G] each [V][P]
template <typename T>
__global__ void __launch_bounds__(256) k_H(const T* __restrict__ phi, const T* __restrict__ psi, const T* __restrict__ omega,
                                           const T* __restrict__ lapomega, const T* __restrict__ lap, const T* __restrict__ bih,
                                           const double* __restrict__ sc, const double* __restrict__ factor,
                                           T* __restrict__ H4, long long VP, Phys ph, Runs rn, EW ew) {
  const int v = blockIdx.y;
  const int r = rn.run_of[v];
  const double R1 = sc[r * 8 + 0], R2 = sc[r * 8 + 1], R3 = sc[r * 8 + 2];
  const double fac = factor[v], pin = rn.psi_in[v], pout = rn.psi_out[v], e = ph.eps;
  EW_LOOP(ew, f, i) {
    long long j = (long long)f * ew.n + i;
    double p = phi[j], s = psi[j], w = omega[j], lw = lapomega[j], l = lap[j], b = bih[j];
    double h1 = (fac * w) / R1;
    double sb = ph.gamma_surf * (3.0 * SQ2 / 4.0) * w +
                ph.gamma_bend * (3.0 * SQ2 / (8.0 * e)) * (w * (3.0 * p * p - 1.0) / e - e * lw);
    double lin = ph.S1 * b - ph.S2 * l + ph.S3 * p;
    double h2 = (sb - lin) / R2;
    double fin = 0.5 * ph.gamma_in * (s - pin) * (s - pin) + ph.beta_in;
    double fout = 0.5 * ph.gamma_out * (s - pout) * (s - pout) + ph.beta_out;
    double h3 = (0.5 * pphip_(p) * (fin - fout)) / R3;
    double P = pphi_(p);
    double G1 = 0.5 * (1.0 + P) * (ph.gamma_in * (s - pin)) + 0.5 * (1.0 - P) * (ph.gamma_out * (s - pout));
    double G = (G1 - ph.S4 * s) / R3;
    H4[j] = (T)h1; H4[VP + j] = (T)h2; H4[2 * VP + j] = (T)h3; H4[3 * VP + j] = (T)G;
  }
}

// y[j] = M[j] * x[j] (each of nf fields of [V][P], M indexed by vesicle)  or  y = c*x (M == nullptr)
template <typename T>
__global__ void k_mul_field(const T* __restrict__ x, const T* __restrict__ M, double c, T* __restrict__ y,
                            long long VP, int nf) {
  long long n = VP * nf;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = M ? (T)((double)M[i % VP] * (double)x[i]) : (T)(c * (double)x[i]);
}

// advection u*.grad(f) for nf2 vesicle fields: out[q][v] = sum_d u*_d[run(v)] * g[q][d][v]
// g layout: [nq][nd][V][P]; ustar: [nd][R][P]
template <typename T>
__global__ void k_advect(const T* __restrict__ g, const T* __restrict__ ustar, T* __restrict__ out, int nq, int nd,
                         Runs rn, long long P) {
  long long VP = (long long)rn.V * P;
  long long n = VP * nq;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int q = (int)(i / VP);
    long long j = i - (long long)q * VP;
    int v = (int)(j / P);
    long long pix = j - (long long)v * P;
    int r = rn.run_of[v];
    double acc = 0.0;
    for (int d = 0; d < nd; ++d)
      acc += (double)ustar[((long long)d * rn.R + r) * P + pix] * (double)g[((long long)(q * nd + d)) * VP + j];
    out[i] = (T)acc;
  }
}

// ---------------------------------------------------------------------------
// k-space helpers
// ---------------------------------------------------------------------------
struct KI {
  int kx, ky, kz;
  double kxv, kyv, kzv;
  __device__ double k2() const { return kxv * kxv + kyv * kyv + kzv * kzv; }
};
__device__ __forceinline__ KI kdecode(long long s, const Geom& g) {
  KI k;
  k.kx = (int)(s % g.kp);
  long long row = s / g.kp;
  k.ky = (int)(row % g.Ny);
  k.kz = (int)(row / g.Ny);
  k.kxv = k.kx * g.kxs;
  k.kyv = kfreq(k.ky, g.Ny) * g.kys;
  k.kzv = (g.nd == 3) ? kfreq(k.kz, g.Nz) * g.kzs : 0.0;
  return k;
}
template <typename C>
__device__ __forceinline__ C d1(const KI& k, int d) { double v = d == 0 ? k.kxv : (d == 1 ? k.kyv : k.kzv); return mk<C>(0.0, v); }

#define K_LOOP(n, i) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// Step 1 k-space assembly (Solvers.jl:85-134, Solvers_3d.jl:35-89)
//  hat4 levels: present/old [4][V][H] (phi, psi, mu, nu).  Hh: [4][V][H] (H1,H2,H3,G hats)
//  fl: [2][V][H] flux hats (2D: rfft(M dG/dx), rfft(M dG/dy); 3D: unused, fl3 has 3)
//  adv: [2][V][H] rfft(u*.grad phi*), rfft(u*.grad psi*)
//  cache: [16][V][H] order phi11 phi12 phi13 phi14 phi21 psi11 psi12 psi21 mu11 mu12 mu13 mu14 mu21 nu11 nu12 nu21
//  rhs: [3][V][H] psi right-hand sides (11, 12, 21); 3D: solves directly (lhs_psi) and writes psi/nu.
template <typename T>
__global__ void k_step1_k(const cplx<T>* __restrict__ hp, const cplx<T>* __restrict__ ho, const cplx<T>* __restrict__ Hh,
                          const cplx<T>* __restrict__ fl, int nfl, const cplx<T>* __restrict__ adv,
                          cplx<T>* __restrict__ cache, cplx<T>* __restrict__ rhs,
                          const double* __restrict__ dtv, double a, double b, double c, Phys ph, Runs rn, Geom g,
                          int psi_div) {
  using C = cplx<T>;
  const long long VH = (long long)rn.V * g.H;
  K_LOOP(VH, i) {
    int v = (int)(i / g.H);
    long long s = i - (long long)v * g.H;
    KI k = kdecode(s, g);
    if (k.kx >= g.nkx) continue;
    double dt = dtv[rn.run_of[v]];
    double K2 = k.k2();
    double Lap = -K2, Bih = K2 * K2;
    double Lphi = ph.S1 * Bih - ph.S2 * Lap + ph.S3;
    double lhs = (a / dt) + ph.M_phi * Lphi;
    auto ld = [&](const C* p) { C z = p[i]; return make_double2((double)z.x, (double)z.y); };
    auto st = [&](int slot, double2 z) { C o; o.x = (decltype(o.x))z.x; o.y = (decltype(o.y))z.y; cache[slot * VH + i] = o; };
    double2 ph_p = ld(hp), ph_o = ld(ho), ps_p = ld(hp + VH), ps_o = ld(ho + VH);
    double2 H1 = ld(Hh), H2 = ld(Hh + VH), H3 = ld(Hh + 2 * VH), Gh = ld(Hh + 3 * VH);
    // 11
    double2 r11 = -(1.0 / dt) * (b * ph_p + c * ph_o);
    r11 = (1.0 / 1.0) * r11;
    double2 p11 = make_double2(r11.x / lhs, r11.y / lhs);
    st(0, p11); st(8, Lphi * p11);
    double2 rp = -(1.0 / dt) * (b * ps_p + c * ps_o);
    // 12
    double2 p12 = make_double2((-ph.M_phi * H1.x) / lhs, (-ph.M_phi * H1.y) / lhs);
    st(1, p12); st(9, Lphi * p12 + H1);
    // 13, 14
    double2 p13 = make_double2((-ph.M_phi * H2.x) / lhs, (-ph.M_phi * H2.y) / lhs);
    double2 p14 = make_double2((-ph.M_phi * H3.x) / lhs, (-ph.M_phi * H3.y) / lhs);
    st(2, p13); st(3, p14); st(10, Lphi * p13 + H2); st(11, Lphi * p14 + H3);
    // 21
    double2 A = ld(adv), B = ld(adv + VH);
    double2 p21 = make_double2(-A.x / lhs, -A.y / lhs);
    st(4, p21); st(12, Lphi * p21);
    // psi right-hand sides: D1 . flux
    double2 f12 = make_double2(0, 0);
    for (int d = 0; d < nfl; ++d) {
      double2 fd = ld(fl + d * VH);
      double kv = d == 0 ? k.kxv : (d == 1 ? k.kyv : k.kzv);
      f12 = f12 + make_double2(-kv * fd.y, kv * fd.x);
    }
    double2 r21 = make_double2(-B.x, -B.y);
    if (!psi_div) {                       // right-hand sides of the psi BiCGSTAB
      C o;
      o.x = rp.x; o.y = rp.y; rhs[i] = o;
      o.x = f12.x; o.y = f12.y; rhs[VH + i] = o;
      o.x = r21.x; o.y = r21.y; rhs[2 * VH + i] = o;
    } else {
      // 3D: psi = rhs / (a/dt - M0_psi S4 Lap)   (Solvers_3d.jl:30,40,57,88)
      double lp = (a / dt) - ph.M0_psi * ph.S4 * Lap;
      double2 q11 = make_double2(rp.x / lp, rp.y / lp);
      double2 q12 = make_double2(f12.x / lp, f12.y / lp);
      double2 q21 = make_double2(r21.x / lp, r21.y / lp);
      st(5, q11); st(6, q12); st(7, q21);
      st(13, ph.S4 * q11); st(14, ph.S4 * q12 + Gh); st(15, ph.S4 * q21);
    }
  }
}

// nu = S4 psi (+ G for the 12 split)  (Solvers.jl:92,107,134)
template <typename T>
__global__ void k_nu(cplx<T>* __restrict__ cache, const cplx<T>* __restrict__ Gh, double S4, long long VH, Geom g) {
  K_LOOP(VH, i) {
    long long s = i % g.H;
    if ((int)(s % g.kp) >= g.nkx) continue;
    for (int q = 0; q < 3; ++q) {
      cplx<T> p = cache[(5 + q) * VH + i];
      double2 n = make_double2(S4 * (double)p.x, S4 * (double)p.y);
      if (q == 1) { n.x += (double)Gh[i].x; n.y += (double)Gh[i].y; }
      cplx<T> o; o.x = n.x; o.y = n.y;
      cache[(13 + q) * VH + i] = o;
    }
  }
}

// ---------------------------------------------------------------------------
// Step 2 inner products (Solvers.jl:160-223).  cp: [8][V][P] = irfft of
// (phi11 phi12 phi13 phi14 phi21 psi11 psi12 psi21); H4 = [H1|H2|H3|G]
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256, 2) k_dot2(const T* __restrict__ H4, const T* __restrict__ phi, const T* __restrict__ phio,
                                                 const T* __restrict__ psi, const T* __restrict__ psio, const T* __restrict__ cp,
                                                 double b, double c, long long VP, EW ew, double2* part) {
  __shared__ double sm[2 * 22 * 8];
  KSum acc[22];
#pragma unroll
  for (int k = 0; k < 22; ++k) acc[k] = {0.0, 0.0};
  EW_LOOP(ew, f, i) {
    long long j = (long long)f * ew.n + i;
    double h1 = H4[j], h2 = H4[VP + j], h3 = H4[2 * VP + j], G = H4[3 * VP + j];
    double hph = b * (double)phi[j] + c * (double)phio[j];
    double hps = b * (double)psi[j] + c * (double)psio[j];
    double p11 = cp[j], p12 = cp[VP + j], p13 = cp[2 * VP + j], p14 = cp[3 * VP + j], p21 = cp[4 * VP + j];
    double s11 = cp[5 * VP + j], s12 = cp[6 * VP + j], s21 = cp[7 * VP + j];
    acc[0].add(h1 * hph); acc[1].add(h2 * hph); acc[2].add(h3 * hph); acc[3].add(G * hps);
    acc[4].add(h1 * p12); acc[5].add(h1 * p13); acc[6].add(h1 * p14);
    acc[7].add(h2 * p12); acc[8].add(h2 * p13); acc[9].add(h2 * p14);
    acc[10].add(h3 * p12); acc[11].add(h3 * p13); acc[12].add(h3 * p14); acc[13].add(G * s12);
    acc[14].add(h1 * p11); acc[15].add(h2 * p11); acc[16].add(h3 * p11); acc[17].add(G * s11);
    acc[18].add(h1 * p21); acc[19].add(h2 * p21); acc[20].add(h3 * p21); acc[21].add(G * s21);
  }
  ew_store_partials<22>(acc, part, ew, sm);
}

// 3x3 solve by Gaussian elimination with partial pivoting (the LU of Julia's `\`)
__device__ inline void solve3(double A[3][3], double bb[3], double x[3]) {
  int pr[3] = {0, 1, 2};
  double M[3][3];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) M[i][j] = A[i][j];
  double y[3] = {bb[0], bb[1], bb[2]};
  for (int k = 0; k < 3; ++k) {
    int p = k;
    for (int i = k + 1; i < 3; ++i) if (fabs(M[i][k]) > fabs(M[p][k])) p = i;
    if (p != k) {
      for (int j = 0; j < 3; ++j) { double t = M[k][j]; M[k][j] = M[p][j]; M[p][j] = t; }
      double t = y[k]; y[k] = y[p]; y[p] = t;
      int ti = pr[k]; pr[k] = pr[p]; pr[p] = ti;
    }
    for (int i = k + 1; i < 3; ++i) {
      double l = M[i][k] / M[k][k];
      for (int j = k + 1; j < 3; ++j) M[i][j] -= l * M[k][j];
      y[i] -= l * y[k];
    }
  }
  for (int i = 2; i >= 0; --i) {
    double s = y[i];
    for (int j = i + 1; j < 3; ++j) s -= M[i][j] * x[j];
    x[i] = s / M[i][i];
  }
}

// Step 2 scalar solve per run.  scp/sco: [R][4] (Q,R1,R2,R3) present/old.
// out r2[r*6 + 0..5] = R11 R21 R31 R12 R22 R32
static __global__ void k_fin_step2(const double* __restrict__ fd, const double* __restrict__ scp, const double* __restrict__ sco,
                            double a, double b, double c, Phys ph, Runs rn, double* __restrict__ r2) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rn.R) return;
  double D[22];
  for (int k = 0; k < 22; ++k) D[k] = 0.0;
  for (int v = rn.vbeg[r]; v < rn.vbeg[r + 1]; ++v)
    for (int k = 0; k < 22; ++k) D[k] += fd[v * 22 + k];
  const double w = ph.cell;
  double U1 = -(b * scp[r * 4 + 1] + c * sco[r * 4 + 1]) / a + (D[0] * w) / (2.0 * a);
  double U2 = -(b * scp[r * 4 + 2] + c * sco[r * 4 + 2]) / a + (D[1] * w) / (2.0 * a);
  double U3 = -(b * scp[r * 4 + 3] + c * sco[r * 4 + 3]) / a + (D[2] * w + D[3] * w) / (2.0 * a);
  double L[3][3];
  L[0][0] = 1.0 - 0.5 * (D[4] * w); L[0][1] = -0.5 * (D[5] * w); L[0][2] = -0.5 * (D[6] * w);
  L[1][0] = -0.5 * (D[7] * w); L[1][1] = 1.0 - 0.5 * (D[8] * w); L[1][2] = -0.5 * (D[9] * w);
  L[2][0] = -0.5 * (D[10] * w); L[2][1] = -0.5 * (D[11] * w); L[2][2] = 1.0 - 0.5 * (D[12] * w + D[13] * w);
  double B1[3] = {0.5 * (D[14] * w) + U1, 0.5 * (D[15] * w) + U2, 0.5 * (D[16] * w + D[17] * w) + U3};
  double B2[3] = {0.5 * (D[18] * w), 0.5 * (D[19] * w), 0.5 * (D[20] * w + D[21] * w)};
  double x1[3], x2[3];
  solve3(L, B1, x1);
  solve3(L, B2, x2);
  for (int k = 0; k < 3; ++k) { r2[r * 6 + k] = x1[k]; r2[r * 6 + 3 + k] = x2[k]; }
}

// Step 3 (Solvers.jl:242-259).  s3 order: phi1 psi1 phi2 psi2 mu1 nu1 mu2 nu2
template <typename T>
__global__ void k_step3(const cplx<T>* __restrict__ cache, const double* __restrict__ r2, cplx<T>* __restrict__ s3,
                        Runs rn, Geom g) {
  using C = cplx<T>;
  const long long VH = (long long)rn.V * g.H;
  K_LOOP(VH, i) {
    int v = (int)(i / g.H);
    long long s = i - (long long)v * g.H;
    if ((int)(s % g.kp) >= g.nkx) continue;
    const double* R = r2 + rn.run_of[v] * 6;
    double R11 = R[0], R21 = R[1], R31 = R[2], R12 = R[3], R22 = R[4], R32 = R[5];
    auto L = [&](int q) { C z = cache[q * VH + i]; return make_double2(z.x, z.y); };
    auto S = [&](int q, double2 z) { C o; o.x = z.x; o.y = z.y; s3[q * VH + i] = o; };
    double2 p11 = L(0), p12 = L(1), p13 = L(2), p14 = L(3), p21 = L(4), s11 = L(5), s12 = L(6), s21 = L(7);
    double2 m11 = L(8), m12 = L(9), m13 = L(10), m14 = L(11), m21 = L(12), n11 = L(13), n12 = L(14), n21 = L(15);
    S(0, p11 + R11 * p12 + R21 * p13 + R31 * p14);
    S(1, s11 + R31 * s12);
    S(2, p21 + R12 * p12 + R22 * p13 + R32 * p14);
    S(3, s21 + R32 * s12);
    S(4, m11 + R11 * m12 + R21 * m13 + R31 * m14);
    S(5, n11 + R31 * n12);
    S(6, m21 + R12 * m12 + R22 * m13 + R32 * m14);
    S(7, n21 + R32 * n12);
  }
}

// Step 4 k-space (Solvers.jl:284-288,321-324):  u1 = (-(b u + c u_old)/dt - D1 p)/lhs ; u2 /= lhs
//  uh levels [nd+1][R][H] (u components then p);  ut: [2][nd][R][H]
template <typename T>
__global__ void k_step4_k(const cplx<T>* __restrict__ up, const cplx<T>* __restrict__ uo, cplx<T>* __restrict__ ut,
                          const double* __restrict__ dtv, double a, double b, double c, Phys ph, int R, Geom g) {
  using C = cplx<T>;
  const long long RH = (long long)R * g.H;
  K_LOOP(RH, i) {
    int r = (int)(i / g.H);
    long long s = i - (long long)r * g.H;
    KI k = kdecode(s, g);
    if (k.kx >= g.nkx) continue;
    double dt = dtv[r];
    double lhs = (a / dt) - ph.eta * (-k.k2());
    C pz = up[g.nd * RH + i];
    double2 p = make_double2(pz.x, pz.y);
    for (int d = 0; d < g.nd; ++d) {
      C u = up[d * RH + i], w = uo[d * RH + i];
      double2 r1 = -(1.0 / dt) * make_double2(b * (double)u.x + c * (double)w.x, b * (double)u.y + c * (double)w.y);
      double2 dp = d1<double2>(k, d) * p;
      double2 u1 = r1 - dp;
      C o; o.x = u1.x / lhs; o.y = u1.y / lhs;
      ut[d * RH + i] = o;
      C z = ut[(g.nd + d) * RH + i];
      o.x = (double)z.x / lhs; o.y = (double)z.y / lhs;
      ut[(g.nd + d) * RH + i] = o;
    }
  }
}

// convection (u*.grad) u* per run:  conv[c] = sum_d u*_d du_c/dx_d   gu: [nd][nd][R][P] (c, d)
// coupling: coupl[d] = sum_{v in run} (phi* dmu_d + psi* dnu_d);  rhs2[d] = -conv[d] - lamda coupl[d]
// (Solvers.jl:294-318, Solvers_3d.jl:247-273)
template <typename T>
__global__ void k_conv_coupl(const T* __restrict__ ustar, const T* __restrict__ gu, const T* __restrict__ phis,
                             const T* __restrict__ psis, const T* __restrict__ gmu, const T* __restrict__ gnu,
                             T* __restrict__ conv, T* __restrict__ coupl, T* __restrict__ rhs2,
                             double lamda, int nd, Runs rn, long long P) {
  const long long RP = (long long)rn.R * P, VP = (long long)rn.V * P;
  K_LOOP(RP, i) {
    int r = (int)(i / P);
    long long pix = i - (long long)r * P;
    for (int cc = 0; cc < nd; ++cc) {
      double cv = 0.0;
      for (int d = 0; d < nd; ++d) cv += (double)ustar[d * RP + i] * (double)gu[(cc * nd + d) * RP + i];
      double cp = 0.0;
      for (int v = rn.vbeg[r]; v < rn.vbeg[r + 1]; ++v) {
        long long j = (long long)v * P + pix;
        cp += (double)phis[j] * (double)gmu[cc * VP + j] + (double)psis[j] * (double)gnu[cc * VP + j];
      }
      conv[cc * RP + i] = (T)cv;
      coupl[cc * RP + i] = (T)cp;
      rhs2[cc * RP + i] = (T)(-cv - lamda * cp);
    }
  }
}

// Step 5 inner products.  per vesicle: adv_phi.mu1, adv_psi.nu1, adv_phi.mu2, adv_psi.nu2
template <typename T>
__global__ void __launch_bounds__(256) k_dot5v(const T* __restrict__ adv, const T* __restrict__ mn, long long VP, EW ew, double2* part) {
  __shared__ double sm[2 * 4 * 8];
  KSum acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  EW_LOOP(ew, f, i) {
    long long j = (long long)f * ew.n + i;
    double ap = adv[j], as = adv[VP + j];
    acc[0].add(ap * (double)mn[j]); acc[1].add(as * (double)mn[VP + j]);
    acc[2].add(ap * (double)mn[2 * VP + j]); acc[3].add(as * (double)mn[3 * VP + j]);
  }
  ew_store_partials<4>(acc, part, ew, sm);
}
// per run: coupl.ut1, conv.ut1, coupl.ut2, conv.ut2  (summed over components)
template <typename T>
__global__ void __launch_bounds__(256) k_dot5r(const T* __restrict__ coupl, const T* __restrict__ conv, const T* __restrict__ utp,
                                               int nd, long long RP, EW ew, double2* part) {
  __shared__ double sm[2 * 4 * 8];
  KSum acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  EW_LOOP(ew, f, i) {
    long long j = (long long)f * ew.n + i;
    for (int d = 0; d < nd; ++d) {
      double cp = coupl[d * RP + j], cv = conv[d * RP + j];
      double u1 = utp[d * RP + j], u2 = utp[(nd + d) * RP + j];
      acc[0].add(cp * u1); acc[1].add(cv * u1); acc[2].add(cp * u2); acc[3].add(cv * u2);
    }
  }
  ew_store_partials<4>(acc, part, ew, sm);
}

// Step 5 scalar (Solvers.jl:407-420).  Writes Q into qv[r], theta into th[2r..]
static __global__ void k_fin_step5(const double* __restrict__ fv, const double* __restrict__ fr, const double* __restrict__ scp,
                            const double* __restrict__ sco, const double* __restrict__ dtv, int use_conf_dt,
                            double a, double b, double c, Phys ph, Runs rn, double* __restrict__ qv, double* __restrict__ th) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rn.R) return;
  double t11 = 0, t12 = 0, t21 = 0, t22 = 0;
  for (int v = rn.vbeg[r]; v < rn.vbeg[r + 1]; ++v) {
    t11 += fv[v * 4 + 0]; t12 += fv[v * 4 + 1]; t21 += fv[v * 4 + 2]; t22 += fv[v * 4 + 3];
  }
  double t13 = fr[r * 4 + 0], t14 = fr[r * 4 + 1], t23 = fr[r * 4 + 2], t24 = fr[r * 4 + 3];
  double th1 = ph.cell * (ph.lamda * (t11 + t12 + t13) + t14);
  double th2 = ph.cell * (ph.lamda * (t21 + t22 + t23) + t24);
  double dt = use_conf_dt ? ph.conf_dt : dtv[r];
  double rhsQ = -(b * scp[r * 4 + 0] + c * sco[r * 4 + 0]) / dt + th1;
  double lhsQ = (a / dt) - th2;
  qv[r] = rhsQ / lhsQ;
  th[2 * r] = th1; th[2 * r + 1] = th2;
}

// Step 6 (Solvers.jl:431-453): new hats into hn (the old level's storage), ut combined in place
template <typename T>
__global__ void k_step6(const cplx<T>* __restrict__ s3, const double* __restrict__ qv, cplx<T>* __restrict__ hn,
                        Runs rn, Geom g) {
  using C = cplx<T>;
  const long long VH = (long long)rn.V * g.H;
  K_LOOP(VH, i) {
    int v = (int)(i / g.H);
    long long s = i - (long long)v * g.H;
    if ((int)(s % g.kp) >= g.nkx) continue;
    double Q = qv[rn.run_of[v]];
    // s3 order: phi1 psi1 phi2 psi2 mu1 nu1 mu2 nu2 ; hn order phi psi mu nu
    const int a1[4] = {0, 1, 4, 5}, a2[4] = {2, 3, 6, 7};
    for (int q = 0; q < 4; ++q) {
      C x = s3[a1[q] * VH + i], y = s3[a2[q] * VH + i];
      C o; o.x = (double)x.x + Q * (double)y.x; o.y = (double)x.y + Q * (double)y.y;
      hn[q * VH + i] = o;
    }
  }
}
static __global__ void k_step6_scalars(const double* __restrict__ r2, const double* __restrict__ qv, double* __restrict__ scn, int R) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  double Q = qv[r];
  scn[r * 4 + 0] = Q;
  scn[r * 4 + 1] = r2[r * 6 + 0] + Q * r2[r * 6 + 3];
  scn[r * 4 + 2] = r2[r * 6 + 1] + Q * r2[r * 6 + 4];
  scn[r * 4 + 3] = r2[r * 6 + 2] + Q * r2[r * 6 + 5];
}

// Step 6 velocity combination + Step 7 projection (Solvers.jl:445,459-498)
//  ut: [2][nd][R][H];  up: present u/p hats;  un: new u/p hats  ([nd+1][R][H])
template <typename T>
__global__ void k_step67(const cplx<T>* __restrict__ ut, const double* __restrict__ qv, const cplx<T>* __restrict__ up,
                         cplx<T>* __restrict__ un, const double* __restrict__ dtv, double a, Phys ph, int R, Geom g) {
  using C = cplx<T>;
  const long long RH = (long long)R * g.H;
  K_LOOP(RH, i) {
    int r = (int)(i / g.H);
    long long s = i - (long long)r * g.H;
    KI k = kdecode(s, g);
    if (k.kx >= g.nkx) continue;
    double Q = qv[r], dt = dtv[r];
    double2 u[3];
    double2 div = make_double2(0, 0);
    for (int d = 0; d < g.nd; ++d) {
      C x = ut[d * RH + i], y = ut[(g.nd + d) * RH + i];
      u[d] = make_double2((double)x.x + Q * (double)y.x, (double)x.y + Q * (double)y.y);
      div = div + d1<double2>(k, d) * u[d];
    }
    double Lap = -k.k2();
    double2 dp = make_double2(0, 0);
    bool zero = (k.kx == 0 && k.ky == 0 && k.kz == 0);
    if (!zero) { double f = a / dt; dp = make_double2(f * div.x / Lap, f * div.y / Lap); }
    for (int d = 0; d < g.nd; ++d) {
      double2 o = u[d] - (dt / a) * (d1<double2>(k, d) * dp);
      C z; z.x = o.x; z.y = o.y; un[d * RH + i] = z;
    }
    C pz = up[g.nd * RH + i];
    double2 pn = make_double2((double)pz.x + dp.x - ph.eta * div.x, (double)pz.y + dp.y - ph.eta * div.y);
    C z; z.x = pn.x; z.y = pn.y; un[g.nd * RH + i] = z;
  }
}

// init (simulation.jl:42-47): mu_hat = Lphi phi_hat + R1 H1h + R2 H2h + R3 H3h ; nu_hat = S4 psi_hat + R3 Gh
template <typename T>
__global__ void k_init_munu(cplx<T>* __restrict__ h4, const cplx<T>* __restrict__ Hh, const double* __restrict__ scp,
                            Phys ph, Runs rn, Geom g) {
  using C = cplx<T>;
  const long long VH = (long long)rn.V * g.H;
  K_LOOP(VH, i) {
    int v = (int)(i / g.H);
    long long s = i - (long long)v * g.H;
    KI k = kdecode(s, g);
    if (k.kx >= g.nkx) continue;
    int r = rn.run_of[v];
    double R1 = scp[r * 4 + 1], R2 = scp[r * 4 + 2], R3 = scp[r * 4 + 3];
    double K2 = k.k2();
    double Lphi = ph.S1 * K2 * K2 + ph.S2 * K2 + ph.S3;
    auto L = [&](const C* p) { C z = p[i]; return make_double2(z.x, z.y); };
    double2 mu = Lphi * L(h4) + R1 * L(Hh) + R2 * L(Hh + VH) + R3 * L(Hh + 2 * VH);
    double2 nu = ph.S4 * L(h4 + VH) + R3 * L(Hh + 3 * VH);
    C o; o.x = mu.x; o.y = mu.y; h4[2 * VH + i] = o;
    o.x = nu.x; o.y = nu.y; h4[3 * VH + i] = o;
  }
}

// ---------------------------------------------------------------------------
// monitoring: compute_modified_energy (Utils.jl:96-141) + area ratio (simulation.jl:147)
//  per vesicle sums (K=8): lap_new^2, lap_star^2, gnew^2, gstar^2, phi^2, phistar^2, psi^2, psistar^2
//  plus f_surf(phi) for the area (K slot 8)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_mon_v(const T* __restrict__ phi, const T* __restrict__ phio, const T* __restrict__ psi,
                                               const T* __restrict__ psio, const T* __restrict__ lapn, const T* __restrict__ laps,
                                               const T* __restrict__ g4, const T* __restrict__ ga, long long VP, Phys ph,
                                               EW ew, double2* part) {
  __shared__ double sm[2 * 9 * 8];
  KSum acc[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) acc[k] = {0.0, 0.0};
  const double e = ph.eps;
  EW_LOOP(ew, f, i) {
    long long j = (long long)f * ew.n + i;
    double p = phi[j], po = phio[j], s = psi[j], so = psio[j];
    double ps = 2.0 * p - po, ss = 2.0 * s - so;
    double ln = lapn[j], ls = laps[j];
    acc[0].add(ln * ln); acc[1].add(ls * ls);
    if (g4) {
      double a0 = g4[j], a1 = g4[VP + j], a2 = g4[2 * VP + j], a3 = g4[3 * VP + j];
      acc[2].add(a0 * a0 + a1 * a1); acc[3].add(a2 * a2 + a3 * a3);
    }
    acc[4].add(p * p); acc[5].add(ps * ps); acc[6].add(s * s); acc[7].add(ss * ss);
    double x = ga[j], y = ga[VP + j];
    acc[8].add((3.0 * SQ2 / 4.0) * (g_(p) / e) + e * (x * x + y * y) / 2.0);
  }
  ew_store_partials<9>(acc, part, ew, sm);
}
// per run (K=3): |u|^2, |2u-uo|^2 (all components), |grad p|^2 (x,y)
template <typename T>
__global__ void __launch_bounds__(256) k_mon_r(const T* __restrict__ up, const T* __restrict__ uo, const T* __restrict__ gp,
                                               int nd, long long RP, EW ew, double2* part) {
  __shared__ double sm[2 * 3 * 8];
  KSum acc[3] = {{0, 0}, {0, 0}, {0, 0}};
  EW_LOOP(ew, f, i) {
    long long j = (long long)f * ew.n + i;
    for (int d = 0; d < nd; ++d) {
      double u = up[d * RP + j], w = uo[d * RP + j];
      double s = 2.0 * u - w;
      acc[0].add(u * u); acc[1].add(s * s);
    }
    double gx = gp[j], gy = gp[RP + j];
    acc[2].add(gx * gx + gy * gy);
  }
  ew_store_partials<3>(acc, part, ew, sm);
}
static __global__ void k_fin_mon(const double* __restrict__ fv, const double* __restrict__ fr, const double* __restrict__ scp,
                          const double* __restrict__ sco, const double* __restrict__ dtv, const double* __restrict__ A0,
                          Phys ph, Runs rn, double* __restrict__ energy, double* __restrict__ aratio, double* __restrict__ area) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rn.R) return;
  const double w = ph.cell;
  double S[9];
  for (int k = 0; k < 9; ++k) S[k] = 0.0;
  double num = 0.0, den = 0.0;
  for (int v = rn.vbeg[r]; v < rn.vbeg[r + 1]; ++v) {
    for (int k = 0; k < 9; ++k) S[k] += fv[v * 9 + k];
    double A = fv[v * 9 + 8] * w;
    area[v] = A;
    num += fabs(A - A0[v]); den += A0[v];
  }
  double kinetic = 0.25 * (fr[r * 3 + 0] * w) + 0.25 * (fr[r * 3 + 1] * w);
  double dt = dtv[r];
  double pressure = (dt * dt / 3.0) * (fr[r * 3 + 2] * w);
  auto se = [](double rn_, double ro) { return 0.5 * rn_ * rn_ + 0.5 * (2.0 * rn_ - ro) * (2.0 * rn_ - ro); };
  double Re = se(scp[r * 4 + 1], sco[r * 4 + 1]) + se(scp[r * 4 + 2], sco[r * 4 + 2]) + se(scp[r * 4 + 3], sco[r * 4 + 3]);
  double Qe = 0.5 * se(scp[r * 4 + 0], sco[r * 4 + 0]);
  double S1t = 0.25 * ph.S1 * (S[0] * w + S[1] * w);
  double S2t = 0.25 * ph.S2 * (S[2] * w + S[3] * w);
  double S3t = 0.25 * ph.S3 * (S[4] * w + S[5] * w);
  double S4t = 0.25 * ph.S4 * (S[6] * w + S[7] * w);
  energy[r] = kinetic + pressure + ph.lamda * Re + Qe + ph.lamda * (S1t + S2t + S3t + S4t) -
              ph.lamda * (ph.C1 + ph.C2 + ph.C3) - 0.5;
  aratio[r] = num / den;
}

}  // namespace vsav
