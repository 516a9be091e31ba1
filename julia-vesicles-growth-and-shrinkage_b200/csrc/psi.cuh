// The 2D psi solve of Step 1 (src/Solvers.jl:39-81):
//   A x = (a/dt) x - sum_d i k_d F( M_psi F^-1( i k_d S4 x ) )
//   preconditioner P^-1 = 1 / (a/dt - M_max S4 Laplacian)
// solved by BiCGSTAB with Krylov.jl 0.10.6 semantics (left preconditioner by
// multiplication, shadow vector c = b, x0 = 0, stop on ||M^-1 r|| <= atol +
// rtol ||M^-1 b|| or itmax).  All three right-hand sides of a step (splits
// 11, 12, 21) and every run of an ensemble are solved together: a "system" is
// (split j, run r); its vector spans the vesicle fields of run r.
//
// Two formulations:
//  FULL  the reference's own: full complex spectra [F][Ny][Nx] with the
//        fftfreq kx0 (Nyquist negative), complex Krylov scalars, solution
//        truncated to the half spectrum (Solvers.jl:79);
//  HALF  the operator restricted to real fields, held as half spectra
//        [F][Ny][kp]: the kx=0 and kx=Nx/2 columns are kept Hermitian
//        (projection), the x derivative at kx=Nx/2 is zero (in the operator
//        and in its preconditioner), inner products are the real
//        Parseval-weighted ones, so the scalars are real.  It moves half the
//        bytes of FULL but is NOT the reference's solve: FULL's Nyquist
//        multipliers feed an anti-Hermitian (imaginary-field) channel that the
//        truncation of Solvers.jl:79 keeps, and HALF drops it.  On resolved
//        interfaces the two agree closely; on under-resolved ones they differ
//        by up to ~1e-2, so FULL is the default in both precisions.
#pragma once
#include "kernels.cuh"
#include "tma.cuh"

namespace vsav {

struct BiState {
  double2 rho, alpha, omega, beta;
  double rnorm, eps;
  int iters, active, solved, status;   // status: 0 running, 1 solved, 2 itmax, 3 breakdown, 4 zero rhs
};

struct SysMap {
  int V, R;
  const int* run_of;
  __device__ __forceinline__ int sys(int field) const { return (field / V) * R + run_of[field % V]; }
};

// ---------------------------------------------------------------------------
// fused x pass of the operator: inverse x transform -> multiply by M_psi (of
// the row's vesicle) and `scale` -> forward x transform, in place, for rows of
// nin consecutive field blocks (t1 | t2).  HALF rows: c2r/r2c of length Nx;
// FULL rows: c2c of length Nx.
// ---------------------------------------------------------------------------
template <typename T, int E, int NT, bool FULL>
__global__ void __launch_bounds__(NT, MinB<E, NT>::v) k_rows_mul(cplx<T>* __restrict__ t, const T* __restrict__ M, T mconst, T scale,
                                                              int logL, int lognl, long long nrows, int rowlen_c,
                                                              int rows_per_field, SysMap sm, const int* __restrict__ active,
                                                              int f0, int fc, const cplx<T>* __restrict__ tab) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  const int L = 1 << logL, LP = line_pitch(L), nl = 1 << lognl, LE = L / E;
  C* sN = s + 2 * nl * LP;
  C* const buf[2] = {s, s + nl * LP};
  const long long row0 = (long long)blockIdx.x * nl;
  // rows hold t1 | t2 of the fc chunk fields starting at global field f0
  const int field = f0 + (int)(row0 / rows_per_field) % fc;
  if (active && !active[sm.sys(field)]) return;
  const int v_ = field % sm.V;
  const int Nx = FULL ? L : 2 * L;
  const long long rows_left = nrows - row0;
  int line, i;
  row_owner<E>(logL, line, i);
  const bool act = line < rows_left;
  const RowLay lay{LP};
  C v[E];
  // the row's M values, loaded before the inverse transform so their latency overlaps it
  T mv[FULL ? E : 2 * E];
  {
    const long long prow0 = (long long)v_ * rows_per_field + (row0 % rows_per_field) + line;
    const T* Mr0 = (M && act) ? M + prow0 * (long long)Nx : nullptr;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int e = i + j * LE;
      if (FULL) mv[j] = (Mr0 ? Mr0[e] : mconst) * scale;
      else { mv[2 * j] = (Mr0 ? Mr0[2 * e] : mconst) * scale; mv[2 * j + 1] = (Mr0 ? Mr0[2 * e + 1] : mconst) * scale; }
    }
  }
  // inverse x transform, result in registers (element i + j L/E of the row)
  if (FULL) {
    if (act) {
#pragma unroll
      for (int j = 0; j < E; ++j) v[j] = t[(row0 + line) * rowlen_c + i + j * LE];
    }
    tile_fft<E, true, true, true>(v, buf, lay, line, i, act, logL, lognl, tab);
  } else {
    load_c2r_tile<T, E>(t, s, sN, row0, rows_left, logL, lognl, rowlen_c, tab);
    tile_fft<E, true, false, true>(v, buf, lay, line, i, act, logL, lognl, tab);
  }
  // multiply by M_psi of the row's vesicle (HALF: z[m] holds x[2m] + i x[2m+1])
  if (act) {
#pragma unroll
    for (int j = 0; j < E; ++j) {
      if (FULL) { v[j].x *= mv[j]; v[j].y *= mv[j]; }
      else { v[j].x *= mv[2 * j]; v[j].y *= mv[2 * j + 1]; }
    }
  }
  __syncthreads();   // smem is reused by the forward transform
  if (FULL) {
    tile_fft<E, false, true, true>(v, buf, lay, line, i, act, logL, lognl, tab);
    if (act) {
#pragma unroll
      for (int j = 0; j < E; ++j) t[(row0 + line) * rowlen_c + i + j * LE] = v[j];
    }
  } else {
    const C* so = buf[tile_fft<E, false, true, false>(v, buf, lay, line, i, act, logL, lognl, tab)];
    const int half = L / 2 + 1;
    for (int f = threadIdx.x; f < nl * half; f += blockDim.x) {
      int ln = f / half, k = f - ln * half;
      if (ln >= rows_left) continue;
      C Zk = so[sidx(ln, LP, k)];
      C Zc = so[sidx(ln, LP, (L - k) & (L - 1))];
      C w = __ldg(&tab[2 * L + k]);
      C Xk, XLk;
      r2c_post(Zk, Zc, w, Xk, XLk);
      C* orow = t + (row0 + ln) * rowlen_c;
      orow[k] = Xk;
      if (k != L - k) orow[L - k] = XLk;
    }
  }
}

// ---------------------------------------------------------------------------
// wavenumbers of a vector slot (HALF: [Ny][kp] with rfftfreq kx; FULL: [Ny][Nx] fftfreq kx0)
// ---------------------------------------------------------------------------
struct VGeom {
  int full;         // 1 = FULL
  int Nx, Ny, kp, nkx, logNx;
  long long n;      // slots per field
  double kxs, kys;
  int nd3 = 0;      // 1: 3D full spectra [Nz][Ny][Nx] (the 3D variable-mobility solve)
  int logNy = 0, Nz = 1;
  double kzs = 0.0;
};
__device__ __forceinline__ void vk(const VGeom& g, long long s, int& kx, int& ky, double& kxv, double& kyv, double& w) {
  // slot < 2^31 within a field: 32-bit index arithmetic (row lengths are powers of two or kp)
  const unsigned su = (unsigned)s;
  if (g.full) {
    kx = (int)(su & (unsigned)(g.Nx - 1)); ky = (int)(su >> g.logNx);
    if (g.nd3) ky &= g.Ny - 1;
  }
  else { ky = (int)(su / (unsigned)g.kp); kx = (int)(su - (unsigned)ky * (unsigned)g.kp); }
  kyv = kfreq(ky, g.Ny) * g.kys;
  if (g.full) { kxv = kfreq(kx, g.Nx) * g.kxs; w = 1.0; }
  else {
    kxv = kx * g.kxs;
    w = (kx >= g.nkx) ? 0.0 : ((kx == 0 || kx == g.Nx / 2) ? 1.0 : 2.0);
  }
}

// kz^2 of a 3D full-spectrum slot (0 in 2D)
__device__ __forceinline__ double vk_kz2(const VGeom& g, long long s) {
  if (!g.nd3) return 0.0;
  const double kzv = kfreq((int)((unsigned)s >> (g.logNx + g.logNy)), g.Nz) * g.kzs;
  return kzv * kzv;
}

// FP32 form of vk + vk_kz2 for the FP32 solve's vector passes: the squared
// wavenumber |k|^2 (HALF: Nyquist x term zero, as the operator) and the slot
// weight w.  Integer index arithmetic, FP32 multipliers.
__device__ __forceinline__ void vk_f32(const VGeom& g, long long s, float& k2, float& w) {
  const unsigned su = (unsigned)s;
  int kx, ky;
  if (g.full) {
    kx = (int)(su & (unsigned)(g.Nx - 1)); ky = (int)(su >> g.logNx);
    if (g.nd3) ky &= g.Ny - 1;
  }
  else { ky = (int)(su / (unsigned)g.kp); kx = (int)(su - (unsigned)ky * (unsigned)g.kp); }
  const float kyv = (float)(ky < g.Ny / 2 ? ky : ky - g.Ny) * (float)g.kys;
  float kxv;
  if (g.full) { kxv = (float)(kx < g.Nx / 2 ? kx : kx - g.Nx) * (float)g.kxs; w = 1.f; }
  else {
    kxv = (kx == g.Nx / 2) ? 0.f : (float)kx * (float)g.kxs;
    w = (kx >= g.nkx) ? 0.f : ((kx == 0 || kx == g.Nx / 2) ? 1.f : 2.f);
  }
  k2 = fmaf(kxv, kxv, kyv * kyv);
  if (g.nd3) {
    const int kz = (int)(su >> (g.logNx + g.logNy));
    const float kzv = (float)(kz < g.Nz / 2 ? kz : kz - g.Nz) * (float)g.kzs;
    k2 = fmaf(kzv, kzv, k2);
  }
}

// y = a_dt * x - ( m_x t1 + i ky t2 ) at slot s of field f (HALF: Nyquist x multiplier zero)
template <typename T>
__device__ __forceinline__ double2 op_out(const VGeom& g, const cplx<T>* x, const cplx<T>* t1, const cplx<T>* t2,
                                          long long j, int kx, double kxv, double kyv, double adt, double sgn) {
  cplx<T> xv = x ? x[j] : cplx<T>{}, a = t1[j], b = t2[j];
  double mx = (!g.full && kx == g.Nx / 2) ? 0.0 : kxv;
  double2 d = make_double2(-(mx * (double)a.y + kyv * (double)b.y), mx * (double)a.x + kyv * (double)b.x);
  return make_double2(adt * (double)xv.x + sgn * d.x, adt * (double)xv.y + sgn * d.y);
}

// Operator output + preconditioner + inner products.
//   y = P^-1 ( a_dt x - (i kx t1 + i ky t2) )   (diag P^-1 = 1/(a_dt + Mmax S4 k^2); identity if !precond)
//   HALF: the kx=0 and kx=Nx/2 columns of the operator output are made Hermitian.
//   dots (per field): K = ndot complex (u_k^H w_k) with (u_k, w_k) from {c, y, s} ...
//   mode 0: out y; dots <c, y>                              (q = A p; v = M^-1 q)
//   mode 1: out y; dots <y, s>, <y, y>                      (t = M^-1 A s)
template <typename T>
__global__ void __launch_bounds__(256) k_psi_combine(const cplx<T>* __restrict__ x, const cplx<T>* __restrict__ t1,
                                                     const cplx<T>* __restrict__ t2, cplx<T>* __restrict__ y,
                                                     const cplx<T>* __restrict__ cvec, const cplx<T>* __restrict__ svec,
                                                     int mode, const double* __restrict__ adt_r, const double* __restrict__ mmax_r,
                                                     double S4, VGeom g, SysMap sm, const int* __restrict__ active,
                                                     int f0, EW ew, double2* part) {
  __shared__ double smm[2 * 4 * 8];
  KSum acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  // t1/t2 are chunk-local (field blockIdx.y of the chunk); x, y, c, s are global (field f0 + blockIdx.y)
  const int f = f0 + blockIdx.y;
  const long long tsh = ((long long)f - blockIdx.y) * g.n;    // global -> chunk-local slot shift
  t1 -= tsh; t2 -= tsh;
  const int sy = sm.sys(f);
  const int r = sm.run_of[f % sm.V];
  const bool act = !active || active[sy];
  if (act) {
    const double adt = adt_r[r], mm = mmax_r ? mmax_r[r] : 0.0;
    const long long beg = (long long)blockIdx.x * ew.chunk, end = min(ew.n, beg + ew.chunk);
    // U elements per thread per round, their loads issued before any use
    constexpr int U = 4;
    for (long long s0 = beg + threadIdx.x; s0 < end; s0 += U * blockDim.x) {
      cplx<T> xv[U], av[U], bv[U], cv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const long long s = s0 + (long long)u * blockDim.x;
        if (s < end) {
          const long long j = (long long)f * g.n + s;
          xv[u] = x ? x[j] : cplx<T>{};
          av[u] = t1[j];
          bv[u] = t2[j];
          cv[u] = mode == 0 ? cvec[j] : svec[j];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
      const long long s = s0 + (long long)u * blockDim.x;
      if (s >= end) break;
      int kx, ky; double kxv, kyv, w;
      vk(g, s, kx, ky, kxv, kyv, w);
      if (w == 0.0) continue;
      long long j = (long long)f * g.n + s;
      double2 o;
      {
        double mx = (!g.full && kx == g.Nx / 2) ? 0.0 : kxv;
        double2 d = make_double2(-(mx * (double)av[u].y + kyv * (double)bv[u].y), mx * (double)av[u].x + kyv * (double)bv[u].x);
        o = make_double2(adt * (double)xv[u].x - d.x, adt * (double)xv[u].y - d.y);
      }
      if (!g.full && (kx == 0 || kx == g.Nx / 2)) {
        int kym = (g.Ny - ky) % g.Ny;
        long long jm = (long long)f * g.n + (long long)kym * g.kp + kx;
        double2 om = op_out<T>(g, x, t1, t2, jm, kx, kxv, kfreq(kym, g.Ny) * g.kys, adt, -1.0);
        o = make_double2(0.5 * (o.x + om.x), 0.5 * (o.y - om.y));
      }
      if (mmax_r) {
        // 1/(a_dt - M_max Lap S4); HALF drops the x derivative at kx = Nx/2, so does its preconditioner
        double kxp = (!g.full && kx == g.Nx / 2) ? 0.0 : kxv;
        double pinv = 1.0 / (adt + mm * S4 * (kxp * kxp + kyv * kyv));
        o = make_double2(o.x * pinv, o.y * pinv);
      }
      cplx<T> ot; ot.x = o.x; ot.y = o.y;
      y[j] = ot;
      double ox = ot.x, oy = ot.y;   // use the stored (rounded) values in the dots
      if (mode == 0) {
        const cplx<T> c = cv[u];
        acc[0].add(w * ((double)c.x * ox + (double)c.y * oy));
        if (g.full) acc[1].add((double)c.x * oy - (double)c.y * ox);
      } else {
        const cplx<T> sv = cv[u];
        acc[0].add(w * (ox * (double)sv.x + oy * (double)sv.y));
        if (g.full) acc[1].add(ox * (double)sv.y - oy * (double)sv.x);
        acc[2].add(w * (ox * ox + oy * oy));
      }
      }
    }
  }
  block_reduce_store<4>(acc, part + ((long long)f * ew.bpf + blockIdx.x) * 4, smm);
}

// ---------------------------------------------------------------------------
// FULL-form operator passes fused around the column FFTs
// ---------------------------------------------------------------------------
// Inverse y pass for both derivative directions from one read of x:
//   t1 = IFFT_y(i kx0 S4 x),  t2 = IFFT_y(i ky S4 x)   (x global field f0 + fl,
// t1/t2 chunk-local field fl).  The second transform re-reads the tile from L2.
// Fields of inactive systems are skipped (the x pass and the combine skip them).
template <typename T, int E, int NT>
__global__ void __launch_bounds__(NT, MinB<E, NT>::v) k_psi_cols_inv2(const cplx<T>* __restrict__ x, cplx<T>* __restrict__ t1,
                                                                   cplx<T>* __restrict__ t2, double S4, ColArgs a, SysMap sm,
                                                                   const int* __restrict__ active, int f0,
                                                                   const cplx<T>* __restrict__ tab) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  const int L = 1 << a.logL, LE = L / E;
  const int tile = blockIdx.x % a.tiles;
  const int fl = blockIdx.x / a.tiles;
  const int f = f0 + fl;
  if (active && !active[sm.sys(f)]) return;                 // block-uniform
  const int cl = threadIdx.x & (a.TW - 1), i = threadIdx.x >> a.logTW, c = tile * a.TW + cl;
  const bool valid = c < a.W;
  const ColLay lay{a.TW, Log2<E>::v};
  C* const buf[2] = {s, s + col_tile_elems(L, a.TW, Log2<E>::v)};
  const C* xin = x + (long long)f * a.O + c;
  // small E: the raw tile stays in registers for the second direction
  constexpr int EK = E <= 8 ? E : 1;
  C xr[EK];
  if constexpr (E <= 8) {
#pragma unroll
    for (int j = 0; j < E; ++j) xr[j] = valid ? xin[(long long)(i + j * LE) * a.S] : mk<C>(0.0, 0.0);
  }
  // FP32: the multipliers i kx0 S4 (per column) and i ky S4 (per element) in FP32 arithmetic,
  // ky from the element's row e = i + j L/E without integer conversions in the loop
  constexpr bool F32 = std::is_same<T, float>::value;
  const float fkx = F32 ? (float)(kfreq(c, a.Nx) * a.kxs * S4) : 0.f, fky = F32 ? (float)(a.kys * S4) : 0.f;
  const float fi = (float)i, fLE = (float)LE, fNy = (float)a.Ny;
#pragma unroll 1
  for (int d = 0; d < 2; ++d) {
    const int mult = d == 0 ? M_DX0 : M_DY;
    C v[E];
    if (valid) {
#pragma unroll
      for (int j = 0; j < E; ++j) {
        C xv;
        if constexpr (E <= 8) xv = xr[j];
        else xv = xin[(long long)(i + j * LE) * a.S];
        if constexpr (F32) {
          float k = fkx;
          if (d == 1) {
            float ke = fmaf((float)j, fLE, fi);
            if (i + j * LE >= (a.Ny >> 1)) ke -= fNy;
            k = ke * fky;
          }
          v[j] = mk<C>(-k * xv.y, k * xv.x);
        } else {
          v[j] = xv * col_mult<C>(a, mult, S4, c, i + j * LE, 0);
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < E; ++j) v[j] = mk<C>(0.0, 0.0);
    }
    if (d == 1) __syncthreads();                             // the first transform's smem reads are done
    tile_fft<E, true, true, true>(v, buf, lay, cl, i, true, a.logL, a.logTW, tab);
    if (valid) {
      C* o = (d == 0 ? t1 : t2) + (long long)fl * a.O + c;
#pragma unroll
      for (int j = 0; j < E; ++j) o[(long long)(i + j * LE) * a.S] = v[j];
    }
  }
}

// Forward y pass of t1 and t2 fused with the operator output, the diagonal
// preconditioner and the dot products (FULL form; k_psi_combine's modes):
//   y = P^-1 (a_dt x - (i kx0 t1^ + i ky t2^)),  P^-1 = 1/(a_dt + Mmax S4 k^2) or 1.
// One block = TW columns of one field; dot partials per (field, tile):
// part[(f * tiles + tile) * 4 + k].  The transformed t2 tile waits in a third
// shared-memory area (natural [row][TW] order, each thread its own elements)
// while t1 is transformed.
template <typename T, int E, int NT>
__global__ void __launch_bounds__(NT, MinB<E, NT>::v) k_psi_cols_comb(const cplx<T>* __restrict__ t1, const cplx<T>* __restrict__ t2,
                                                                   const cplx<T>* __restrict__ x, cplx<T>* __restrict__ y,
                                                                   const cplx<T>* __restrict__ cvec, const cplx<T>* __restrict__ svec,
                                                                   int mode, const double* __restrict__ adt_r,
                                                                   const double* __restrict__ mmax_r, double S4, ColArgs a,
                                                                   SysMap sm, const int* __restrict__ active, int f0,
                                                                   const cplx<T>* __restrict__ tab, double2* __restrict__ part) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double smm[2 * 4 * (NT / 32)];
  C* s = reinterpret_cast<C*>(smraw);
  const int L = 1 << a.logL, LE = L / E;
  const int tile = blockIdx.x % a.tiles;
  const int fl = blockIdx.x / a.tiles;
  const int f = f0 + fl;
  KSum acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  if (!active || active[sm.sys(f)]) {                       // block-uniform
    const int cl = threadIdx.x & (a.TW - 1), i = threadIdx.x >> a.logTW, c = tile * a.TW + cl;
    const bool valid = c < a.W;
    const ColLay lay{a.TW, Log2<E>::v};
    C* const buf[2] = {s, s + col_tile_elems(L, a.TW, Log2<E>::v)};
    C* const res = s + 2 * col_tile_elems(L, a.TW, Log2<E>::v);
    C v[E];
    const long long off = (long long)fl * a.O + c;
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = valid ? t2[off + (long long)(i + j * LE) * a.S] : mk<C>(0.0, 0.0);
    tile_fft<E, false, true, true>(v, buf, lay, cl, i, true, a.logL, a.logTW, tab);
#pragma unroll
    for (int j = 0; j < E; ++j) res[(i + j * LE) * a.TW + cl] = v[j];
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = valid ? t1[off + (long long)(i + j * LE) * a.S] : mk<C>(0.0, 0.0);
    // x and c/s are read in the epilogue: prefetching them into registers during the t1
    // transform measured slower (register pressure, spills) than the plain loads
    const long long gbase = (long long)f * a.O + c;
    __syncthreads();                                        // the first transform's smem reads are done
    tile_fft<E, false, true, true>(v, buf, lay, cl, i, true, a.logL, a.logTW, tab);
    if (valid) {
      const int r = sm.run_of[f % sm.V];
      const double adt = adt_r[r], mm = mmax_r ? mmax_r[r] : 0.0;
      const double kxv = kfreq(c, a.Nx) * a.kxs;
#pragma unroll
      for (int j = 0; j < E; ++j) {
        const int e = i + j * LE;
        const double kyv = kfreq(e, a.Ny) * a.kys;
        const long long idx = gbase + (long long)e * a.S;
        const C xv = x ? x[idx] : mk<C>(0.0, 0.0), cv = mode == 0 ? cvec[idx] : svec[idx];
        const C w2 = res[e * a.TW + cl];
        const double dx = -(kxv * (double)v[j].y + kyv * (double)w2.y);
        const double dy = kxv * (double)v[j].x + kyv * (double)w2.x;
        double ox = adt * (double)xv.x - dx, oy = adt * (double)xv.y - dy;
        if (mmax_r) {
          const double pinv = 1.0 / (adt + mm * S4 * (kxv * kxv + kyv * kyv));
          ox *= pinv; oy *= pinv;
        }
        C ot; ot.x = ox; ot.y = oy;
        y[idx] = ot;
        ox = ot.x; oy = ot.y;                               // the dots use the stored (rounded) values
        if (mode == 0) {
          acc[0].add((double)cv.x * ox + (double)cv.y * oy);
          acc[1].add((double)cv.x * oy - (double)cv.y * ox);
        } else {
          acc[0].add(ox * (double)cv.x + oy * (double)cv.y);
          acc[1].add(ox * (double)cv.y - oy * (double)cv.x);
          acc[2].add(ox * ox + oy * oy);
        }
      }
    }
  }
  block_reduce_store<4>(acc, part + ((long long)f * a.tiles + tile) * 4, smm);
}

// ---------------------------------------------------------------------------
// TMA-fed persistent forms of the two FULL-form column passes (FP32).
//
// A tile is TW consecutive columns of one field, all L rows.  Each block is
// resident for the whole launch and walks the tiles blockIdx.x, + gridDim.x,
// ...; the inputs of a tile arrive in a shared-memory staging area by 2D bulk
// tensor copies (one thread issues them; boxes of TW columns x min(L, 256)
// rows), so the copies of tile k+1 run while tile k is transformed.  The two
// transforms of a tile (t1 and t2, or the two derivative directions) run as
// one tile of 2 TW lines through the single-buffer FFT, whose arithmetic is
// that of the ping-pong kernels: the transforms are bit-identical to those of
// k_psi_cols_inv2 / k_psi_cols_comb.
//
// Shared memory (dynamic, 1024-byte aligned):
//   staging  A arrays x [L][TW] (TMA box layout), A = 1 (inv2) or 4 (comb: t1 t2 x c)
//   work     col_tile_elems(L, 2 TW, log2 E) complex (the FFT buffer)
//   2 mbarriers (64 bytes)
//   twx      the last FFT pass's per-butterfly twiddles (tw_last_table), staged once
//            per block, so that pass reads consecutive shared words instead of
//            strided entries of the global table
// ---------------------------------------------------------------------------
struct TmaTiles {
  int total;        // tiles over the chunk's fields: fc * tiles
  int tiles;        // column tiles per field: Nx / TW
  int TW, logTW;
  int BH, nbox;     // rows per box, boxes per column tile (BH * nbox = L)
};

__host__ __device__ __forceinline__ size_t tma_col_smem(int L, int TW, int E, int narrays) {
  const size_t stage = (size_t)narrays * L * TW * sizeof(float2);
  int loge = 0;
  while ((1 << loge) < E) ++loge;
  const size_t work = (size_t)col_tile_elems(L, 2 * TW, loge) * sizeof(float2);
  const size_t twx = (size_t)(E >= 16 ? 3 + E / 4 - 1 : E - 1) * (L / E) * sizeof(float2);
  return 1024 + stage + work + 64 + twx;
}

// the last-pass twiddle table (tw_last_table) of a TMA column pass, after its mbarriers
__device__ __forceinline__ float2* tma_twx(uint64_t* bar) { return reinterpret_cast<float2*>(reinterpret_cast<unsigned char*>(bar) + 64); }

__device__ __forceinline__ unsigned char* tma_smem_base() {
  extern __shared__ __align__(16) unsigned char smraw_tma[];
  return reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw_tma) + 1023) & ~(uintptr_t)1023);
}

// Inverse y pass of both derivative directions (k_psi_cols_inv2, FP32):
//   t1 = IFFT_y(i kx0 S4 x),  t2 = IFFT_y(i ky S4 x)   (x global field f0 + fl; t1/t2 chunk-local fl)
template <int E, int NT, int LOGL>
__global__ void __launch_bounds__(NT, NT <= 512 ? 2 : 1) k_psi_cols_inv2_tma(const __grid_constant__ CUtensorMap mx, float2* __restrict__ t1,
                                                              float2* __restrict__ t2, double S4, ColArgs a, TmaTiles tt,
                                                              SysMap sm, const int* __restrict__ active, int f0,
                                                              const float2* __restrict__ tab, int* __restrict__ err) {
  using C = float2;
  // the tile geometry is compile-time (L = 2^LOGL rows, TW = E NT / (2 L) columns), so
  // the shared-memory index arithmetic folds to constants
  constexpr int L = 1 << LOGL, LE = L / E, TW = E * NT / (2 * L), LOGTW = Log2<TW>::v;
  static_assert(TW >= 2 && TW <= 16 && L >= E * E, "tile geometry");
  constexpr int BH = L < 256 ? L : 256, NBOX = L / BH;     // rows per TMA box, boxes per column tile
  unsigned char* base = tma_smem_base();
  C* sx = reinterpret_cast<C*>(base);
  C* work = sx + (size_t)L * TW;
  uint64_t* bar = reinterpret_cast<uint64_t*>(work + col_tile_elems(L, 2 * TW, Log2<E>::v));
  constexpr int lognl = LOGTW + 1;
  const int tid = threadIdx.x;
  const int line = tid & (2 * TW - 1), i = tid >> lognl, cl = line & (TW - 1);
  const bool dir_y = line >= TW;
  const uint32_t tx = (uint32_t)((size_t)L * TW * sizeof(C));
  auto act = [&](int t) { return !active || active[sm.sys(f0 + t / tt.tiles)]; };
  auto next = [&](int t) { while (t < tt.total && !act(t)) t += gridDim.x; return t; };
  auto issue = [&](int t) {
    const int fl = t / tt.tiles, c0 = (t % tt.tiles) * TW;
    mbar_arrive_expect_tx(bar, tx);
    for (int q = 0; q < NBOX; ++q) tma_load_2d(sx + (size_t)q * BH * TW, &mx, c0, (f0 + fl) * a.Ny + q * BH, bar);
  };
  C* twx = tma_twx(bar);
  if (tid == 0) { mbar_init(bar, 1); mbar_fence_init(); }
  tw_last_table<E>(twx, LOGL, tab);
  __syncthreads();
  int t = next(blockIdx.x);
  if (tid == 0 && t < tt.total) issue(t);
  const ColLay lay{2 * TW, Log2<E>::v};
  const float fi = (float)i, fLE = (float)LE, fNy = (float)a.Ny, fky = (float)(a.kys * S4);
  uint32_t ph = 0;
  while (t < tt.total) {
    const int fl = t / tt.tiles, c = (t % tt.tiles) * TW + cl;
    const bool ok = mbar_wait(bar, ph, err);
    if (__syncthreads_or(!ok)) return;
    const float fkx = (float)(kfreq(c, a.Nx) * a.kxs * S4);
    C v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const C xv = sx[(i + j * LE) * TW + cl];
      float k = fkx;
      if (dir_y) {
        float ke = fmaf((float)j, fLE, fi);
        if (i + j * LE >= (a.Ny >> 1)) ke -= fNy;
        k = ke * fky;
      }
      v[j] = mk<C>(-k * xv.y, k * xv.x);
    }
    __syncthreads();                                          // staging consumed by every thread
    const int tn = next(t + gridDim.x);
    if (tid == 0 && tn < tt.total) { fence_proxy_async(); issue(tn); }
    tile_fft_1buf<E, true>(v, work, lay, line, i, LOGL, lognl, tab, twx);
    C* o = (dir_y ? t2 : t1) + (long long)fl * a.O + c;
#pragma unroll
    for (int j = 0; j < E; ++j) o[(long long)(i + j * LE) * a.S] = v[j];
    __syncthreads();                                          // work buffer free for the next tile
    ph ^= 1;
    t = tn;
  }
}

// Forward y pass of t1 and t2 fused with the operator output, the diagonal
// preconditioner and the dot products (k_psi_cols_comb, FP32, x given):
//   y = P^-1 (a_dt x - (i kx0 t1^ + i ky t2^)); mode 0: dots <c, y>; mode 1: <y, s>, <y, y>.
// The two transforms are lines 0..TW-1 (t1) and TW..2TW-1 (t2) of one tile; the
// holders of a column's t1 and t2 sit TW lanes apart and trade halves of their
// elements by shuffle, so each computes the epilogue of E/2 rows.  Unlike
// k_psi_cols_comb, whose epilogue runs in FP64, y is formed in FP32 (its
// transforms are bit-identical; y differs by FP32 rounding), with the dots in FP64.
template <int E, int NT, int LOGL>
__global__ void __launch_bounds__(NT, E * NT <= 4096 ? 2 : 1) k_psi_cols_comb_tma(
    const __grid_constant__ CUtensorMap mt1, const __grid_constant__ CUtensorMap mt2,
    const __grid_constant__ CUtensorMap mx, const __grid_constant__ CUtensorMap mc, float2* __restrict__ y, int mode,
    const double* __restrict__ adt_r, const double* __restrict__ mmax_r, double S4, ColArgs a, TmaTiles tt, SysMap sm,
    const int* __restrict__ active, int f0, const float2* __restrict__ tab, double2* __restrict__ part,
    int* __restrict__ err) {
  using C = float2;
  constexpr int L = 1 << LOGL, LE = L / E, TW = E * NT / (2 * L), LOGTW = Log2<TW>::v;
  static_assert(TW >= 2 && TW <= 16 && L >= E * E, "tile geometry");
  constexpr int BH = L < 256 ? L : 256, NBOX = L / BH;     // rows per TMA box, boxes per column tile
  __shared__ double smm[2 * 4 * (NT / 32)];
  unsigned char* base = tma_smem_base();
  constexpr size_t tile_n = (size_t)L * TW;
  C* s1 = reinterpret_cast<C*>(base);
  C* s2 = s1 + tile_n;
  C* sxv = s2 + tile_n;
  C* scv = sxv + tile_n;
  C* work = scv + tile_n;
  uint64_t* bar = reinterpret_cast<uint64_t*>(work + col_tile_elems(L, 2 * TW, Log2<E>::v));   // [0] t1 t2, [1] x c
  constexpr int lognl = LOGTW + 1;
  const int tid = threadIdx.x;
  const int line = tid & (2 * TW - 1), i = tid >> lognl, cl = line & (TW - 1);
  const bool is1 = line < TW;
  const uint32_t tx2 = (uint32_t)(2 * tile_n * sizeof(C));
  auto act = [&](int t) { return !active || active[sm.sys(f0 + t / tt.tiles)]; };
  auto next = [&](int t) { while (t < tt.total && !act(t)) t += gridDim.x; return t; };
  auto issue_t = [&](int t) {
    const int fl = t / tt.tiles, c0 = (t % tt.tiles) * TW;
    mbar_arrive_expect_tx(&bar[0], tx2);
    for (int q = 0; q < NBOX; ++q) {
      tma_load_2d(s1 + (size_t)q * BH * TW, &mt1, c0, fl * a.Ny + q * BH, &bar[0]);
      tma_load_2d(s2 + (size_t)q * BH * TW, &mt2, c0, fl * a.Ny + q * BH, &bar[0]);
    }
  };
  auto issue_xc = [&](int t) {
    const int fl = t / tt.tiles, c0 = (t % tt.tiles) * TW;
    mbar_arrive_expect_tx(&bar[1], tx2);
    for (int q = 0; q < NBOX; ++q) {
      tma_load_2d(sxv + (size_t)q * BH * TW, &mx, c0, (f0 + fl) * a.Ny + q * BH, &bar[1]);
      tma_load_2d(scv + (size_t)q * BH * TW, &mc, c0, (f0 + fl) * a.Ny + q * BH, &bar[1]);
    }
  };
  C* twx = tma_twx(bar);
  if (tid == 0) { mbar_init(&bar[0], 1); mbar_init(&bar[1], 1); mbar_fence_init(); }
  tw_last_table<E>(twx, LOGL, tab);
  __syncthreads();
  // tiles of inactive systems get zero dot partials (the per-tile layout of k_psi_cols_comb)
  for (int t = blockIdx.x; t < tt.total; t += gridDim.x)
    if (!act(t) && tid < 4) part[((long long)(f0 + t / tt.tiles) * tt.tiles + t % tt.tiles) * 4 + tid] = make_double2(0.0, 0.0);
  int t = next(blockIdx.x);
  if (tid == 0 && t < tt.total) { issue_t(t); issue_xc(t); }
  const ColLay lay{2 * TW, Log2<E>::v};
  uint32_t ph = 0;
  while (t < tt.total) {
    const int fl = t / tt.tiles, tile = t % tt.tiles, f = f0 + fl, c = tile * TW + cl;
    bool ok = mbar_wait(&bar[0], ph, err);
    if (__syncthreads_or(!ok)) return;
    C v[E];
    const C* st = is1 ? s1 : s2;
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = st[(i + j * LE) * TW + cl];
    __syncthreads();                                          // t1 / t2 staging consumed
    const int tn = next(t + gridDim.x);
    if (tid == 0 && tn < tt.total) { fence_proxy_async(); issue_t(tn); }
    tile_fft_1buf<E, false>(v, work, lay, line, i, LOGL, lognl, tab, twx);
    // trade halves with the partner TW lanes away: the t1 holder keeps rows j < E/2,
    // the t2 holder rows j >= E/2
    constexpr int H = E / 2;
    C w1[H], w2[H];
#pragma unroll
    for (int h = 0; h < H; ++h) {
      const C snd = is1 ? v[h + H] : v[h];
      C rcv;
      rcv.x = __shfl_xor_sync(0xffffffffu, snd.x, TW);
      rcv.y = __shfl_xor_sync(0xffffffffu, snd.y, TW);
      w1[h] = is1 ? v[h] : rcv;                               // t1^ at the row this thread finishes
      w2[h] = is1 ? rcv : v[h + H];                           // t2^
    }
    ok = mbar_wait(&bar[1], ph, err);
    if (__syncthreads_or(!ok)) return;
    // epilogue in FP32 (the solver's arithmetic), the dot products of the stored FP32
    // values in FP64: a plain FP64 sum over this thread's E/2 rows, compensated across
    // threads and blocks
    double d0 = 0.0, d1 = 0.0, d2 = 0.0;
    {
      const int r = sm.run_of[f % sm.V];
      const float adt = (float)adt_r[r], mms4 = mmax_r ? (float)(mmax_r[r] * S4) : 0.f;
      const float kx = (float)(kfreq(c, a.Nx) * a.kxs), fky = (float)a.kys;
      const float fi = (float)i, fLE = (float)LE, fNy = (float)a.Ny;
      C* yo = y + (long long)f * a.O + c;
#pragma unroll
      for (int h = 0; h < H; ++h) {
        const int jj = is1 ? h : h + H;
        const int e = i + jj * LE;
        float ke = fmaf((float)jj, fLE, fi);
        if (e >= (a.Ny >> 1)) ke -= fNy;
        const float ky = ke * fky;
        const C xv = sxv[e * TW + cl], cv = scv[e * TW + cl];
        float ox = fmaf(adt, xv.x, fmaf(kx, w1[h].y, ky * w2[h].y));
        float oy = fmaf(adt, xv.y, -fmaf(kx, w1[h].x, ky * w2[h].x));
        if (mmax_r) {
          const float pinv = 1.0f / fmaf(mms4, fmaf(kx, kx, ky * ky), adt);
          ox *= pinv; oy *= pinv;
        }
        yo[(long long)e * a.S] = mk<C>(ox, oy);
        const double dx = ox, dy = oy, cx = cv.x, cy = cv.y;
        if (mode == 0) {
          d0 = fma(cx, dx, fma(cy, dy, d0));
          d1 = fma(cx, dy, fma(-cy, dx, d1));
        } else {
          d0 = fma(dx, cx, fma(dy, cy, d0));
          d1 = fma(dx, cy, fma(-dy, cx, d1));
          d2 = fma(dx, dx, fma(dy, dy, d2));
        }
      }
    }
    // the tile's dot partials: plain FP64 warp sums (32 terms), compensated across warps
    double d[3] = {d0, d1, d2};
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) d[k] += __shfl_xor_sync(0xffffffffu, d[k], o);
    const int lane = tid & 31, warp = tid >> 5;
    if (lane == 0) { smm[warp] = d[0]; smm[NT / 32 + warp] = d[1]; smm[2 * (NT / 32) + warp] = d[2]; }
    __syncthreads();                                          // x / c staging consumed, warp sums visible
    if (tid == 0 && tn < tt.total) { fence_proxy_async(); issue_xc(tn); }
    if (tid < 4) {
      KSum a2{0.0, 0.0};
      if (tid < 3)
        for (int w = 0; w < NT / 32; ++w) a2.add(smm[tid * (NT / 32) + w]);
      part[((long long)f * tt.tiles + tile) * 4 + tid] = make_double2(a2.s, a2.c);
    }
    ph ^= 1;
    t = tn;
  }
}

// ---------------------------------------------------------------------------
// The FULL x pass of the operator (k_rows_mul, FP32) as a persistent pipeline fed
// by bulk copies.  A tile is NL = NT E / L consecutive rows of one plane (t1 or t2
// of one field) -- one contiguous block of NL L complex floats -- with the NL rows
// of M_psi it needs.  One thread moves both into a ring of S shared-memory slots by
// cp.async.bulk, completed on the slot's mbarrier; the block transforms the tile in
// its slot (the rows are read into registers, then the slot is the padded exchange
// of both transforms), writes the result back into the slot and one thread stores
// it with a bulk copy, so the loads of the next tiles and the store of the last one
// run on the copy engine while a tile is transformed.  The tiles of a row group are
// ordered plane-fastest (t1 and t2 of field 0, then of field 1, ...), so the M_psi
// rows of a group are read from HBM once and reused from L2 by the other planes.
// The butterflies, twiddles and radix split are those of the ping-pong kernel, so
// the results are bit-identical to k_rows_mul<float, E, *, true>.
//   t rows: [2][fc][Ny][L] (t1 | t2 of the chunk's fields f0 .. f0+fc-1).
// Waits on the mbarriers are bounded (tma.cuh): a copy that never lands sets the
// error word and every thread of the block returns.
// ---------------------------------------------------------------------------
template <int E, int NT, int LOGL, int S>
struct BulkRows {
  static constexpr int L = 1 << LOGL, LE = L / E, NL = NT * E / L, LOGE = Log2<E>::v;
  static constexpr int LP = RowLayP<LOGE>::pitch(L);            // padded line of the in-slot exchange
  static constexpr size_t t_elems = ((size_t)NL * LP + 1) / 2 * 2; // complex slots of a ring entry's tile part (16-B multiple)
  static constexpr uint32_t TB = NL * L * 8, MB = NL * L * 4;    // bytes copied per tile: t rows, M rows
  static constexpr size_t slot_bytes = t_elems * 8 + MB;
  static constexpr size_t tw_bytes = (size_t)tw_last_rows<E>() * LE * 8;
  static constexpr size_t smem = 1024 + S * slot_bytes + tw_bytes + 8 * S;
  static constexpr bool ok = NL >= 1 && L >= E * E && NT % 32 == 0 && S >= 2;
};

template <int E, int NT, int LOGL, int S>
__global__ void __launch_bounds__(NT, 2) k_rows_mul_bulk(float2* __restrict__ t, const float* __restrict__ M, float scale,
                                                         int Ny, int fc, int f0, long long ntiles, SysMap sm,
                                                         const int* __restrict__ active, const float2* __restrict__ tab,
                                                         int* __restrict__ err) {
  using C = float2;
  using G = BulkRows<E, NT, LOGL, S>;
  constexpr int L = G::L, LE = G::LE, NL = G::NL, LOGNL = Log2<NL>::v;
  static_assert(G::ok, "tile geometry");
  unsigned char* base = tma_smem_base();
  // ring entry s: the tile's t rows (landing unpadded, then the padded exchange of both
  // transforms, then the result) followed by its M rows
  auto tslot = [&](int s_) { return reinterpret_cast<C*>(base + (size_t)s_ * G::slot_bytes); };
  auto mslot = [&](int s_) { return reinterpret_cast<float*>(base + (size_t)s_ * G::slot_bytes + G::t_elems * 8); };
  C* twx = reinterpret_cast<C*>(base + S * G::slot_bytes);        // twiddles of the last pass, per butterfly
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + S * G::slot_bytes + G::tw_bytes);
  const int tid = threadIdx.x;
  int line, i;
  row_owner<E>(LOGL, line, i);
  const int planes = 2 * fc;
  // tile tau: plane p = tau % planes (t1/t2 of chunk field p / 2), row group tau / planes
  auto act = [&](long long tau) { return !active || active[sm.sys(f0 + (int)(tau % planes) / 2)]; };
  auto next = [&](long long tau) { while (tau < ntiles && !act(tau)) tau += gridDim.x; return tau; };
  auto row_of = [&](long long tau) {
    const int p = (int)(tau % planes), rg = (int)(tau / planes);
    return ((long long)(p & 1) * fc + (p >> 1)) * Ny + (long long)rg * NL;
  };
  auto issue = [&](long long tau, int s_) {
    const long long row = row_of(tau);
    const int field = f0 + (int)(tau % planes) / 2;
    const long long mrow = (long long)(field % sm.V) * Ny + row % Ny;
    mbar_arrive_expect_tx(&bar[s_], G::TB + G::MB);
    bulk_load(tslot(s_), t + row * L, G::TB, &bar[s_]);
    bulk_load(mslot(s_), M + mrow * L, G::MB, &bar[s_]);
  };
  tw_last_table<E>(twx, LOGL, tab);
  if (tid == 0) {
    for (int s_ = 0; s_ < S; ++s_) mbar_init(&bar[s_], 1);
    mbar_fence_init();
  }
  __syncthreads();
  long long cur = next(blockIdx.x);
  long long ld = cur;                       // thread 0: the next tile to load
  if (tid == 0)
    for (int s_ = 0; s_ < S && ld < ntiles; ++s_) { issue(ld, s_); ld = next(ld + gridDim.x); }
  const RowLayP<G::LOGE> lay{G::LP};
  for (int k = 0; cur < ntiles; ++k) {
    const int s_ = k % S;
    const long long row = row_of(cur);
    const bool ok = mbar_wait(&bar[s_], (uint32_t)((k / S) & 1), err);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) bulk_wait_all();
      return;
    }
    C* ts = tslot(s_);
    C v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = ts[(size_t)line * L + i + j * LE];
    __syncthreads();                                          // the landed rows are consumed: the slot is the exchange
    // the slot of the previous tile: its bulk store has had this tile's wait to read it; refill
    if (tid == 0 && k > 0 && ld < ntiles) {
      bulk_wait_read_all();
      issue(ld, (k + S - 1) % S);
      ld = next(ld + gridDim.x);
    }
    tile_fft_1buf<E, true>(v, ts, lay, line, i, LOGL, LOGNL, tab, twx);
    const float* ms = mslot(s_) + (size_t)line * L + i;
#pragma unroll
    for (int j = 0; j < E; ++j) { const float mv = ms[j * LE] * scale; v[j].x *= mv; v[j].y *= mv; }
    __syncthreads();                                          // exchange reused by the forward transform
    tile_fft_1buf<E, false>(v, ts, lay, line, i, LOGL, LOGNL, tab, twx);
    __syncthreads();                                          // every exchange read done: the slot takes the result
#pragma unroll
    for (int j = 0; j < E; ++j) ts[(size_t)line * L + i + j * LE] = v[j];
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) { bulk_store(t + row * L, ts, G::TB); bulk_commit(); }
    cur = next(cur + gridDim.x);
  }
  if (tid == 0) bulk_wait_all();
}

// The 3D full-spectrum operator output (the 2D FULL form with a z direction):
//   y = P^-1 ( a_dt x - (i kx0 t1 + i ky t2 + i kz t3) ),  P^-1 = 1/(a_dt + Mmax S4 k^2) or 1,
// with k_psi_combine's modes and dot products.  t1..t3 hold F fields each.
template <typename T>
__global__ void __launch_bounds__(256) k_psi_combine3(const cplx<T>* __restrict__ x, const cplx<T>* __restrict__ t1,
                                                      const cplx<T>* __restrict__ t2, const cplx<T>* __restrict__ t3,
                                                      cplx<T>* __restrict__ y, const cplx<T>* __restrict__ cvec,
                                                      const cplx<T>* __restrict__ svec, int mode,
                                                      const double* __restrict__ adt_r, const double* __restrict__ mmax_r,
                                                      double S4, VGeom g, SysMap sm, const int* __restrict__ active, EW ew,
                                                      double2* part) {
  __shared__ double smm[2 * 4 * 8];
  KSum acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  const int f = blockIdx.y;
  if (!active || active[sm.sys(f)]) {
    const int r = sm.run_of[f % sm.V];
    const double adt = adt_r[r], mm = mmax_r ? mmax_r[r] : 0.0;
    const long long beg = (long long)blockIdx.x * ew.chunk, end = min(ew.n, beg + ew.chunk);
    for (long long s = beg + threadIdx.x; s < end; s += blockDim.x) {
      const unsigned su = (unsigned)s;
      const double kxv = kfreq((int)(su & (unsigned)(g.Nx - 1)), g.Nx) * g.kxs;
      const double kyv = kfreq((int)((su >> g.logNx) & (unsigned)(g.Ny - 1)), g.Ny) * g.kys;
      const double kzv = kfreq((int)(su >> (g.logNx + g.logNy)), g.Nz) * g.kzs;
      const long long j = (long long)f * g.n + s;
      const cplx<T> xv = x ? x[j] : cplx<T>{}, a = t1[j], b = t2[j], c = t3[j];
      const double dx = -(kxv * (double)a.y + kyv * (double)b.y + kzv * (double)c.y);
      const double dy = kxv * (double)a.x + kyv * (double)b.x + kzv * (double)c.x;
      double ox = adt * (double)xv.x - dx, oy = adt * (double)xv.y - dy;
      if (mmax_r) {
        const double pinv = 1.0 / (adt + mm * S4 * (kxv * kxv + kyv * kyv + kzv * kzv));
        ox *= pinv; oy *= pinv;
      }
      cplx<T> ot; ot.x = ox; ot.y = oy;
      y[j] = ot;
      ox = ot.x; oy = ot.y;                                 // the dots use the stored (rounded) values
      if (mode == 0) {
        const cplx<T> cv = cvec[j];
        acc[0].add((double)cv.x * ox + (double)cv.y * oy);
        acc[1].add((double)cv.x * oy - (double)cv.y * ox);
      } else {
        const cplx<T> sv = svec[j];
        acc[0].add(ox * (double)sv.x + oy * (double)sv.y);
        acc[1].add(ox * (double)sv.y - oy * (double)sv.x);
        acc[2].add(ox * ox + oy * oy);
      }
    }
  }
  block_reduce_store<4>(acc, part + ((long long)f * ew.bpf + blockIdx.x) * 4, smm);
}

// The same forward pass split in two (the autotuner picks whichever is faster):
//  k_psi_cols_fwd2: forward y pass of t1 and t2 reduced to z = i kx0 t1^ + i ky t2^,
//                   written over t1 (the CTA has read its tile before it writes);
//  k_psi_combz:     y = P^-1 (a_dt x - z) with the dot products, a streaming pass.
template <typename T, int E, int NT>
__global__ void __launch_bounds__(NT, MinB<E, NT>::v) k_psi_cols_fwd2(cplx<T>* t1, const cplx<T>* __restrict__ t2, ColArgs a,
                                                                   SysMap sm, const int* __restrict__ active, int f0,
                                                                   const cplx<T>* __restrict__ tab) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  const int L = 1 << a.logL, LE = L / E;
  const int tile = blockIdx.x % a.tiles;
  const int fl = blockIdx.x / a.tiles;
  if (active && !active[sm.sys(f0 + fl)]) return;          // block-uniform
  const int cl = threadIdx.x & (a.TW - 1), i = threadIdx.x >> a.logTW, c = tile * a.TW + cl;
  const bool valid = c < a.W;
  const ColLay lay{a.TW, Log2<E>::v};
  C* const buf[2] = {s, s + col_tile_elems(L, a.TW, Log2<E>::v)};
  C* const res = s + 2 * col_tile_elems(L, a.TW, Log2<E>::v);
  const long long off = (long long)fl * a.O + c;
  C v[E];
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = valid ? t2[off + (long long)(i + j * LE) * a.S] : mk<C>(0.0, 0.0);
  tile_fft<E, false, true, true>(v, buf, lay, cl, i, true, a.logL, a.logTW, tab);
#pragma unroll
  for (int j = 0; j < E; ++j) res[(i + j * LE) * a.TW + cl] = v[j];
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = valid ? t1[off + (long long)(i + j * LE) * a.S] : mk<C>(0.0, 0.0);
  __syncthreads();                                          // the first transform's smem reads are done
  tile_fft<E, false, true, true>(v, buf, lay, cl, i, true, a.logL, a.logTW, tab);
  if (!valid) return;
  if constexpr (std::is_same<T, float>::value) {
    const float kxv = (float)(kfreq(c, a.Nx) * a.kxs), fky = (float)a.kys;
    const float fi = (float)i, fLE = (float)LE, fNy = (float)a.Ny;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int e = i + j * LE;
      float ke = fmaf((float)j, fLE, fi);
      if (e >= (a.Ny >> 1)) ke -= fNy;
      const float kyv = ke * fky;
      const C w2 = res[e * a.TW + cl];
      t1[off + (long long)e * a.S] = mk<C>(-(kxv * v[j].y + kyv * w2.y), kxv * v[j].x + kyv * w2.x);
    }
  } else {
    const double kxv = kfreq(c, a.Nx) * a.kxs;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int e = i + j * LE;
      const double kyv = kfreq(e, a.Ny) * a.kys;
      const C w2 = res[e * a.TW + cl];
      t1[off + (long long)e * a.S] = mk<C>(-(kxv * (double)v[j].y + kyv * (double)w2.y),
                                           kxv * (double)v[j].x + kyv * (double)w2.x);
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_psi_combz(const cplx<T>* __restrict__ x, const cplx<T>* __restrict__ z,
                                                   cplx<T>* __restrict__ y, const cplx<T>* __restrict__ cvec,
                                                   const cplx<T>* __restrict__ svec, int mode,
                                                   const double* __restrict__ adt_r, const double* __restrict__ mmax_r,
                                                   double S4, VGeom g, SysMap sm, const int* __restrict__ active, int f0,
                                                   EW ew, double2* part) {
  __shared__ double smm[2 * 4 * 8];
  KSum acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  // z is chunk-local (field blockIdx.y of the chunk); x, y, c, s are global (field f0 + blockIdx.y)
  const int f = f0 + blockIdx.y;
  z -= ((long long)f - blockIdx.y) * g.n;
  const int sy = sm.sys(f);
  const int r = sm.run_of[f % sm.V];
  if (!active || active[sy]) {
    const double adt = adt_r[r], mm = mmax_r ? mmax_r[r] : 0.0;
    const long long beg = (long long)blockIdx.x * ew.chunk, end = min(ew.n, beg + ew.chunk);
    constexpr int U = 4;
    for (long long s0 = beg + threadIdx.x; s0 < end; s0 += U * blockDim.x) {
      cplx<T> xv[U], zv[U], cv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const long long s = s0 + (long long)u * blockDim.x;
        if (s < end) {
          const long long j = (long long)f * g.n + s;
          xv[u] = x ? x[j] : cplx<T>{};
          zv[u] = z[j];
          cv[u] = mode == 0 ? cvec[j] : svec[j];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const long long s = s0 + (long long)u * blockDim.x;
        if (s >= end) break;
        int kx, ky; double kxv, kyv, w;
        vk(g, s, kx, ky, kxv, kyv, w);
        double ox = adt * (double)xv[u].x - (double)zv[u].x, oy = adt * (double)xv[u].y - (double)zv[u].y;
        if (mmax_r) {
          const double pinv = 1.0 / (adt + mm * S4 * (kxv * kxv + kyv * kyv));
          ox *= pinv; oy *= pinv;
        }
        cplx<T> ot; ot.x = ox; ot.y = oy;
        y[(long long)f * g.n + s] = ot;
        ox = ot.x; oy = ot.y;                               // the dots use the stored (rounded) values
        const cplx<T> c = cv[u];
        if (mode == 0) {
          acc[0].add((double)c.x * ox + (double)c.y * oy);
          acc[1].add((double)c.x * oy - (double)c.y * ox);
        } else {
          acc[0].add(ox * (double)c.x + oy * (double)c.y);
          acc[1].add(ox * (double)c.y - oy * (double)c.x);
          acc[2].add(ox * ox + oy * oy);
        }
      }
    }
  }
  block_reduce_store<4>(acc, part + ((long long)f * ew.bpf + blockIdx.x) * 4, smm);
}

// slots per thread per round of the Krylov vector passes (loads in flight together)
constexpr int VB = 4;

// r = M^-1 b, x = 0, p = r, dots <b, r>, ||r||^2, ||b||^2  (Krylov.jl bicgstab initialisation)
template <typename T>
__global__ void __launch_bounds__(256) k_psi_init(const cplx<T>* __restrict__ b, cplx<T>* __restrict__ x, cplx<T>* __restrict__ r,
                                                  cplx<T>* __restrict__ p, const double* __restrict__ adt_r,
                                                  const double* __restrict__ mmax_r, double S4, VGeom g, SysMap sm,
                                                  EW ew, double2* part) {
  __shared__ double smm[2 * 4 * 8];
  KSum acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  const int f = blockIdx.y;
  const int rr = sm.run_of[f % sm.V];
  const double adt = adt_r[rr], mm = mmax_r ? mmax_r[rr] : 0.0;
  const long long beg = (long long)blockIdx.x * ew.chunk, end = min(ew.n, beg + ew.chunk);
  if constexpr (std::is_same<T, float>::value) {
    // FP32 solve: r = M^-1 b in FP32, the dot terms as FP32 products summed over a
    // round of VB slots, the rounds accumulated in FP64 (as k_psi_update)
    const float fadt = (float)adt, mms4 = (float)(mm * S4);
    for (long long qb = beg + threadIdx.x; qb < end; qb += VB * blockDim.x) {
      float2 bv[VB];
#pragma unroll
      for (int u = 0; u < VB; ++u) {
        const long long q = qb + (long long)u * blockDim.x;
        if (q < end) bv[u] = b[(long long)f * g.n + q];
      }
      float d0 = 0.f, d1 = 0.f, d2 = 0.f, d3 = 0.f;
#pragma unroll
      for (int u = 0; u < VB; ++u) {
        const long long q = qb + (long long)u * blockDim.x;
        if (q >= end) break;
        const long long j = (long long)f * g.n + q;
        float k2, w;
        vk_f32(g, q, k2, w);
        const float2 z = make_float2(0.f, 0.f);
        x[j] = z;
        if (w == 0.f) { r[j] = z; p[j] = z; continue; }
        const float pinv = mmax_r ? 1.0f / fmaf(mms4, k2, fadt) : 1.f;
        const float2 rv = make_float2(bv[u].x * pinv, bv[u].y * pinv);
        r[j] = rv; p[j] = rv;
        d0 = fmaf(w, fmaf(bv[u].x, rv.x, bv[u].y * rv.y), d0);
        d1 += fmaf(bv[u].x, rv.y, -bv[u].y * rv.x);
        d2 = fmaf(w, fmaf(rv.x, rv.x, rv.y * rv.y), d2);
        d3 = fmaf(w, fmaf(bv[u].x, bv[u].x, bv[u].y * bv[u].y), d3);
      }
      acc[0].add((double)d0);
      if (g.full) acc[1].add((double)d1);
      acc[2].add((double)d2);
      acc[3].add((double)d3);
    }
  } else {
#pragma unroll 4
    for (long long s = beg + threadIdx.x; s < end; s += blockDim.x) {
      int kx, ky; double kxv, kyv, w;
      vk(g, s, kx, ky, kxv, kyv, w);
      long long j = (long long)f * g.n + s;
      cplx<T> z{};
      x[j] = z;
      if (w == 0.0) { r[j] = z; p[j] = z; continue; }
      cplx<T> bv = b[j];
      double kxp = (!g.full && kx == g.Nx / 2) ? 0.0 : kxv;
      double pinv = mmax_r ? 1.0 / (adt + mm * S4 * (kxp * kxp + kyv * kyv + vk_kz2(g, s))) : 1.0;
      cplx<T> rv; rv.x = (double)bv.x * pinv; rv.y = (double)bv.y * pinv;
      r[j] = rv; p[j] = rv;
      acc[0].add(w * ((double)bv.x * (double)rv.x + (double)bv.y * (double)rv.y));
      if (g.full) acc[1].add((double)bv.x * (double)rv.y - (double)bv.y * (double)rv.x);
      acc[2].add(w * ((double)rv.x * (double)rv.x + (double)rv.y * (double)rv.y));
      acc[3].add(w * ((double)bv.x * (double)bv.x + (double)bv.y * (double)bv.y));   // ||b||^2: the true residual of x0 = 0
    }
  }
  block_reduce_store<4>(acc, part + ((long long)blockIdx.y * ew.bpf + blockIdx.x) * 4, smm);
}

// s = r - alpha v.  Each thread loads VB slots of both operands before it
// computes, so several loads per thread are in flight.
template <typename T>
__global__ void __launch_bounds__(256) k_psi_s(const cplx<T>* __restrict__ r, const cplx<T>* __restrict__ v,
                                               cplx<T>* __restrict__ s, const BiState* __restrict__ st, SysMap sm, EW ew) {
  const BiState& b = st[sm.sys(blockIdx.y)];
  if (!b.active) return;
  const double2 a = b.alpha;
  const long long base = (long long)blockIdx.y * ew.n;
  const long long q0 = (long long)blockIdx.x * ew.chunk, q1 = min(ew.n, q0 + ew.chunk);
  for (long long qb = q0 + threadIdx.x; qb < q1; qb += VB * blockDim.x) {
    cplx<T> rv[VB], vv[VB];
#pragma unroll
    for (int u = 0; u < VB; ++u) {
      const long long q = qb + (long long)u * blockDim.x;
      if (q < q1) { rv[u] = r[base + q]; vv[u] = v[base + q]; }
    }
#pragma unroll
    for (int u = 0; u < VB; ++u) {
      const long long q = qb + (long long)u * blockDim.x;
      if (q >= q1) break;
      cplx<T> o;
      o.x = (double)rv[u].x - (a.x * (double)vv[u].x - a.y * (double)vv[u].y);
      o.y = (double)rv[u].y - (a.x * (double)vv[u].y + a.y * (double)vv[u].x);
      s[base + q] = o;
    }
  }
}

// x = (x + alpha p) + omega s ;  r = s - omega t ; dots <c, r>, ||r||^2, ||D r||^2
// (flexible right-preconditioned form: p and shat are the preconditioned
// directions used for x, s the unpreconditioned one used for r).
// D = a_dt + M_max S4 |k|^2 is the inverse of the diagonal preconditioner: in the
// left-preconditioned form r = M^-1 (b - A x), so ||D r|| is the norm of the true
// residual b - A x, at no extra pass (mmax_r == nullptr: D = 1, r is already true).
template <typename T>
__global__ void __launch_bounds__(256, 2) k_psi_update(cplx<T>* __restrict__ x, cplx<T>* __restrict__ r, const cplx<T>* __restrict__ p,
                                                    const cplx<T>* __restrict__ s, const cplx<T>* __restrict__ t,
                                                    const cplx<T>* __restrict__ cvec, const BiState* __restrict__ st,
                                                    VGeom g, SysMap sm, EW ew, double2* part,
                                                    const cplx<T>* __restrict__ shat, const double* __restrict__ adt_r,
                                                    const double* __restrict__ mmax_r, double S4) {
  __shared__ double smm[2 * 4 * 8];
  // per-thread sums: compensated in the FP64 solve (parity path); plain FP64 in the
  // FP32 solve, whose terms are products of FP32 values (a thread sums ~100 of them,
  // ~1e-14 relative), compensated across threads and blocks either way
  using Acc = typename std::conditional<std::is_same<T, float>::value, PlainSum, KSum>::type;
  Acc acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  const int f = blockIdx.y;
  const BiState& b = st[sm.sys(f)];
  if constexpr (std::is_same<T, float>::value) {
    // FP32 solve: the updates in FP32 arithmetic (the solve's own precision) and the
    // dot terms as FP32 products summed over the VB slots of a round, each round's
    // four partials added in FP64 -- one float-to-double conversion per slot instead
    // of ~20, which otherwise bound this pass below the copy bandwidth
    if (b.active) {
      const float2 al = make_float2((float)b.alpha.x, (float)b.alpha.y);
      const float2 om = make_float2((float)b.omega.x, (float)b.omega.y);
      const int run = sm.run_of[f % sm.V];
      const float adt = mmax_r ? (float)adt_r[run] : 0.f, mms4 = mmax_r ? (float)(mmax_r[run] * S4) : 0.f;
      const long long base = (long long)f * g.n;
      const long long beg = (long long)blockIdx.x * ew.chunk, end = min(ew.n, beg + ew.chunk);
      for (long long qb = beg + threadIdx.x; qb < end; qb += VB * blockDim.x) {
        float2 xv[VB], pv[VB], sv[VB], tv[VB], hv[VB], cv[VB];
#pragma unroll
        for (int u = 0; u < VB; ++u) {
          const long long q = qb + (long long)u * blockDim.x;
          if (q < end) {
            const long long j = base + q;
            xv[u] = x[j]; pv[u] = p[j]; sv[u] = s[j]; tv[u] = t[j]; cv[u] = cvec[j];
            hv[u] = shat ? shat[j] : sv[u];
          }
        }
        float d0 = 0.f, d1 = 0.f, d2 = 0.f, d3 = 0.f;
#pragma unroll
        for (int u = 0; u < VB; ++u) {
          const long long q = qb + (long long)u * blockDim.x;
          if (q >= end) break;
          float k2, w;
          vk_f32(g, q, k2, w);
          if (w == 0.f) continue;
          const long long j = base + q;
          float2 xa, xn, rn;
          xa.x = fmaf(al.x, pv[u].x, fmaf(-al.y, pv[u].y, xv[u].x));
          xa.y = fmaf(al.x, pv[u].y, fmaf(al.y, pv[u].x, xv[u].y));
          xn.x = fmaf(om.x, hv[u].x, fmaf(-om.y, hv[u].y, xa.x));
          xn.y = fmaf(om.x, hv[u].y, fmaf(om.y, hv[u].x, xa.y));
          x[j] = xn;
          rn.x = fmaf(-om.x, tv[u].x, fmaf(om.y, tv[u].y, sv[u].x));
          rn.y = fmaf(-om.x, tv[u].y, fmaf(-om.y, tv[u].x, sv[u].y));
          r[j] = rn;
          const float2 c = cv[u];
          d0 = fmaf(w, fmaf(c.x, rn.x, c.y * rn.y), d0);
          d1 += fmaf(c.x, rn.y, -c.y * rn.x);
          const float rr = fmaf(rn.x, rn.x, rn.y * rn.y);
          d2 = fmaf(w, rr, d2);
          const float dd = mmax_r ? fmaf(mms4, k2, adt) : 1.f;
          d3 = fmaf(w * dd, dd * rr, d3);
        }
        acc[0].add((double)d0);
        if (g.full) acc[1].add((double)d1);
        acc[2].add((double)d2);
        acc[3].add((double)d3);
      }
    }
  } else if (b.active) {
    const double2 al = b.alpha, om = b.omega;
    const int run = sm.run_of[f % sm.V];
    const double adt = mmax_r ? adt_r[run] : 0.0, mm = mmax_r ? mmax_r[run] : 0.0;
    const long long base = (long long)f * g.n;
    const long long beg = (long long)blockIdx.x * ew.chunk, end = min(ew.n, beg + ew.chunk);
    // VB slots per thread per round: every operand of the round is loaded before any
    // arithmetic, so the loads are in flight together
    for (long long qb = beg + threadIdx.x; qb < end; qb += VB * blockDim.x) {
      cplx<T> xv[VB], pv[VB], sv[VB], tv[VB], hv[VB], cv[VB];
#pragma unroll
      for (int u = 0; u < VB; ++u) {
        const long long q = qb + (long long)u * blockDim.x;
        if (q < end) {
          const long long j = base + q;
          xv[u] = x[j]; pv[u] = p[j]; sv[u] = s[j]; tv[u] = t[j]; cv[u] = cvec[j];
          hv[u] = shat ? shat[j] : sv[u];
        }
      }
#pragma unroll
      for (int u = 0; u < VB; ++u) {
        const long long q = qb + (long long)u * blockDim.x;
        if (q >= end) break;
        int kx, ky; double kxv, kyv, w;
        vk(g, q, kx, ky, kxv, kyv, w);
        if (w == 0.0) continue;
        const long long j = base + q;
        cplx<T> xa;
        xa.x = (double)xv[u].x + (al.x * (double)pv[u].x - al.y * (double)pv[u].y);
        xa.y = (double)xv[u].y + (al.x * (double)pv[u].y + al.y * (double)pv[u].x);
        cplx<T> xn;
        xn.x = (double)xa.x + (om.x * (double)hv[u].x - om.y * (double)hv[u].y);
        xn.y = (double)xa.y + (om.x * (double)hv[u].y + om.y * (double)hv[u].x);
        x[j] = xn;
        cplx<T> rn;
        rn.x = (double)sv[u].x - (om.x * (double)tv[u].x - om.y * (double)tv[u].y);
        rn.y = (double)sv[u].y - (om.x * (double)tv[u].y + om.y * (double)tv[u].x);
        r[j] = rn;
        const cplx<T> c = cv[u];
        acc[0].add(w * ((double)c.x * (double)rn.x + (double)c.y * (double)rn.y));
        if (g.full) acc[1].add((double)c.x * (double)rn.y - (double)c.y * (double)rn.x);
        const double rr = (double)rn.x * (double)rn.x + (double)rn.y * (double)rn.y;
        acc[2].add(w * rr);
        double dd = 1.0;
        if (mmax_r) {
          const double kxp = (!g.full && kx == g.Nx / 2) ? 0.0 : kxv;
          dd = adt + mm * S4 * (kxp * kxp + kyv * kyv + vk_kz2(g, q));
        }
        acc[3].add(w * dd * dd * rr);
      }
    }
  }
  KSum ks[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) ks[k] = {acc[k].s, acc[k].c};
  block_reduce_store<4>(ks, part + ((long long)blockIdx.y * ew.bpf + blockIdx.x) * 4, smm);
}

// p = r + beta (p - omega v)   (only systems that were active in this iteration: flag `upd`)
template <typename T>
__global__ void __launch_bounds__(256) k_psi_p(cplx<T>* __restrict__ p, const cplx<T>* __restrict__ r,
                                               const cplx<T>* __restrict__ v, const BiState* __restrict__ st,
                                               const int* __restrict__ upd, SysMap sm, EW ew) {
  const int sy = sm.sys(blockIdx.y);
  if (!upd[sy]) return;
  const double2 be = st[sy].beta, om = st[sy].omega;
  const long long base = (long long)blockIdx.y * ew.n;
  const long long q0 = (long long)blockIdx.x * ew.chunk, q1 = min(ew.n, q0 + ew.chunk);
  for (long long qb = q0 + threadIdx.x; qb < q1; qb += VB * blockDim.x) {
    cplx<T> pv[VB], rv[VB], vv[VB];
#pragma unroll
    for (int u = 0; u < VB; ++u) {
      const long long q = qb + (long long)u * blockDim.x;
      if (q < q1) { pv[u] = p[base + q]; rv[u] = r[base + q]; vv[u] = v[base + q]; }
    }
#pragma unroll
    for (int u = 0; u < VB; ++u) {
      const long long q = qb + (long long)u * blockDim.x;
      if (q >= q1) break;
      const double ax = (double)pv[u].x - (om.x * (double)vv[u].x - om.y * (double)vv[u].y);
      const double ay = (double)pv[u].y - (om.x * (double)vv[u].y + om.y * (double)vv[u].x);
      cplx<T> o;
      o.x = (double)rv[u].x + (be.x * ax - be.y * ay);
      o.y = (double)rv[u].y + (be.x * ay + be.y * ax);
      p[base + q] = o;
    }
  }
}

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

// sums per system of per-field dot totals fd[f*4 + 0..3]
__device__ __forceinline__ void sys_sums(const double* fd, int sy, const SysMap& sm, int F, double out[4]) {
  out[0] = out[1] = out[2] = out[3] = 0.0;
  int j = sy / sm.R, r = sy % sm.R;
  for (int v = 0; v < sm.V; ++v) {
    if (sm.run_of[v] != r) continue;
    int f = j * sm.V + v;
    for (int k = 0; k < 4; ++k) out[k] += fd[f * 4 + k];
  }
}

// stop_true: stop on the true residual ||b - A x|| <= atol + rtol ||b|| (slot 3 of the
// dots) instead of Krylov.jl's preconditioned ||M^-1 r|| <= atol + rtol ||M^-1 b|| (slot 2)
static __global__ void k_bi_init(const double* __restrict__ fd, BiState* __restrict__ st, int* __restrict__ upd, SysMap sm, int S, int F,
                          double atol, double rtol, int itmax, int stop_true) {
  int sy = blockIdx.x * blockDim.x + threadIdx.x;
  if (sy >= S) return;
  double d[4];
  sys_sums(fd, sy, sm, F, d);
  BiState b{};
  b.rnorm = sqrt(stop_true ? d[3] : d[2]);
  b.eps = atol + rtol * b.rnorm;
  b.rho = make_double2(d[0], d[1]);
  b.alpha = b.omega = make_double2(1.0, 0.0);
  b.iters = 0;
  if (b.rnorm == 0.0) { b.solved = 1; b.status = 4; b.active = 0; }
  else if (b.rho.x == 0.0 && b.rho.y == 0.0) { b.solved = 0; b.status = 3; b.active = 0; }
  else {
    b.solved = b.rnorm <= b.eps;
    b.active = !(b.solved || itmax <= 0);
    b.status = b.solved ? 1 : (b.active ? 0 : 2);
  }
  st[sy] = b;
  upd[sy] = b.active;
}
static __global__ void k_bi_alpha(const double* __restrict__ fd, BiState* __restrict__ st, SysMap sm, int S, int F) {
  int sy = blockIdx.x * blockDim.x + threadIdx.x;
  if (sy >= S || !st[sy].active) return;
  double d[4];
  sys_sums(fd, sy, sm, F, d);
  st[sy].alpha = cdiv(st[sy].rho, make_double2(d[0], d[1]));
}
static __global__ void k_bi_omega(const double* __restrict__ fd, BiState* __restrict__ st, SysMap sm, int S, int F) {
  int sy = blockIdx.x * blockDim.x + threadIdx.x;
  if (sy >= S || !st[sy].active) return;
  double d[4];
  sys_sums(fd, sy, sm, F, d);
  st[sy].omega = cdiv(make_double2(d[0], d[1]), make_double2(d[2], 0.0));
}
static __global__ void k_bi_beta(const double* __restrict__ fd, BiState* __restrict__ st, int* __restrict__ upd, SysMap sm, int S, int F,
                          int itmax, int* __restrict__ any_active, int stop_true) {
  int sy = blockIdx.x * blockDim.x + threadIdx.x;
  if (sy >= S) return;
  BiState b = st[sy];
  upd[sy] = b.active;
  if (!b.active) return;
  double d[4];
  sys_sums(fd, sy, sm, F, d);
  double2 nr = make_double2(d[0], d[1]);
  b.beta = cmul(cdiv(nr, b.rho), cdiv(b.alpha, b.omega));
  b.rho = nr;
  b.rnorm = sqrt(stop_true ? d[3] : d[2]);
  b.iters += 1;
  bool mach = (b.rnorm + 1.0 <= 1.0);
  bool solved = (b.rnorm <= b.eps) || mach;
  bool tired = b.iters >= itmax;
  bool brk = (b.alpha.x == 0.0 && b.alpha.y == 0.0) || isnan(b.alpha.x) || isnan(b.alpha.y);
  b.solved = solved;
  b.active = !(solved || tired || brk);
  b.status = solved ? 1 : (brk ? 3 : (tired ? 2 : 0));
  st[sy] = b;
  if (b.active) atomicOr(any_active, 1);
}

// ---------------------------------------------------------------------------
// measured true residual of a finished solve: per field ||b - Ax||^2 and ||b||^2
// (slots 0 and 1), then per system ||b - Ax|| / ||b||
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_psi_resnorm(const cplx<T>* __restrict__ b, const cplx<T>* __restrict__ ax, VGeom g,
                                                     EW ew, double2* part) {
  __shared__ double smm[2 * 4 * 8];
  KSum acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  const int f = blockIdx.y;
  const long long beg = (long long)blockIdx.x * ew.chunk, end = min(ew.n, beg + ew.chunk);
  for (long long q = beg + threadIdx.x; q < end; q += blockDim.x) {
    int kx, ky; double kxv, kyv, w;
    vk(g, q, kx, ky, kxv, kyv, w);
    if (w == 0.0) continue;
    const long long j = (long long)f * g.n + q;
    const cplx<T> bv = b[j], av = ax[j];
    const double rx = (double)bv.x - (double)av.x, ry = (double)bv.y - (double)av.y;
    acc[0].add(w * (rx * rx + ry * ry));
    acc[1].add(w * ((double)bv.x * (double)bv.x + (double)bv.y * (double)bv.y));
  }
  block_reduce_store<4>(acc, part + ((long long)blockIdx.y * ew.bpf + blockIdx.x) * 4, smm);
}
static __global__ void k_psi_true_res(const double* __restrict__ fd, double* __restrict__ out, SysMap sm, int S, int F) {
  int sy = blockIdx.x * blockDim.x + threadIdx.x;
  if (sy >= S) return;
  double d[4];
  sys_sums(fd, sy, sm, F, d);
  out[sy] = d[1] > 0.0 ? sqrt(d[0] / d[1]) : 0.0;
}

// ---------------------------------------------------------------------------
// flexible BiCGSTAB preconditioners (an addition: the reference preconditions
// on the left with the diagonal only)
// ---------------------------------------------------------------------------
// out = D^-1 in,  D = a_dt + M_max S4 |k|^2  (the diagonal of Solvers.jl:57)
template <typename T>
__global__ void k_psi_diag(const cplx<T>* __restrict__ in, cplx<T>* __restrict__ out, const double* __restrict__ adt_r,
                           const double* __restrict__ mmax_r, double S4, VGeom g, SysMap sm, EW ew) {
  const int f = blockIdx.y;
  const int r = sm.run_of[f % sm.V];
  const double adt = adt_r[r], mm = mmax_r[r];
  const long long beg = (long long)blockIdx.x * ew.chunk, end = min(ew.n, beg + ew.chunk);
  for (long long q = beg + threadIdx.x; q < end; q += blockDim.x) {
    int kx, ky; double kxv, kyv, w;
    vk(g, q, kx, ky, kxv, kyv, w);
    const long long j = (long long)f * g.n + q;
    cplx<T> o{};
    if (w != 0.0) {
      double kxp = (!g.full && kx == g.Nx / 2) ? 0.0 : kxv;
      double pinv = 1.0 / (adt + mm * S4 * (kxp * kxp + kyv * kyv));
      cplx<T> v = in[j];
      o.x = (double)v.x * pinv; o.y = (double)v.y * pinv;
    }
    out[j] = o;
  }
}

// per-field sum of (Re w)^2 over a complex physical field [F][n]
template <typename T>
__global__ void __launch_bounds__(256) k_re_sumsq(const cplx<T>* __restrict__ w, EW ew, double2* part) {
  __shared__ double smm[2 * 1 * 8];
  KSum acc[1] = {{0, 0}};
  const int f = blockIdx.y;
  const long long beg = (long long)blockIdx.x * ew.chunk, end = min(ew.n, beg + ew.chunk);
  for (long long q = beg + threadIdx.x; q < end; q += blockDim.x) {
    const double v = (double)w[(long long)f * ew.n + q].x;
    acc[0].add(v * v);
  }
  block_reduce_store<1>(acc, part + ((long long)f * ew.bpf + blockIdx.x), smm);
}
// inv_s[f] = 1 / RMS (0 for a zero field)
static __global__ void k_inv_rms(const double* __restrict__ fd, double n, float* __restrict__ inv_s, int F) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  double ms = fd[f] / n;
  inv_s[f] = ms > 0.0 ? (float)(1.0 / sqrt(ms)) : 0.f;
}
// out[i] = (float) Re z[i]
template <typename T>
__global__ void k_take_re(const cplx<T>* __restrict__ z, float* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)z[i].x;
}

// full -> half truncation of the solution (Solvers.jl:79):  half[f][y][kx] = full[f][y][kx], kx < nkx
template <typename T>
__global__ void k_trunc(const cplx<T>* __restrict__ full, cplx<T>* __restrict__ half, int Nx, int Ny, int kp, int nkx, int F) {
  long long tot = (long long)F * Ny * kp;
  K_LOOP(tot, i) {
    int kx = (int)(i % kp);
    long long row = i / kp;
    cplx<T> z{};
    if (kx < nkx) z = full[row * Nx + kx];
    half[i] = z;
  }
}

}  // namespace vsav
