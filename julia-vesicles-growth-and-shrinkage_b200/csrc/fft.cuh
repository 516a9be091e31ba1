// Batched power-of-two FFTs for the SAV step, written for sm_100a.
//
// Replaces the FFTW plans of the reference (src/SpectralUtils.jl:61-71,
// src/SpectralUtils_3d.jl:72-82): rfft / irfft over (x, y[, z]) for N-batched,
// single and velocity fields, and the full complex fft / ifft of the psi
// BiCGSTAB (src/Solvers.jl:45-50,70-71).
//
// Design:
//  * one CTA owns a tile of E*nthreads complex elements in shared memory:
//    nl whole rows (x pass) or TW whole columns (y / z pass), so each pass over
//    HBM reads and writes every element exactly once, coalesced;
//  * inside the tile: Stockham autosort passes of radix 2..16; every thread
//    stages its E elements of a pass in registers (read all, barrier, write
//    all), so the transform is in place with one padded buffer;
//  * real transforms use the half-length complex trick with the pre/post
//    processing fused into the x pass; the c2r keeps only Re of the kx=0 and
//    kx=Nx/2 bins, the FFTW/pocketfft convention the reference relies on;
//  * the first pass of an inverse and the last pass of a forward transform
//    take fused pointwise work (linear combinations, derivative multipliers).
//  Twiddles come from one host-built table: tab[n + m] = exp(-2 pi i m / n).
#pragma once
#include "vsav_internal.cuh"

namespace vsav {

// ---------------------------------------------------------------------------
// shared-memory layout: one pad slot every 16 elements, plus an odd shift per
// line so transposed (column) loads spread over the banks
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int line_pitch(int L) { return L + (L >> 4) + 1; }
__device__ __forceinline__ int sidx(int line, int LP, int e) { return line * LP + e + (e >> 4); }

// in-register DFT of size R (power of two <= 16), radix-2 DIT on bit-reversed input
template <int R> struct Log2 { static constexpr int v = (R <= 1) ? 0 : 1 + Log2<R / 2>::v; };

template <typename C, bool INV>
__device__ __forceinline__ C tw16(C a, int m) {
  // multiply by exp(-+2 pi i m/16), m in [0,8)
  const double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173, h = 0.70710678118654752440;
  double cr, ci;
  switch (m) {
    case 0: return a;
    case 1: cr = c1; ci = s1; break;
    case 2: cr = h; ci = h; break;
    case 3: cr = s1; ci = c1; break;
    case 4: { C r; if (INV) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; } return r; }
    case 5: cr = -s1; ci = c1; break;
    case 6: cr = -h; ci = h; break;
    default: cr = -c1; ci = s1; break;
  }
  using S = decltype(a.x);
  S wr = (S)cr, wi = INV ? (S)ci : (S)(-ci);
  C r; r.x = a.x * wr - a.y * wi; r.y = a.x * wi + a.y * wr; return r;
}

template <int R, bool INV, typename C>
__device__ __forceinline__ void dft_reg(C* v) {
  constexpr int LG = Log2<R>::v;
  C a[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    int rev = 0;
#pragma unroll
    for (int b = 0; b < LG; ++b) rev |= ((i >> b) & 1) << (LG - 1 - b);
    a[rev] = v[i];
  }
#pragma unroll
  for (int len = 2; len <= R; len <<= 1) {
#pragma unroll
    for (int i = 0; i < R; i += len) {
#pragma unroll
      for (int j = 0; j < len / 2; ++j) {
        C u = a[i + j];
        C t = tw16<C, INV>(a[i + j + len / 2], j * (16 / len));
        a[i + j] = u + t;
        a[i + j + len / 2] = u - t;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < R; ++i) v[i] = a[i];
}

// one Stockham pass of radix R over nl lines of length L held in smem
template <int R, int E, bool INV, typename C>
__device__ __forceinline__ void stockham_pass(C* s, int LP, int logL, int nl, int p, const C* __restrict__ tab) {
  constexpr int NB = E / R;
  constexpr int LGR = Log2<R>::v;
  const int logLR = logL - LGR;
  const int LR = 1 << logLR;
  const int nbut = nl << logLR;
  const int nthr = blockDim.x, tid = threadIdx.x;
  C v[NB][R];
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    int b = q * nthr + tid;
    if (b < nbut) {
      int line = b >> logLR, i = b & (LR - 1);
#pragma unroll
      for (int r = 0; r < R; ++r) v[q][r] = s[sidx(line, LP, i + r * LR)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    int b = q * nthr + tid;
    if (b < nbut) {
      int line = b >> logLR, i = b & (LR - 1);
      int k = i & (p - 1);
      if (p > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = __ldg(&tab[p * R + r * k]);
          if (INV) w.y = -w.y;
          v[q][r] = v[q][r] * w;
        }
      }
      dft_reg<R, INV>(v[q]);
      int o = (i - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) s[sidx(line, LP, o + r * p)] = v[q][r];
    }
  }
  __syncthreads();
}

// full FFT of nl lines (length L = 2^logL) in smem, all threads of the CTA
template <int E, bool INV, typename C>
__device__ __forceinline__ void smem_fft(C* s, int LP, int logL, int nl, const C* __restrict__ tab) {
  constexpr int LOGE = Log2<E>::v;
  const int npass = (logL + LOGE - 1) / LOGE;
  const int base = logL / npass, extra = logL % npass;
  int p = 1;
  for (int ip = 0; ip < npass; ++ip) {
    int lr = base + (ip < extra ? 1 : 0);
    switch (lr) {
      case 1: stockham_pass<2, E, INV>(s, LP, logL, nl, p, tab); break;
      case 2: stockham_pass<4, E, INV>(s, LP, logL, nl, p, tab); break;
      case 3: stockham_pass<8, E, INV>(s, LP, logL, nl, p, tab); break;
      default:
        if constexpr (E >= 16) stockham_pass<16, E, INV>(s, LP, logL, nl, p, tab);
        break;
    }
    p <<= lr;
  }
}

template <typename T> struct FFTCfg;
template <> struct FFTCfg<float> { static constexpr int E = 16; static constexpr int CHUNK = 4096; };
template <> struct FFTCfg<double> { static constexpr int E = 8; static constexpr int CHUNK = 2048; };

// ---------------------------------------------------------------------------
// real-to-complex / complex-to-real pair processing (half-length trick)
//   forward:  X[k] = E + W^k O,  X[L-k] = conj(E - W^k O),
//             E = (Z[k] + conj Z[L-k])/2,  O = -i (Z[k] - conj Z[L-k])/2
//   inverse:  Z[k] = E + i O,  Z[L-k] = conj(E) + i conj(O),
//             E = X[k] + conj X[L-k],  O = (X[k] - conj X[L-k]) W^-k
//   with W = exp(-2 pi i / Nx) = tab[Nx + k].
// ---------------------------------------------------------------------------
template <typename C>
__device__ __forceinline__ void r2c_post(C Zk, C Zc_raw, C w, C& Xk, C& XLk) {
  using S = decltype(Zk.x);
  C Zc = conjg(Zc_raw);
  C Ev = (S)0.5 * (Zk + Zc);
  C D = Zk - Zc;                                  // O = -i D / 2
  C Ov; Ov.x = (S)0.5 * D.y; Ov.y = (S)(-0.5) * D.x;
  C WO = w * Ov;
  Xk = Ev + WO;
  XLk = conjg(Ev - WO);
}

template <typename C>
__device__ __forceinline__ void c2r_pre(C A, C Braw, C w, C& Zk, C& ZLk) {
  C B = conjg(Braw);
  C Ev = A + B;
  C wc = conjg(w);
  C Ov = (A - B) * wc;
  Zk = Ev + mul_i(Ov);
  ZLk = conjg(Ev) + mul_i(conjg(Ov));
}

// ---------------------------------------------------------------------------
// x pass, real -> half spectrum.  in = a0*in0 [+ a1*in1]  (rows of Nx reals)
// out rows have pitch kp (complex).  nrows = F*Nz*Ny.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_rows_r2c(const T* __restrict__ in0, const T* __restrict__ in1,
                                                  T a0, T a1, cplx<T>* __restrict__ out,
                                                  int logL, int nl, long long nrows, int kp,
                                                  const cplx<T>* __restrict__ tab) {
  using C = cplx<T>;
  constexpr int E = FFTCfg<T>::E;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  const int L = 1 << logL, LP = line_pitch(L);
  const long long row0 = (long long)blockIdx.x * nl;
  const int nthr = blockDim.x;
  const int total = nl * L;
  const C* zin0 = reinterpret_cast<const C*>(in0) + row0 * L;
  const C* zin1 = in1 ? reinterpret_cast<const C*>(in1) + row0 * L : nullptr;
  for (int f = threadIdx.x; f < total; f += nthr) {
    int line = f >> logL, e = f & (L - 1);
    if (row0 + line >= nrows) continue;
    C z = zin0[f];
    if (zin1) { C y = zin1[f]; z.x = a0 * z.x + a1 * y.x; z.y = a0 * z.y + a1 * y.y; }
    else if (a0 != (T)1) { z.x *= a0; z.y *= a0; }
    s[sidx(line, LP, e)] = z;
  }
  __syncthreads();
  smem_fft<E, false>(s, LP, logL, nl, tab);
  const int half = L / 2 + 1;
  for (int f = threadIdx.x; f < nl * half; f += nthr) {
    int line = f / half, k = f - line * half;
    long long row = row0 + line;
    if (row >= nrows) continue;
    C Zk = s[sidx(line, LP, k)];
    C Zc = s[sidx(line, LP, (L - k) & (L - 1))];
    C w = __ldg(&tab[2 * L + k]);
    C Xk, XLk;
    r2c_post(Zk, Zc, w, Xk, XLk);
    C* orow = out + row * kp;
    orow[k] = Xk;
    if (k != L - k) orow[L - k] = XLk;
  }
}

// ---------------------------------------------------------------------------
// x pass, half spectrum -> real, scaled.  in rows pitch kp.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_rows_c2r(const cplx<T>* __restrict__ in, T* __restrict__ out, T scale,
                                                  int logL, int nl, long long nrows, int kp,
                                                  const cplx<T>* __restrict__ tab) {
  using C = cplx<T>;
  constexpr int E = FFTCfg<T>::E;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  const int L = 1 << logL, LP = line_pitch(L);
  C* sN = s + nl * LP;                           // the kx = Nx/2 bin of each line
  const long long row0 = (long long)blockIdx.x * nl;
  const int nthr = blockDim.x;
  for (int f = threadIdx.x; f < nl * (L + 1); f += nthr) {
    int line = f / (L + 1), k = f - line * (L + 1);
    if (row0 + line >= nrows) continue;
    C x = in[(row0 + line) * kp + k];
    if (k == 0 || k == L) x.y = (T)0;           // c2r keeps Re of the DC and Nyquist bins
    if (k == L) sN[line] = x; else s[sidx(line, LP, k)] = x;
  }
  __syncthreads();
  const int half = L / 2 + 1;
  for (int f = threadIdx.x; f < nl * half; f += nthr) {
    int line = f / half, k = f - line * half;
    C A = s[sidx(line, LP, k)];
    C B = (k == 0) ? sN[line] : s[sidx(line, LP, L - k)];
    C w = __ldg(&tab[2 * L + k]);
    C Zk, ZLk;
    c2r_pre(A, B, w, Zk, ZLk);
    s[sidx(line, LP, k)] = Zk;
    if (k != 0 && k != L - k) s[sidx(line, LP, L - k)] = ZLk;
  }
  __syncthreads();
  smem_fft<E, true>(s, LP, logL, nl, tab);
  C* zo = reinterpret_cast<C*>(out) + row0 * L;
  for (int f = threadIdx.x; f < nl * L; f += nthr) {
    int line = f >> logL, e = f & (L - 1);
    if (row0 + line >= nrows) continue;
    C z = s[sidx(line, LP, e)];
    z.x *= scale; z.y *= scale;
    zo[f] = z;
  }
}

// ---------------------------------------------------------------------------
// x pass, full complex rows (length L = Nx).  in_real: input is a real field.
// ---------------------------------------------------------------------------
template <typename T, bool INV>
__global__ void __launch_bounds__(256) k_rows_c2c(const cplx<T>* __restrict__ in, const T* __restrict__ in_real,
                                                  cplx<T>* __restrict__ out, T scale, int logL, int nl,
                                                  long long nrows, const cplx<T>* __restrict__ tab) {
  using C = cplx<T>;
  constexpr int E = FFTCfg<T>::E;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  const int L = 1 << logL, LP = line_pitch(L);
  const long long row0 = (long long)blockIdx.x * nl;
  const int nthr = blockDim.x;
  for (int f = threadIdx.x; f < nl * L; f += nthr) {
    int line = f >> logL, e = f & (L - 1);
    if (row0 + line >= nrows) continue;
    C z;
    if (in_real) { z.x = in_real[row0 * L + f]; z.y = (T)0; } else z = in[row0 * L + f];
    s[sidx(line, LP, e)] = z;
  }
  __syncthreads();
  smem_fft<E, INV>(s, LP, logL, nl, tab);
  for (int f = threadIdx.x; f < nl * L; f += nthr) {
    int line = f >> logL, e = f & (L - 1);
    if (row0 + line >= nrows) continue;
    C z = s[sidx(line, LP, e)];
    if (scale != (T)1) { z.x *= scale; z.y *= scale; }
    out[row0 * L + f] = z;
  }
}

// ---------------------------------------------------------------------------
// y / z pass over strided columns.  Line (o, c): element e at
//   o*O + e*S + c,   c in [0, W),  valid iff (c % kpv) < nkv.
// Load:  v = (a0*in0 + a1*in1) * mult(k) * mscale  (multiplier only if mult != M_ONE)
// Store: out = v * oscale.  CTA = (tile of TW consecutive c, outer o).
// geo selects how (kx,ky,kz) are decoded for the multiplier:
//   0: 2D y pass (kx=c, ky=e)   1: 3D z pass (kx=c%kp, ky=c/kp, kz=e)
//   2: 3D y pass (kx=c, ky=e, kz=o%Nz)   3: 2D full-spectrum y pass (kx=c in [0,Nx))
// ---------------------------------------------------------------------------
struct ColArgs {
  int logL, S, W, TW, tiles;
  long long O;
  int kpv, nkv;      // validity: (c % kpv) < nkv
  int geo;
  int Nx, Ny, Nz, kp;
  double kxs, kys, kzs;
};

template <typename C>
__device__ __forceinline__ C col_mult(const ColArgs& a, int mult, double ms, int c, int e, long long o) {
  double kx, ky, kz = 0.0;
  switch (a.geo) {
    case 0: kx = c; ky = kfreq(e, a.Ny); break;
    case 1: kx = c % a.kp; ky = kfreq(c / a.kp, a.Ny); kz = kfreq(e, a.Nz); break;
    case 2: kx = c; ky = kfreq(e, a.Ny); kz = kfreq((int)(o % a.Nz), a.Nz); break;
    default: kx = (mult == M_DX0) ? kfreq(c, a.Nx) : (double)c; ky = kfreq(e, a.Ny); break;
  }
  if (mult == M_DXZ && (int)kx == a.Nx / 2) return mk<C>(0.0, 0.0);
  return mult_value<C>(mult, kx * a.kxs, ky * a.kys, kz * a.kzs, ms);
}

template <typename T, bool INV>
__global__ void __launch_bounds__(256) k_cols(const cplx<T>* __restrict__ in0, const cplx<T>* __restrict__ in1,
                                              T a0, T a1, int mult, double mscale,
                                              cplx<T>* __restrict__ out, T oscale, ColArgs a,
                                              const cplx<T>* __restrict__ tab) {
  using C = cplx<T>;
  constexpr int E = FFTCfg<T>::E;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  const int L = 1 << a.logL, LP = line_pitch(L);
  const int tile = blockIdx.x % a.tiles;
  const long long o = blockIdx.x / a.tiles;
  const int c0 = tile * a.TW;
  const long long base = o * a.O + c0;
  const int nthr = blockDim.x;
  const int total = a.TW * L;
  for (int f = threadIdx.x; f < total; f += nthr) {
    int cl = f % a.TW, e = f / a.TW;
    int c = c0 + cl;
    C v = mk<C>(0.0, 0.0);
    if (c < a.W && (c % a.kpv) < a.nkv) {
      long long idx = base + (long long)e * a.S + cl;
      v = in0[idx];
      if (in1) { C y = in1[idx]; v.x = a0 * v.x + a1 * y.x; v.y = a0 * v.y + a1 * y.y; }
      else if (a0 != (T)1) { v.x *= a0; v.y *= a0; }
      if (mult != M_ONE) v = v * col_mult<C>(a, mult, mscale, c, e, o);
    }
    s[sidx(cl, LP, e)] = v;
  }
  __syncthreads();
  smem_fft<E, INV>(s, LP, a.logL, a.TW, tab);
  for (int f = threadIdx.x; f < total; f += nthr) {
    int cl = f % a.TW, e = f / a.TW;
    int c = c0 + cl;
    if (c < a.W && (c % a.kpv) < a.nkv) {
      C v = s[sidx(cl, LP, e)];
      if (oscale != (T)1) { v.x *= oscale; v.y *= oscale; }
      out[base + (long long)e * a.S + cl] = v;
    }
  }
}

}  // namespace vsav
