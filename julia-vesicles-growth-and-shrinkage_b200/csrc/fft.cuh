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
//  * inside the tile: thread t owns one radix-E butterfly (E elements spaced
//    L/E apart), so the first and the last radix-E passes run in registers
//    straight from / to global memory; the middle Stockham passes (radix <= 32)
//    go through two padded shared-memory buffers (ping-pong, one barrier each);
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

template <int R> struct Log2 { static constexpr int v = (R <= 1) ? 0 : 1 + Log2<R / 2>::v; };

// cos(2 pi m / 32), m = 0..8 (mathematical constants)
__host__ __device__ constexpr double cos32(int m) {
  return m == 0 ? 1.0 : m == 1 ? 0.98078528040323044913 : m == 2 ? 0.92387953251128675613 :
         m == 3 ? 0.83146961230254523708 : m == 4 ? 0.70710678118654752440 : m == 5 ? 0.55557023301960222474 :
         m == 6 ? 0.38268343236508977173 : m == 7 ? 0.19509032201612826785 : 0.0;
}
// multiply a by exp(-2 pi i m/32) (forward) or exp(+2 pi i m/32) (inverse), 0 <= m < 16
template <typename C, bool INV>
__device__ __forceinline__ C tw32(C a, int m) {
  if (m == 0) return a;
  if (m == 8) { C r; if (INV) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; } return r; }
  // cos and sin of 2 pi m / 32 from the first-octant table
  const double c = (m < 8) ? cos32(m) : -cos32(16 - m);
  const double sn = (m < 8) ? cos32(8 - m) : cos32(m - 8);
  using S = decltype(a.x);
  S wr = (S)c, wi = INV ? (S)sn : (S)(-sn);
  C r; r.x = a.x * wr - a.y * wi; r.y = a.x * wi + a.y * wr; return r;
}
template <typename C, bool INV>
__device__ __forceinline__ C tw16(C a, int m) { return tw32<C, INV>(a, 2 * m); }

// In-register DFT of size R (power of two <= 32): in-place radix-2
// decimation-in-frequency network (no temporaries), then the bit-reversal
// permutation as a register renaming (all indices compile-time constants).
__host__ __device__ constexpr int brev(int r, int lg) {
  int o = 0;
  for (int b = 0; b < lg; ++b) o |= ((r >> b) & 1) << (lg - 1 - b);
  return o;
}
template <int R, bool INV, typename C>
__device__ __forceinline__ void dft_reg(C* v) {
  constexpr int LG = Log2<R>::v;
#pragma unroll
  for (int len = R; len >= 2; len >>= 1) {
    const int h = len / 2;
#pragma unroll
    for (int i = 0; i < R; i += len) {
#pragma unroll
      for (int j = 0; j < h; ++j) {
        C u = v[i + j], w = v[i + j + h];
        v[i + j] = u + w;
        v[i + j + h] = tw32<C, INV>(u - w, j * (32 / len));
      }
    }
  }
  C t[R];
#pragma unroll
  for (int r = 0; r < R; ++r) t[r] = v[brev(r, LG)];
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = t[r];
}

// shared-memory layouts of a tile of nl lines of length L
//  RowLay: line-major, padded (x pass: lines are contiguous rows)
//  ColLay: element-major [e][nl] with the line index fastest -- the natural
//          layout of a tile of nl consecutive columns, conflict-free when
//          consecutive threads take consecutive lines
struct RowLay {
  int LP;
  __device__ __forceinline__ int operator()(int line, int e) const { return sidx(line, LP, e); }
  static constexpr bool line_fast = false;
};
struct ColLay {
  int nl, loge;    // nl lines; one nl-wide pad row every 2^loge elements (bank spreading)
  __device__ __forceinline__ int operator()(int line, int e) const { return (e + (e >> loge)) * nl + line; }
  static constexpr bool line_fast = true;
};
__host__ __device__ __forceinline__ int col_tile_elems(int L, int TW, int loge) { return (L + (L >> loge)) * TW; }

// one out-of-place Stockham pass of radix R: src -> dst (ping-pong buffers),
// one butterfly at a time (R complex registers + twiddles), one barrier
template <int R, int E, bool INV, typename C, typename Lay>
__device__ __forceinline__ void stockham_pass(const C* src, C* dst, const Lay lay, int logL, int lognl, int p,
                                              const C* __restrict__ tab) {
  constexpr int NB = E / R;
  constexpr int LGR = Log2<R>::v;
  const int logLR = logL - LGR;
  const int LR = 1 << logLR;
  const int nbut = 1 << (lognl + logLR);
  const int nthr = blockDim.x, tid = threadIdx.x;
#pragma unroll 1
  for (int q = 0; q < NB; ++q) {
    int b = q * nthr + tid;
    if (b < nbut) {
      int line, i;
      if (Lay::line_fast) { line = b & ((1 << lognl) - 1); i = b >> lognl; }
      else { line = b >> logLR; i = b & (LR - 1); }
      int k = i & (p - 1);
      C v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = src[lay(line, i + r * LR)];
      if (p > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = __ldg(&tab[p * R + r * k]);
          if (INV) w.y = -w.y;
          v[r] = v[r] * w;
        }
      }
      dft_reg<R, INV>(v);
      int o = (i - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) dst[lay(line, o + r * p)] = v[r];
    }
  }
  __syncthreads();
}

// Generic middle passes (ping-pong): Stockham passes of radix <= E from span p
// over `bits` bits, starting in buf[cur]; returns the buffer index holding the result.
template <int E, bool INV, typename C, typename Lay>
__device__ __forceinline__ int smem_passes(C* const (&buf)[2], int cur, const Lay lay, int logL, int lognl, int p, int bits,
                                           const C* __restrict__ tab) {
  constexpr int LOGE = Log2<E>::v < 5 ? Log2<E>::v : 5;
  if (bits <= 0) return cur;
  const int npass = (bits + LOGE - 1) / LOGE;
  const int base = bits / npass, extra = bits % npass;
  for (int ip = 0; ip < npass; ++ip) {
    int lr = base + (ip < extra ? 1 : 0);
    const C* src = buf[cur];
    C* dst = buf[cur ^ 1];
    switch (lr) {
      case 1: stockham_pass<2, E, INV>(src, dst, lay, logL, lognl, p, tab); break;
      case 2: if constexpr (E >= 4) stockham_pass<4, E, INV>(src, dst, lay, logL, lognl, p, tab); break;
      case 3: if constexpr (E >= 8) stockham_pass<8, E, INV>(src, dst, lay, logL, lognl, p, tab); break;
      case 4: if constexpr (E >= 16) stockham_pass<16, E, INV>(src, dst, lay, logL, lognl, p, tab); break;
      default:
        if constexpr (E >= 32) stockham_pass<32, E, INV>(src, dst, lay, logL, lognl, p, tab);
        break;
    }
    cur ^= 1;
    p <<= lr;
  }
  return cur;
}

// FFT of a tile of 2^lognl lines of length L = 2^logL in which thread t owns
// butterfly (line, i), i < L/E, i.e. the E elements i + j*(L/E) of `line`.
//  ENTRY_REG: the input is in v[] (else: already in buf[0], natural order);
//  EXIT_REG:  the output is returned in v[] (else: left in smem, natural order,
//             in the buffer whose index is returned).
// With L >= E^2 the first and the last radix-E passes run in registers and
// only the middle passes go through shared memory (ping-pong buffers).
template <int E, bool INV, bool ENTRY_REG, bool EXIT_REG, typename C, typename Lay>
__device__ __forceinline__ int tile_fft(C (&v)[E], C* const (&buf)[2], const Lay lay, int line, int i, bool active,
                                        int logL, int lognl, const C* __restrict__ tab) {
  constexpr int LOGE = Log2<E>::v;
  const int LE = 1 << (logL - LOGE);
  int cur = 0;
  if (logL >= 2 * LOGE) {
    int p = 1, bits = logL;
    if (ENTRY_REG) {
      if (active) {
        dft_reg<E, INV>(v);
#pragma unroll
        for (int r = 0; r < E; ++r) buf[0][lay(line, i * E + r)] = v[r];
      }
      __syncthreads();
      p = E; bits -= LOGE;
    }
    cur = smem_passes<E, INV>(buf, 0, lay, logL, lognl, p, bits - (EXIT_REG ? LOGE : 0), tab);
    if (EXIT_REG) {
      if (active) {
        const C* s = buf[cur];
#pragma unroll
        for (int r = 0; r < E; ++r) v[r] = s[lay(line, i + r * LE)];
        // last pass: radix E at span p = L/E, so k = i; twiddles exp(-+2 pi i r i / L)
        if constexpr (E >= 16) {
          // w^(r i) = w^(4 (r/4) i) * w^((r%4) i): 3 + E/4 - 1 table loads, 2-ulp products
          C lo[4], hi[E / 4];
#pragma unroll
          for (int q = 1; q < 4; ++q) { lo[q] = __ldg(&tab[(1 << logL) + q * i]); if (INV) lo[q].y = -lo[q].y; }
#pragma unroll
          for (int q = 1; q < E / 4; ++q) { hi[q] = __ldg(&tab[(1 << logL) + 4 * q * i]); if (INV) hi[q].y = -hi[q].y; }
#pragma unroll
          for (int r = 1; r < E; ++r) {
            C w = (r & 3) == 0 ? hi[r >> 2] : ((r >> 2) == 0 ? lo[r & 3] : hi[r >> 2] * lo[r & 3]);
            v[r] = v[r] * w;
          }
        } else {
#pragma unroll
          for (int r = 1; r < E; ++r) {
            C w = __ldg(&tab[(1 << logL) + r * i]);
            if (INV) w.y = -w.y;
            v[r] = v[r] * w;
          }
        }
        dft_reg<E, INV>(v);
      }
    }
  } else {
    if (ENTRY_REG) {
      if (active) {
#pragma unroll
        for (int j = 0; j < E; ++j) buf[0][lay(line, i + j * LE)] = v[j];
      }
      __syncthreads();
    }
    cur = smem_passes<E, INV>(buf, 0, lay, logL, lognl, 1, logL, tab);
    if (EXIT_REG && active) {
      const C* s = buf[cur];
#pragma unroll
      for (int r = 0; r < E; ++r) v[r] = s[lay(line, i + r * LE)];
    }
  }
  return cur;
}


// ---------------------------------------------------------------------------
// Single-buffer variants (half the shared memory of the ping-pong passes): a
// pass reads all of its butterflies into registers, waits for every thread,
// then writes.  Every thread holds E / R butterflies of every pass, so the
// block must cover the whole tile (blockDim.x * E = lines * L).  The butterflies, their twiddles and the radix split are those
// of stockham_pass / smem_passes / tile_fft, so the results are bit-identical.
// ---------------------------------------------------------------------------
template <int R, int E, bool INV, typename C, typename Lay>
__device__ __forceinline__ void stockham_pass_1buf(C* buf, const Lay lay, int logL, int lognl, int p,
                                                   const C* __restrict__ tab) {
  constexpr int NB = E / R;
  constexpr int LGR = Log2<R>::v;
  const int logLR = logL - LGR;
  const int LR = 1 << logLR;
  const int nthr = blockDim.x, tid = threadIdx.x;
  C v[NB][R];
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int b = q * nthr + tid;
    int line, i;
    if (Lay::line_fast) { line = b & ((1 << lognl) - 1); i = b >> lognl; }
    else { line = b >> logLR; i = b & (LR - 1); }
#pragma unroll
    for (int r = 0; r < R; ++r) v[q][r] = buf[lay(line, i + r * LR)];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int b = q * nthr + tid;
    int line, i;
    if (Lay::line_fast) { line = b & ((1 << lognl) - 1); i = b >> lognl; }
    else { line = b >> logLR; i = b & (LR - 1); }
    const int k = i & (p - 1);
    if (p > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = __ldg(&tab[p * R + r * k]);
        if (INV) w.y = -w.y;
        v[q][r] = v[q][r] * w;
      }
    }
    dft_reg<R, INV>(v[q]);
    const int o = (i - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) buf[lay(line, o + r * p)] = v[q][r];
  }
  __syncthreads();
}

template <int E, bool INV, typename C, typename Lay>
__device__ __forceinline__ void smem_passes_1buf(C* buf, const Lay lay, int logL, int lognl, int p, int bits,
                                                 const C* __restrict__ tab) {
  constexpr int LOGE = Log2<E>::v < 5 ? Log2<E>::v : 5;
  if (bits <= 0) return;
  const int npass = (bits + LOGE - 1) / LOGE;
  const int base = bits / npass, extra = bits % npass;
  for (int ip = 0; ip < npass; ++ip) {
    const int lr = base + (ip < extra ? 1 : 0);
    switch (lr) {
      case 1: stockham_pass_1buf<2, E, INV>(buf, lay, logL, lognl, p, tab); break;
      case 2: if constexpr (E >= 4) stockham_pass_1buf<4, E, INV>(buf, lay, logL, lognl, p, tab); break;
      case 3: if constexpr (E >= 8) stockham_pass_1buf<8, E, INV>(buf, lay, logL, lognl, p, tab); break;
      case 4: if constexpr (E >= 16) stockham_pass_1buf<16, E, INV>(buf, lay, logL, lognl, p, tab); break;
      default:
        if constexpr (E >= 32) stockham_pass_1buf<32, E, INV>(buf, lay, logL, lognl, p, tab);
        break;
    }
    p <<= lr;
  }
}

// tile_fft with the input in v[] and the output returned in v[] (ENTRY_REG and
// EXIT_REG), through one shared-memory buffer.  Needs L >= E^2 and every
// thread of the block holding one butterfly (a full tile).
template <int E, bool INV, typename C, typename Lay>
__device__ __forceinline__ void tile_fft_1buf(C (&v)[E], C* buf, const Lay lay, int line, int i, int logL, int lognl,
                                              const C* __restrict__ tab, const C* twx = nullptr) {
  constexpr int LOGE = Log2<E>::v;
  const int LE = 1 << (logL - LOGE);
  dft_reg<E, INV>(v);
#pragma unroll
  for (int r = 0; r < E; ++r) buf[lay(line, i * E + r)] = v[r];
  __syncthreads();
  smem_passes_1buf<E, INV>(buf, lay, logL, lognl, E, logL - 2 * LOGE, tab);
#pragma unroll
  for (int r = 0; r < E; ++r) v[r] = buf[lay(line, i + r * LE)];
  // twiddles of the last pass: exp(-+2 pi i m / L), from the table row of length L in
  // global memory, or from a per-butterfly table the caller staged in shared memory
  // (tw_last_table: twx[(q - 1) LE + i] = w^(q i), q = 1..3, then twx[(q + 2) LE + i] =
  // w^(4 q i), q = 1..E/4-1, so consecutive butterflies read consecutive words)
  const int LEv = 1 << (logL - LOGE);
  if constexpr (E >= 16) {
    C lo[4], hi[E / 4];
#pragma unroll
    for (int q = 1; q < 4; ++q) { lo[q] = twx ? twx[(q - 1) * LEv + i] : __ldg(&tab[(1 << logL) + q * i]); if (INV) lo[q].y = -lo[q].y; }
#pragma unroll
    for (int q = 1; q < E / 4; ++q) { hi[q] = twx ? twx[(q + 2) * LEv + i] : __ldg(&tab[(1 << logL) + 4 * q * i]); if (INV) hi[q].y = -hi[q].y; }
#pragma unroll
    for (int r = 1; r < E; ++r) {
      C w = (r & 3) == 0 ? hi[r >> 2] : ((r >> 2) == 0 ? lo[r & 3] : hi[r >> 2] * lo[r & 3]);
      v[r] = v[r] * w;
    }
  } else {
#pragma unroll
    for (int r = 1; r < E; ++r) {
      C w = twx ? twx[(r - 1) * LEv + i] : __ldg(&tab[(1 << logL) + r * i]);
      if (INV) w.y = -w.y;
      v[r] = v[r] * w;
    }
  }
  dft_reg<E, INV>(v);
}

// the per-butterfly twiddle table of tile_fft_1buf's last pass (twx), built by the
// block from the global table: entries of the row exp(-2 pi i m / L)
template <int E>
__host__ __device__ constexpr int tw_last_rows() { return E >= 16 ? 3 + E / 4 - 1 : E - 1; }
template <int E, typename C>
__device__ __forceinline__ void tw_last_table(C* twx, int logL, const C* __restrict__ tab) {
  constexpr int LOGE = Log2<E>::v, NR = tw_last_rows<E>();
  const int L = 1 << logL, LE = 1 << (logL - LOGE);
  for (int k = threadIdx.x; k < NR * LE; k += blockDim.x) {
    const int q = k / LE, i = k - q * LE;
    int m;
    if (E >= 16) m = (q < 3) ? (q + 1) * i : 4 * (q - 2) * i;
    else m = (q + 1) * i;
    twx[k] = tab[L + m];
  }
}

// row layout with one pad slot every 2^SH elements (SH = log2 of the register radix,
// so the stride-E writes after the first register pass spread over all banks) and an
// odd shift per line
template <int SH>
struct RowLayP {
  int LP;
  __device__ __forceinline__ int operator()(int line, int e) const { return line * LP + e + (e >> SH); }
  static constexpr bool line_fast = false;
  static __host__ __device__ constexpr int pitch(int L) { return L + (L >> SH) + 1; }
};

// minimum resident CTAs that the register budget must allow, per (E, NT)
template <int E, int NT> struct MinB {
  static constexpr int v = (NT >= 1024) ? 1 : (NT >= 512) ? ((E <= 8) ? 2 : 1) : ((E <= 4) ? 4 : ((E <= 8) ? 3 : 2));
};
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
// thread -> butterfly (line, i) of a row tile: line = tid / (L/E), i = tid % (L/E)
template <int E>
__device__ __forceinline__ void row_owner(int logL, int& line, int& i) {
  constexpr int LOGE = Log2<E>::v;
  const int logLE = logL - LOGE;
  line = threadIdx.x >> logLE;
  i = threadIdx.x & ((1 << logLE) - 1);
}

template <typename T, int E, int NT>
__global__ void __launch_bounds__(NT, MinB<E, NT>::v) k_rows_r2c(const T* __restrict__ in0, const T* __restrict__ in1,
                                                              T a0, T a1, cplx<T>* __restrict__ out,
                                                              int logL, int lognl, long long nrows, int kp,
                                                              const cplx<T>* __restrict__ tab) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  const int L = 1 << logL, LP = line_pitch(L), nl = 1 << lognl, LE = L / E;
  const long long row0 = (long long)blockIdx.x * nl;
  const long long rows_left = nrows - row0;
  int line, i;
  row_owner<E>(logL, line, i);
  const bool active = line < rows_left;
  C v[E];
  if (active) {
    const C* z0 = reinterpret_cast<const C*>(in0) + (row0 + line) * L + i;
    const C* z1 = in1 ? reinterpret_cast<const C*>(in1) + (row0 + line) * L + i : nullptr;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      C z = z0[j * LE];
      if (z1) { C y = z1[j * LE]; z.x = a0 * z.x + a1 * y.x; z.y = a0 * z.y + a1 * y.y; }
      else if (a0 != (T)1) { z.x *= a0; z.y *= a0; }
      v[j] = z;
    }
  }
  C* const buf[2] = {s, s + nl * LP};
  const C* so = buf[tile_fft<E, false, true, false>(v, buf, RowLay{LP}, line, i, active, logL, lognl, tab)];
  const int half = L / 2 + 1;
  for (int f = threadIdx.x; f < nl * half; f += blockDim.x) {
    int ln = f / half, k = f - ln * half;
    if (ln >= rows_left) continue;
    C Zk = so[sidx(ln, LP, k)];
    C Zc = so[sidx(ln, LP, (L - k) & (L - 1))];
    C w = __ldg(&tab[2 * L + k]);
    C Xk, XLk;
    r2c_post(Zk, Zc, w, Xk, XLk);
    C* orow = out + (row0 + ln) * kp;
    orow[k] = Xk;
    if (k != L - k) orow[L - k] = XLk;
  }
}

// load a half-spectrum row block [nl][L+1] (pitch kp) into smem, keeping only
// Re of the kx=0 and kx=Nx/2 bins, and apply the c2r pre-processing in place
template <typename T, int E>
__device__ __forceinline__ void load_c2r_tile(const cplx<T>* __restrict__ in, cplx<T>* s, cplx<T>* sN, long long row0,
                                              long long rows_left, int logL, int lognl, int kp,
                                              const cplx<T>* __restrict__ tab) {
  using C = cplx<T>;
  const int L = 1 << logL, LP = line_pitch(L), nl = 1 << lognl, LE = L / E;
  int line, i;
  row_owner<E>(logL, line, i);
  if (line < rows_left) {
    C xl[E];
    const C* src = in + (row0 + line) * kp + i;
#pragma unroll
    for (int j = 0; j < E; ++j) xl[j] = src[j * LE];
    if (i == 0) xl[0].y = (T)0;                  // c2r keeps Re of the DC and Nyquist bins
#pragma unroll
    for (int j = 0; j < E; ++j) s[sidx(line, LP, i + j * LE)] = xl[j];
  }
  for (int ln = threadIdx.x; ln < nl; ln += blockDim.x)
    if (ln < rows_left) { C x = in[(row0 + ln) * kp + L]; x.y = (T)0; sN[ln] = x; }
  __syncthreads();
  const int half = L / 2 + 1;
  for (int f = threadIdx.x; f < nl * half; f += blockDim.x) {
    int ln = f / half, k = f - ln * half;
    C A = s[sidx(ln, LP, k)];
    C B = (k == 0) ? sN[ln] : s[sidx(ln, LP, L - k)];
    C w = __ldg(&tab[2 * L + k]);
    C Zk, ZLk;
    c2r_pre(A, B, w, Zk, ZLk);
    s[sidx(ln, LP, k)] = Zk;
    if (k != 0 && k != L - k) s[sidx(ln, LP, L - k)] = ZLk;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// x pass, half spectrum -> real, scaled.  in rows pitch kp.
// ---------------------------------------------------------------------------
template <typename T, int E, int NT>
__global__ void __launch_bounds__(NT, MinB<E, NT>::v) k_rows_c2r(const cplx<T>* __restrict__ in, T* __restrict__ out, T scale,
                                                              int logL, int lognl, long long nrows, int kp,
                                                              const cplx<T>* __restrict__ tab) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  const int L = 1 << logL, LP = line_pitch(L), nl = 1 << lognl, LE = L / E;
  C* sN = s + 2 * nl * LP;
  const long long row0 = (long long)blockIdx.x * nl;
  const long long rows_left = nrows - row0;
  load_c2r_tile<T, E>(in, s, sN, row0, rows_left, logL, lognl, kp, tab);
  int line, i;
  row_owner<E>(logL, line, i);
  const bool active = line < rows_left;
  C v[E];
  C* const buf[2] = {s, s + nl * LP};
  tile_fft<E, true, false, true>(v, buf, RowLay{LP}, line, i, active, logL, lognl, tab);
  if (active) {
    C* zo = reinterpret_cast<C*>(out) + (row0 + line) * L + i;
#pragma unroll
    for (int j = 0; j < E; ++j) { C z = v[j]; z.x *= scale; z.y *= scale; zo[j * LE] = z; }
  }
}

// ---------------------------------------------------------------------------
// x pass, full complex rows (length L = Nx).  in_real: input is a real field.
// ---------------------------------------------------------------------------
template <typename T, int E, int NT, bool INV>
__global__ void __launch_bounds__(NT, MinB<E, NT>::v) k_rows_c2c(const cplx<T>* __restrict__ in, const T* __restrict__ in_real,
                                                              cplx<T>* __restrict__ out, T scale, int logL, int lognl,
                                                              long long nrows, const cplx<T>* __restrict__ tab) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  const int L = 1 << logL, LP = line_pitch(L), nl = 1 << lognl, LE = L / E;
  const long long row0 = (long long)blockIdx.x * nl;
  const long long rows_left = nrows - row0;
  int line, i;
  row_owner<E>(logL, line, i);
  const bool active = line < rows_left;
  C v[E];
  const long long off = (row0 + line) * L + i;
  if (active) {
#pragma unroll
    for (int j = 0; j < E; ++j) {
      if (in_real) { v[j].x = in_real[off + j * LE]; v[j].y = (T)0; } else v[j] = in[off + j * LE];
    }
  }
  C* const buf[2] = {s, s + nl * LP};
  tile_fft<E, INV, true, true>(v, buf, RowLay{LP}, line, i, active, logL, lognl, tab);
  if (active) {
#pragma unroll
    for (int j = 0; j < E; ++j) {
      C z = v[j];
      if (scale != (T)1) { z.x *= scale; z.y *= scale; }
      out[off + j * LE] = z;
    }
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
//   4: 3D full-spectrum z pass (kx=c%Nx, ky=c/Nx, kz=e)   5: 3D full-spectrum y pass (kx=c, ky=e, kz=o%Nz)
// ---------------------------------------------------------------------------
struct ColArgs {
  int logL, S, W, TW, logTW, tiles;
  long long O;
  int kpv, nkv;      // validity: (c % kpv) < nkv
  int geo;
  int Nx, Ny, Nz, kp;
  double kxs, kys, kzs;
  float fkxs, fkys, fkzs;   // the same in FP32 (col_mult_f)
};

template <typename C>
__device__ __forceinline__ C col_mult(const ColArgs& a, int mult, double ms, int c, int e, long long o) {
  double kx, ky, kz = 0.0;
  switch (a.geo) {
    case 0: kx = c; ky = kfreq(e, a.Ny); break;
    case 1: kx = c % a.kp; ky = kfreq(c / a.kp, a.Ny); kz = kfreq(e, a.Nz); break;
    case 2: kx = c; ky = kfreq(e, a.Ny); kz = kfreq((int)(o % a.Nz), a.Nz); break;
    case 4: {
      const int cx = c & (a.Nx - 1);
      kx = (mult == M_DX0) ? kfreq(cx, a.Nx) : (double)cx; ky = kfreq(c / a.Nx, a.Ny); kz = kfreq(e, a.Nz);
      break;
    }
    case 5: kx = (mult == M_DX0) ? kfreq(c, a.Nx) : (double)c; ky = kfreq(e, a.Ny); kz = kfreq((int)(o % a.Nz), a.Nz); break;
    default: kx = (mult == M_DX0) ? kfreq(c, a.Nx) : (double)c; ky = kfreq(e, a.Ny); break;
  }
  if (mult == M_DXZ && (int)kx == a.Nx / 2) return mk<C>(0.0, 0.0);
  return mult_value<C>(mult, kx * a.kxs, ky * a.kys, kz * a.kzs, ms);
}

// col_mult in FP32 arithmetic (the FP32 kernels): the same wavenumber decoding,
// no FP64 conversions or products per element
__device__ __forceinline__ int kfreq_i(int j, int n) { return (j < n / 2) ? j : j - n; }
__device__ __forceinline__ cplx<float> col_mult_f(const ColArgs& a, int mult, float ms, int c, int e, long long o) {
  int kx, ky, kz = 0;
  switch (a.geo) {
    case 0: kx = c; ky = kfreq_i(e, a.Ny); break;
    case 1: kx = c % a.kp; ky = kfreq_i(c / a.kp, a.Ny); kz = kfreq_i(e, a.Nz); break;
    case 2: kx = c; ky = kfreq_i(e, a.Ny); kz = kfreq_i((int)(o % a.Nz), a.Nz); break;
    case 4: { const int cx = c & (a.Nx - 1); kx = (mult == M_DX0) ? kfreq_i(cx, a.Nx) : cx; ky = kfreq_i(c / a.Nx, a.Ny); kz = kfreq_i(e, a.Nz); break; }
    case 5: kx = (mult == M_DX0) ? kfreq_i(c, a.Nx) : c; ky = kfreq_i(e, a.Ny); kz = kfreq_i((int)(o % a.Nz), a.Nz); break;
    default: kx = (mult == M_DX0) ? kfreq_i(c, a.Nx) : c; ky = kfreq_i(e, a.Ny); break;
  }
  if (mult == M_DXZ && kx == a.Nx / 2) return mk<cplx<float>>(0.0, 0.0);
  const float fx = (float)kx * a.fkxs, fy = (float)ky * a.fkys, fz = (float)kz * a.fkzs;
  switch (mult) {
    case M_DX: case M_DX0: case M_DXZ: return cplx<float>{0.f, ms * fx};
    case M_DY: return cplx<float>{0.f, ms * fy};
    case M_DZ: return cplx<float>{0.f, ms * fz};
    case M_LAP: return cplx<float>{-ms * (fx * fx + fy * fy + fz * fz), 0.f};
    case M_BIH: { const float k2 = fx * fx + fy * fy + fz * fz; return cplx<float>{ms * k2 * k2, 0.f}; }
    default: return cplx<float>{ms, 0.f};
  }
}

template <typename T, int E, int NT, bool INV>
__global__ void __launch_bounds__(NT, MinB<E, NT>::v) k_cols(const cplx<T>* __restrict__ in0, const cplx<T>* __restrict__ in1,
                                                          T a0, T a1, int mult, double mscale,
                                                          cplx<T>* __restrict__ out, T oscale, ColArgs a,
                                                          const cplx<T>* __restrict__ tab) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  const int L = 1 << a.logL, LE = L / E;
  const int tile = blockIdx.x % a.tiles;
  const long long o = blockIdx.x / a.tiles;
  const int c0 = tile * a.TW;
  const long long base = o * a.O + c0;
  // thread -> column cl of the tile and butterfly i (elements i + j*L/E);
  // the tile sits in smem in its global layout [e][TW]
  const int cl = threadIdx.x & (a.TW - 1);
  const int i = threadIdx.x >> a.logTW;
  const int c = c0 + cl;
  const bool valid = c < a.W && (c % a.kpv) < a.nkv;
  const ColLay lay{a.TW, Log2<E>::v};
  C v[E];
  if (valid) {
#pragma unroll
    for (int j = 0; j < E; ++j) {
      long long idx = base + (long long)(i + j * LE) * a.S + cl;
      v[j] = in0[idx];
      if (in1) { C y = in1[idx]; v[j].x = a0 * v[j].x + a1 * y.x; v[j].y = a0 * v[j].y + a1 * y.y; }
    }
#pragma unroll
    for (int j = 0; j < E; ++j) {
      if (!in1 && a0 != (T)1) { v[j].x *= a0; v[j].y *= a0; }
      if (mult != M_ONE) {
        if constexpr (std::is_same<T, float>::value) v[j] = v[j] * col_mult_f(a, mult, (float)mscale, c, i + j * LE, o);
        else v[j] = v[j] * col_mult<C>(a, mult, mscale, c, i + j * LE, o);
      }
    }
  } else {
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = mk<C>(0.0, 0.0);
  }
  C* const buf[2] = {s, s + col_tile_elems(L, a.TW, Log2<E>::v)};
  tile_fft<E, INV, true, true>(v, buf, lay, cl, i, true, a.logL, a.logTW, tab);
  if (valid) {
#pragma unroll
    for (int j = 0; j < E; ++j) {
      C z = v[j];
      if (oscale != (T)1) { z.x *= oscale; z.y *= oscale; }
      out[base + (long long)(i + j * LE) * a.S + cl] = z;
    }
  }
}

}  // namespace vsav
