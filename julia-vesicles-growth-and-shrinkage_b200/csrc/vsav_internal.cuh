// Internal types and helpers of the B200 SAV vesicle library (libvsav).
//
// Layout conventions (C order, x fastest; identical to the reference's
// column-major Julia arrays (Nx, Ny[, Nz], N)):
//   real field      [F][Nz][Ny][Nx]          (Nz = 1 in 2D)
//   half spectrum   [F][Nz][Ny][kp]  complex, kp = round_up(Nx/2+1, 16);
//                   columns kx >= Nx/2+1 are padding and stay zero
//   full spectrum   [F][Ny][Nx]      complex (reference-form psi solve)
// F counts "fields": V vesicle fields or R run fields (velocity/pressure).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>
#include <cstdio>
#include <cmath>
#include <string>
#include <stdexcept>
#include <atomic>

namespace vsav {

#define VSAV_CUDA(x)                                                              \
  do {                                                                            \
    cudaError_t e_ = (x);                                                         \
    if (e_ != cudaSuccess)                                                        \
      throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(e_) + \
                               " at " + __FILE__ + ":" + std::to_string(__LINE__)); \
  } while (0)

#define VSAV_LAUNCH_CHECK() VSAV_CUDA(cudaGetLastError())

// number of kernels this library has launched (all handles, all threads)
inline std::atomic<long long>& launch_counter() { static std::atomic<long long> c{0}; return c; }
#define VSAV_COUNT_LAUNCH() (::vsav::launch_counter().fetch_add(1, std::memory_order_relaxed))

template <typename T> struct CplxOf;
template <> struct CplxOf<float> { using type = float2; };
template <> struct CplxOf<double> { using type = double2; };
template <typename T> using cplx = typename CplxOf<T>::type;

template <typename C> __host__ __device__ __forceinline__ C mk(double re, double im) {
  C c; c.x = (decltype(c.x))re; c.y = (decltype(c.y))im; return c;
}
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator*(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ __forceinline__ float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator*(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ float2 conjg(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 conjg(double2 a) { return make_double2(a.x, -a.y); }
// i * a
template <typename C> __host__ __device__ __forceinline__ C mul_i(C a) { C r; r.x = -a.y; r.y = a.x; return r; }

// ---------------------------------------------------------------------------
// grid geometry shared by every kernel
// ---------------------------------------------------------------------------
struct Geom {
  int nd;            // 2 or 3
  int Nx, Ny, Nz;    // Nz = 1 in 2D
  int nkx, kp;       // Nx/2+1 and padded pitch
  long long P;       // real points per field   (Nz*Ny*Nx)
  long long H;       // complex slots per field (Nz*Ny*kp)
  long long Pfull;   // full complex per field  (Nz*Ny*Nx)
  double kxs, kys, kzs;  // 2*pi/L per axis
};

// wavenumbers of half-spectrum slot (kx index, ky index, kz index)
__device__ __forceinline__ double kfreq(int j, int n) { return (double)((j < n / 2) ? j : j - n); }   // fftfreq: Nyquist negative
// half spectrum: kx is rfftfreq (Nyquist positive)

enum Mult : int {
  M_ONE = 0,   // 1
  M_DX = 1,    // i kx   (rfftfreq, Nyquist +pi Nx/Lx; SpectralUtils.jl:42,46)
  M_DY = 2,    // i ky   (fftfreq)
  M_DZ = 3,    // i kz
  M_LAP = 4,   // -(kx^2+ky^2[+kz^2])
  M_BIH = 5,   // (kx^2+ky^2[+kz^2])^2
  M_DX0 = 6,   // i kx0  (fftfreq along x; full-spectrum D1_full, SpectralUtils.jl:43,47)
  M_DXZ = 7,   // i kx with the Nyquist column multiplier set to zero
};

// Multiplier value at wavenumber (kx,ky,kz) (already scaled).  Returns complex.
template <typename C>
__device__ __forceinline__ C mult_value(int m, double kx, double ky, double kz, double s) {
  switch (m) {
    case M_DX: case M_DY: case M_DZ: case M_DX0: case M_DXZ: {
      double k = (m == M_DY) ? ky : (m == M_DZ ? kz : kx);
      return mk<C>(0.0, s * k);
    }
    case M_LAP: return mk<C>(-s * (kx * kx + ky * ky + kz * kz), 0.0);
    case M_BIH: { double k2 = kx * kx + ky * ky + kz * kz; return mk<C>(s * k2 * k2, 0.0); }
    default: return mk<C>(s, 0.0);
  }
}
__device__ __forceinline__ bool mult_is_real(int m) { return m == M_ONE || m == M_LAP || m == M_BIH; }

// ---------------------------------------------------------------------------
// compensated (Neumaier / TwoSum) accumulation in double
// ---------------------------------------------------------------------------
struct KSum {
  double s, c;
  __device__ __forceinline__ void add(double x) {
    double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x; else c += (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ void merge(double s2, double c2) { add(s2); c += c2; }
  __device__ __forceinline__ double val() const { return s + c; }
};

// a plain FP64 running sum with KSum's interface (c stays 0)
struct PlainSum {
  double s, c;
  __device__ __forceinline__ void add(double x) { s += x; }
};

// Block-wide reduction of K compensated sums; thread 0 writes (s,c) pairs to
// out[k] (as double2).  smem must hold 2*K*nwarps doubles.
template <int K>
__device__ __forceinline__ void block_reduce_store(KSum (&acc)[K], double2* out, double* smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double s2 = __shfl_down_sync(0xffffffffu, acc[k].s, o);
      double c2 = __shfl_down_sync(0xffffffffu, acc[k].c, o);
      if (lane + o < 32) acc[k].merge(s2, c2);
    }
  }
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) { smem[(k * nw + warp) * 2] = acc[k].s; smem[(k * nw + warp) * 2 + 1] = acc[k].c; }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      KSum t{0.0, 0.0};
      for (int w = 0; w < nw; ++w) t.merge(smem[(k * nw + w) * 2], smem[(k * nw + w) * 2 + 1]);
      out[k] = make_double2(t.s, t.c);
    }
  }
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace vsav
