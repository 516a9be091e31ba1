// y pass of the 2D half-spectrum field transforms (the column pass of k_cols with
// geo 0) as a persistent kernel fed by TMA tile copies, in FP64 or FP32.
//
// k_cols loads a tile of TW columns x L rows with plain strided loads, transforms
// it and stores it, one tile per block: the loads of a block are not overlapped
// with its own transform.  Here one block per SM slot walks the tiles
// blockIdx.x, +gridDim.x, ...; one thread copies a tile's input columns (one or
// two fields) into a shared-memory staging area with 2D bulk tensor copies (boxes
// of TW columns x min(L, 256) rows, tensor maps over this GPU's own buffers, no
// cluster multicast) completed on an mbarrier, and the copies of tile k+1 are in
// flight while tile k is transformed.  The load-side work (a0 in0 + a1 in1, the
// derivative / Laplacian / biharmonic multiplier, the scale) and the butterflies,
// twiddles and radix split are those of k_cols with the same E, through the
// single-buffer form of the Stockham passes, so the output is bit-identical to
// k_cols<T, E, NT, INV> for geo 0.  Columns outside the valid range (the padding
// of the half spectrum) are neither transformed nor written, as in k_cols; tiles
// that hold only padding columns are skipped.
//
// Shared memory (dynamic, 1024-byte aligned):
//   staging  NIN arrays [L][TW] of complex T (TMA box layout)
//   work     col_tile_elems(L, TW, log2 E) complex T (the FFT buffer)
//   1 mbarrier (64 bytes reserved)
//   twx      the last pass's per-butterfly twiddles (tw_last_table)
// Waits on the mbarrier are bounded (tma.cuh): a copy that never lands sets the
// error word and every thread of the block returns.
#pragma once
#include "psi.cuh"

namespace vsav {

struct ColsTmaTiles {
  int per_field;    // column tiles per field that hold a valid column: ceil(nkv / TW)
  int total;        // per_field * fields
};

template <int E>
__host__ __device__ constexpr int cols_tma_twx_rows() { return E >= 16 ? 3 + E / 4 - 1 : E - 1; }

template <typename T, int E, int NT, int LOGL, int NIN>
__host__ __device__ constexpr size_t cols_tma_smem() {
  constexpr int L = 1 << LOGL, TW = E * NT / L;
  return 1024 + (size_t)NIN * L * TW * sizeof(cplx<T>) + (size_t)(L + (L >> Log2<E>::v)) * TW * sizeof(cplx<T>) + 64 +
         (size_t)cols_tma_twx_rows<E>() * (L / E) * sizeof(cplx<T>);
}

// register budget: three 128-thread or two 256-thread blocks per SM
template <int NT>
struct ColsTmaMinB { static constexpr int v = NT <= 128 ? 3 : 2; };

template <typename T, int E, int NT, int LOGL, bool INV, int NIN>
__global__ void __launch_bounds__(NT, ColsTmaMinB<NT>::v) k_cols_tma(const __grid_constant__ CUtensorMap m0, const __grid_constant__ CUtensorMap m1,
                                                    T a0, T a1, int mult, double mscale, cplx<T>* __restrict__ out,
                                                    T oscale, ColArgs a, ColsTmaTiles tt,
                                                    const cplx<T>* __restrict__ tab, int* __restrict__ err) {
  using C = cplx<T>;
  constexpr int L = 1 << LOGL, LE = L / E, TW = E * NT / L, LOGTW = Log2<TW>::v, LOGE = Log2<E>::v;
  static_assert(TW >= 2 && TW <= 16 && L >= E * E, "tile geometry");
  constexpr int BH = L < 256 ? L : 256, NBOX = L / BH;     // rows per TMA box, boxes per column tile
  constexpr int XU = (int)(sizeof(C) / 8);                 // 8-byte units of the tensor map per element
  unsigned char* base = tma_smem_base();
  C* s0 = reinterpret_cast<C*>(base);
  C* s1 = s0 + (size_t)L * TW;
  C* work = s0 + (size_t)NIN * L * TW;
  uint64_t* bar = reinterpret_cast<uint64_t*>(work + (L + (L >> LOGE)) * TW);
  C* twx = reinterpret_cast<C*>(reinterpret_cast<unsigned char*>(bar) + 64);
  const int tid = threadIdx.x;
  const int cl = tid & (TW - 1), i = tid >> LOGTW;
  const uint32_t tx = (uint32_t)((size_t)NIN * L * TW * sizeof(C));
  auto issue = [&](int t) {
    const int o = t / tt.per_field, c0 = (t % tt.per_field) * TW;
    mbar_arrive_expect_tx(bar, tx);
    for (int q = 0; q < NBOX; ++q) {
      tma_load_2d(s0 + (size_t)q * BH * TW, &m0, c0 * XU, o * L + q * BH, bar);
      if constexpr (NIN == 2) tma_load_2d(s1 + (size_t)q * BH * TW, &m1, c0 * XU, o * L + q * BH, bar);
    }
  };
  if (tid == 0) { mbar_init(bar, 1); mbar_fence_init(); }
  tw_last_table<E>(twx, LOGL, tab);
  __syncthreads();
  int t = blockIdx.x;
  if (tid == 0 && t < tt.total) issue(t);
  const ColLay lay{TW, LOGE};
  uint32_t ph = 0;
  while (t < tt.total) {
    const int o = t / tt.per_field, c0 = (t % tt.per_field) * TW, c = c0 + cl;
    const bool valid = c < a.W && (c % a.kpv) < a.nkv;
    const bool ok = mbar_wait(bar, ph, err);
    if (__syncthreads_or(!ok)) return;
    C v[E];
    if (valid) {
#pragma unroll
      for (int j = 0; j < E; ++j) {
        v[j] = s0[(i + j * LE) * TW + cl];
        if constexpr (NIN == 2) {
          const C y = s1[(i + j * LE) * TW + cl];
          v[j].x = a0 * v[j].x + a1 * y.x; v[j].y = a0 * v[j].y + a1 * y.y;
        }
      }
#pragma unroll
      for (int j = 0; j < E; ++j) {
        if (NIN == 1 && a0 != (T)1) { v[j].x *= a0; v[j].y *= a0; }
        if (mult != M_ONE) {
          if constexpr (std::is_same<T, float>::value) v[j] = v[j] * col_mult_f(a, mult, (float)mscale, c, i + j * LE, o);
          else v[j] = v[j] * col_mult<C>(a, mult, mscale, c, i + j * LE, o);
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < E; ++j) v[j] = mk<C>(0.0, 0.0);
    }
    __syncthreads();                                          // staging consumed by every thread
    const int tn = t + gridDim.x;
    if (tid == 0 && tn < tt.total) { fence_proxy_async(); issue(tn); }
    tile_fft_1buf<E, INV>(v, work, lay, cl, i, LOGL, LOGTW, tab, twx);
    if (valid) {
      C* op = out + (long long)o * a.O + c;
#pragma unroll
      for (int j = 0; j < E; ++j) {
        C z = v[j];
        if (oscale != (T)1) { z.x *= oscale; z.y *= oscale; }
        op[(long long)(i + j * LE) * a.S] = z;
      }
    }
    __syncthreads();                                          // work buffer free for the next tile
    ph ^= 1;
    t = tn;
  }
}

}  // namespace vsav
