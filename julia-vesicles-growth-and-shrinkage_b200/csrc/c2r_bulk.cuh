// x pass of the half-spectrum -> real field transforms (k_rows_c2r) as a persistent
// kernel fed by bulk copies, in FP64 or FP32.
//
// k_rows_c2r loads a block of NL rows with plain loads, applies the c2r
// pre-processing in shared memory, transforms and stores, one row block per CTA,
// so a block's loads are not overlapped with its own work.  Here one block per SM
// slot walks the row blocks blockIdx.x, +gridDim.x, ...: the NL input rows of a
// block are one contiguous run of NL kp complex values, which one thread copies
// into a shared-memory slot with cp.async.bulk, completed on an mbarrier (bounded
// wait).  The block reads the landed rows, applies the pre-processing (Re of the
// DC and Nyquist bins, the half-length pair step c2r_pre) into the padded FFT
// buffer, hands the slot back to the copy engine for the next row block and
// transforms while that copy is in flight.  The pre-processing, butterflies and
// twiddles are those of k_rows_c2r with the same E, so the output is
// bit-identical to k_rows_c2r<T, E, NT>.
//
// Shared memory (dynamic, 1024-byte aligned):
//   slot   NL kp complex T (the landed input rows, unpadded)
//   buf    2 NL line_pitch(L) complex T (the FFT ping-pong buffers)
//   1 mbarrier (64 bytes reserved)
#pragma once
#include "psi.cuh"

namespace vsav {

template <typename T, int E, int NT, int LOGL>
__host__ __device__ inline size_t c2r_bulk_smem(int kp) {
  constexpr int L = 1 << LOGL, NL = E * NT / L;
  return 1024 + ((size_t)NL * kp * sizeof(cplx<T>) + 15) / 16 * 16 + 2 * (size_t)NL * line_pitch(L) * sizeof(cplx<T>) + 64;
}

template <typename T, int E, int NT, int LOGL>
__global__ void __launch_bounds__(NT, 2) k_rows_c2r_bulk(const cplx<T>* __restrict__ in, T* __restrict__ out, T scale,
                                                         long long nblocks, int kp, const cplx<T>* __restrict__ tab,
                                                         int* __restrict__ err) {
  using C = cplx<T>;
  constexpr int L = 1 << LOGL, NL = E * NT / L, LE = L / E, LOGNL = Log2<NL>::v, HALF = L / 2 + 1;
  static_assert(NL >= 1 && (NL & (NL - 1)) == 0 && L >= E * E, "tile geometry");
  const int LP = line_pitch(L);
  unsigned char* base = tma_smem_base();
  C* slot = reinterpret_cast<C*>(base);
  const size_t slot_bytes = ((size_t)NL * kp * sizeof(C) + 15) / 16 * 16;
  C* b0 = reinterpret_cast<C*>(base + slot_bytes);
  C* const buf[2] = {b0, b0 + (size_t)NL * LP};
  uint64_t* bar = reinterpret_cast<uint64_t*>(b0 + 2 * (size_t)NL * LP);
  const uint32_t bytes = (uint32_t)((size_t)NL * kp * sizeof(C));
  const int tid = threadIdx.x;
  auto issue = [&](long long t) {
    mbar_arrive_expect_tx(bar, bytes);
    bulk_load(slot, in + t * NL * kp, bytes, bar);
  };
  if (tid == 0) { mbar_init(bar, 1); mbar_fence_init(); }
  __syncthreads();
  long long t = blockIdx.x;
  if (tid == 0 && t < nblocks) issue(t);
  int line, i;
  row_owner<E>(LOGL, line, i);
  uint32_t ph = 0;
  while (t < nblocks) {
    const bool ok = mbar_wait(bar, ph, err);
    if (__syncthreads_or(!ok)) return;
    // c2r pre-processing (load_c2r_tile's arithmetic): pairs (k, L - k) of each row
    for (int f = tid; f < NL * HALF; f += NT) {
      const int ln = f / HALF, k = f - ln * HALF;
      const C* row = slot + (size_t)ln * kp;
      C A = row[k];
      if (k == 0) A.y = (T)0;                           // c2r keeps Re of the DC and Nyquist bins
      C B;
      if (k == 0) { B = row[L]; B.y = (T)0; }
      else B = row[L - k];
      const C w = __ldg(&tab[2 * L + k]);
      C Zk, ZLk;
      c2r_pre(A, B, w, Zk, ZLk);
      buf[0][sidx(ln, LP, k)] = Zk;
      if (k != 0 && k != L - k) buf[0][sidx(ln, LP, L - k)] = ZLk;
    }
    __syncthreads();                                          // slot consumed, buffer filled
    const long long tn = t + gridDim.x;
    if (tid == 0 && tn < nblocks) { fence_proxy_async(); issue(tn); }
    C v[E];
    tile_fft<E, true, false, true>(v, buf, RowLay{LP}, line, i, true, LOGL, LOGNL, tab);
    C* zo = reinterpret_cast<C*>(out) + (t * NL + line) * L + i;
#pragma unroll
    for (int j = 0; j < E; ++j) { C z = v[j]; z.x *= scale; z.y *= scale; zo[j * LE] = z; }
    __syncthreads();                                          // buffers free for the next row block
    ph ^= 1;
    t = tn;
  }
}

}  // namespace vsav
