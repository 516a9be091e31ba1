// Inference of the learned psi-preconditioner network on periodic 2D fields,
// all five layers fused in one kernel on the tensor cores (mma.sync
// m16n8k16, BF16 operands, FP32 accumulation).
//
// A CTA owns a 32x32 output tile of one field and keeps every intermediate
// activation in shared memory: the 42x42 input tile (2 channels, periodic
// halo of 5), then layer outputs 40x40, 38x38, 36x36, 34x34 (16 channels,
// BF16, pixel-major, 32 B per pixel, two 16 B channel halves swapped on every
// other group of four pixels so ldmatrix rows of consecutive pixels hit
// distinct banks) and finally the 32x32 output written to global memory.
// Each layer is an implicit GEMM: rows = output pixels (16 per mma), K =
// 16 input channels of one 3x3 tap (9 taps accumulate), N = 16 output
// channels (two n8 tiles).  ldmatrix takes per-lane row addresses, so the
// shifted pixel rows of every tap are read straight from the activation
// buffer without an im2col copy.  Layer 0 (2 input channels) packs K = tap*2
// + channel (taps 0..8 in two k-steps); layer 4 (one output channel) uses one
// n8 tile of which column 0 is live.
//
// The B operands (weights) are pre-packed per lane in mma fragment order by
// net_pack() and read from global memory (L1/L2 resident, 17 KB) into
// registers at the start of each layer.
#pragma once
#include "net_common.cuh"

namespace vsav {

// fragment table layout (uint32 words), see net_pack()
constexpr int NF_L0 = 0;                          // [ks 2][nt 2][lane 32][2]
constexpr int NF_LH = NF_L0 + 2 * 2 * 32 * 2;     // 3 x [tap 9][nt 2][lane 32][2]
constexpr int NF_LH_SIZE = 9 * 2 * 32 * 2;
constexpr int NF_L4 = NF_LH + 3 * NF_LH_SIZE;     // [tap 9][lane 32][2]
constexpr int NF_WORDS = NF_L4 + 9 * 32 * 2;
constexpr int NF_BIAS = 16 * 4 + 1;               // biases of layers 0..4 (FP32)

inline uint32_t bf16_bits_host(float x) {          // x already BF16-representable
  uint32_t u;
  std::memcpy(&u, &x, 4);
  return u >> 16;
}
inline uint32_t pack2(float lo, float hi) { return bf16_bits_host(lo) | (bf16_bits_host(hi) << 16); }

// wb: BF16-rounded weights + biases in the theta layout (host).
inline void net_pack(const float* wb, uint32_t* fr, float* bias) {
  auto W = [&](int l, int o, int i, int tap) { return wb[net_woff(l) + (o * net_cin(l) + i) * 9 + tap]; };
  for (int ks = 0; ks < 2; ++ks)
    for (int nt = 0; nt < 2; ++nt)
      for (int lane = 0; lane < 32; ++lane) {
        const int g = lane >> 2, t = lane & 3, n = 8 * nt + g;
        const int tap0 = ks * 8 + t, tap1 = ks * 8 + t + 4;
        uint32_t* o = fr + NF_L0 + ((ks * 2 + nt) * 32 + lane) * 2;
        o[0] = tap0 < 9 ? pack2(W(0, n, 0, tap0), W(0, n, 1, tap0)) : 0u;
        o[1] = tap1 < 9 ? pack2(W(0, n, 0, tap1), W(0, n, 1, tap1)) : 0u;
      }
  for (int l = 1; l <= 3; ++l)
    for (int tap = 0; tap < 9; ++tap)
      for (int nt = 0; nt < 2; ++nt)
        for (int lane = 0; lane < 32; ++lane) {
          const int g = lane >> 2, t = lane & 3, n = 8 * nt + g;
          uint32_t* o = fr + NF_LH + (l - 1) * NF_LH_SIZE + ((tap * 2 + nt) * 32 + lane) * 2;
          o[0] = pack2(W(l, n, 2 * t, tap), W(l, n, 2 * t + 1, tap));
          o[1] = pack2(W(l, n, 2 * t + 8, tap), W(l, n, 2 * t + 9, tap));
        }
  for (int tap = 0; tap < 9; ++tap)
    for (int lane = 0; lane < 32; ++lane) {
      const int g = lane >> 2, t = lane & 3;
      uint32_t* o = fr + NF_L4 + (tap * 32 + lane) * 2;
      o[0] = g == 0 ? pack2(W(4, 0, 2 * t, tap), W(4, 0, 2 * t + 1, tap)) : 0u;
      o[1] = g == 0 ? pack2(W(4, 0, 2 * t + 8, tap), W(4, 0, 2 * t + 9, tap)) : 0u;
    }
  for (int l = 0; l < NET_NL; ++l)
    for (int o = 0; o < net_cout(l); ++o) bias[16 * l + o] = wb[net_woff(l) + net_wsize(l) + o];
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(addr));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);   // .x = lo (low half)
  return *reinterpret_cast<uint32_t*>(&v);
}
// byte offset of channel half h of pixel p in a 16-channel activation buffer
__device__ __forceinline__ uint32_t act_off(int p, int h) { return (uint32_t)p * 32u + ((uint32_t)(h ^ ((p >> 2) & 1)) << 4); }

constexpr int NA_T = 32;                 // output tile
constexpr int NA_IN = NA_T + 10;         // input tile with halo
constexpr int NA_THREADS = 256;
constexpr int NA_SMEM = NA_IN * NA_IN * 4 + (NA_T + 8) * (NA_T + 8) * 32 + (NA_T + 6) * (NA_T + 6) * 32;

// one 16 -> 16 layer: in (width Win = Wout + 2) -> out (Wout x Wout)
__device__ __forceinline__ void na_hidden(uint32_t s_in, unsigned char* out, int Wout, const uint32_t* __restrict__ fr,
                                          const float* __restrict__ bias) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = NA_THREADS / 32;
  const int Win = Wout + 2, P = Wout * Wout, nmt = (P + 15) >> 4;
  uint32_t bf[9][2][2];
#pragma unroll
  for (int tap = 0; tap < 9; ++tap)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
      uint2 v = __ldg(reinterpret_cast<const uint2*>(fr) + (tap * 2 + nt) * 32 + lane);
      bf[tap][nt][0] = v.x;
      bf[tap][nt][1] = v.y;
    }
  const int g = lane >> 2, t = lane & 3;
  float bi[2][2];
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) { bi[nt][0] = bias[8 * nt + 2 * t]; bi[nt][1] = bias[8 * nt + 2 * t + 1]; }
  const int r = (lane & 7) + ((lane >> 3) & 1) * 8, h = lane >> 4;
  for (int mt = warp; mt < nmt; mt += nw) {
    const int q0 = mt << 4;
    const int q = min(q0 + r, P - 1);
    const int oy = q / Wout, ox = q - oy * Wout;
    const int base = oy * Win + ox;
    float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int p = base + (tap / 3) * Win + (tap % 3);
      uint32_t a0, a1, a2, a3;
      ldsm_x4(s_in + act_off(p, h), a0, a1, a2, a3);
      mma_bf16(acc[0], a0, a1, a2, a3, bf[tap][0][0], bf[tap][0][1]);
      mma_bf16(acc[1], a0, a1, a2, a3, bf[tap][1][0], bf[tap][1][1]);
    }
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      const int qq = q0 + g + 8 * hh;
      if (qq < P) {
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
          float v0 = fmaxf(acc[nt][2 * hh] + bi[nt][0], 0.f), v1 = fmaxf(acc[nt][2 * hh + 1] + bi[nt][1], 0.f);
          *reinterpret_cast<uint32_t*>(out + act_off(qq, nt) + 4 * t) = pack_bf16x2(v0, v1);
        }
      }
    }
  }
}

// MODE 0: in = [B][2][H][W] network input, out = [B][H][W] network output (float)
// MODE 1: preconditioner correction of complex physical fields
//         in  = w [F][H][W] float2 (channel 0 = Re w * inv_s[f]),
//         aux = M_psi [V][H][W] (channel 1 = (M - 0.075) / 0.025, vesicle f % V),
//         out = z [F][H][W] float2 = w + (s[f] * net, 0);  s = 1 / inv_s (0 if inv_s = 0)
// in and out must not overlap: neighbouring CTAs read the input halo.  H and W
// are powers of two, multiples of 32.
template <int MODE>
__global__ void __launch_bounds__(NA_THREADS, 2) k_net_apply(const void* __restrict__ in, const float* __restrict__ aux,
                                                             const float* __restrict__ inv_s, void* __restrict__ out,
                                                             int H, int W, int V, const uint32_t* __restrict__ fr,
                                                             const float* __restrict__ bias) {
  extern __shared__ __align__(128) unsigned char na_smem[];
  uint32_t* s_in = reinterpret_cast<uint32_t*>(na_smem);                    // [42*42] bf16x2
  unsigned char* bufA = na_smem + NA_IN * NA_IN * 4;                        // 40x40 / 36x36
  unsigned char* bufB = bufA + (NA_T + 8) * (NA_T + 8) * 32;                // 38x38 / 34x34
  const int f = blockIdx.y;
  const int ntx = W / NA_T;
  const int ty0 = (blockIdx.x / ntx) * NA_T, tx0 = (blockIdx.x % ntx) * NA_T;
  const long long fo = (long long)f * H * W;
  const float is = MODE == 1 ? inv_s[f] : 1.f;
  const float sc = is > 0.f ? 1.f / is : 0.f;      // field RMS (0 for a zero field)
  // ---- input tile (periodic halo of 5)
  for (int k = threadIdx.x; k < NA_IN * NA_IN; k += NA_THREADS) {
    const int yy = k / NA_IN, xx = k - yy * NA_IN;
    const int gy = (ty0 + yy - 5) & (H - 1), gx = (tx0 + xx - 5) & (W - 1);
    const long long j = (long long)gy * W + gx;
    float c0, c1;
    if (MODE == 0) {
      const float* x = reinterpret_cast<const float*>(in) + 2 * fo;
      c0 = x[j];
      c1 = x[(long long)H * W + j];
    } else {
      const float2* w = reinterpret_cast<const float2*>(in);
      c0 = w[fo + j].x * is;
      c1 = (aux[(long long)(f % V) * H * W + j] - 0.075f) * 40.f;
    }
    s_in[k] = pack_bf16x2(c0, c1);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = NA_THREADS / 32;
  const int g = lane >> 2, t = lane & 3;
  // ---- layer 0: 2 -> 16, 42x42 -> 40x40; K = tap*2 + channel
  {
    const int Wout = NA_T + 8, Win = NA_IN, P = Wout * Wout, nmt = (P + 15) >> 4;
    uint32_t bf[2][2][2];
#pragma unroll
    for (int ks = 0; ks < 2; ++ks)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
        uint2 v = __ldg(reinterpret_cast<const uint2*>(fr + NF_L0) + (ks * 2 + nt) * 32 + lane);
        bf[ks][nt][0] = v.x;
        bf[ks][nt][1] = v.y;
      }
    float bi[2][2];
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) { bi[nt][0] = bias[8 * nt + 2 * t]; bi[nt][1] = bias[8 * nt + 2 * t + 1]; }
    for (int mt = warp; mt < nmt; mt += nw) {
      const int q0 = mt << 4;
      const int qa = min(q0 + g, P - 1), qb = min(q0 + g + 8, P - 1);
      const int ya = qa / Wout, yb = qb / Wout;
      const int ba = ya * Win + (qa - ya * Wout), bb = yb * Win + (qb - yb * Wout);
      const int o0 = (t / 3) * Win + t % 3, o1 = ((t + 4) / 3) * Win + (t + 4) % 3, o8 = 2 * Win + 2;
      float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
      uint32_t a0 = s_in[ba + o0], a1 = s_in[bb + o0], a2 = s_in[ba + o1], a3 = s_in[bb + o1];
      mma_bf16(acc[0], a0, a1, a2, a3, bf[0][0][0], bf[0][0][1]);
      mma_bf16(acc[1], a0, a1, a2, a3, bf[0][1][0], bf[0][1][1]);
      a0 = t == 0 ? s_in[ba + o8] : 0u;
      a1 = t == 0 ? s_in[bb + o8] : 0u;
      mma_bf16(acc[0], a0, a1, 0u, 0u, bf[1][0][0], bf[1][0][1]);
      mma_bf16(acc[1], a0, a1, 0u, 0u, bf[1][1][0], bf[1][1][1]);
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int qq = q0 + g + 8 * hh;
        if (qq < P) {
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) {
            float v0 = fmaxf(acc[nt][2 * hh] + bi[nt][0], 0.f), v1 = fmaxf(acc[nt][2 * hh + 1] + bi[nt][1], 0.f);
            *reinterpret_cast<uint32_t*>(bufA + act_off(qq, nt) + 4 * t) = pack_bf16x2(v0, v1);
          }
        }
      }
    }
  }
  __syncthreads();
  const uint32_t sA = (uint32_t)__cvta_generic_to_shared(bufA), sB = (uint32_t)__cvta_generic_to_shared(bufB);
  na_hidden(sA, bufB, NA_T + 6, fr + NF_LH, bias + 16);
  __syncthreads();
  na_hidden(sB, bufA, NA_T + 4, fr + NF_LH + NF_LH_SIZE, bias + 32);
  __syncthreads();
  na_hidden(sA, bufB, NA_T + 2, fr + NF_LH + 2 * NF_LH_SIZE, bias + 48);
  __syncthreads();
  // ---- layer 4: 16 -> 1, 34x34 -> 32x32, output to global
  {
    const int Wout = NA_T, Win = NA_T + 2, P = Wout * Wout, nmt = P >> 4;
    uint32_t bf[9][2];
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      uint2 v = __ldg(reinterpret_cast<const uint2*>(fr + NF_L4) + tap * 32 + lane);
      bf[tap][0] = v.x;
      bf[tap][1] = v.y;
    }
    const float b4 = bias[64];
    const int r = (lane & 7) + ((lane >> 3) & 1) * 8, h = lane >> 4;
    for (int mt = warp; mt < nmt; mt += nw) {
      const int q0 = mt << 4;
      const int q = q0 + r;
      const int oy = q / Wout, ox = q - oy * Wout;
      const int base = oy * Win + ox;
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        const int p = base + (tap / 3) * Win + (tap % 3);
        uint32_t a0, a1, a2, a3;
        ldsm_x4(sB + act_off(p, h), a0, a1, a2, a3);
        mma_bf16(acc, a0, a1, a2, a3, bf[tap][0], bf[tap][1]);
      }
      if (t == 0) {
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          const int qq = q0 + g + 8 * hh;
          const int oy2 = qq / Wout, ox2 = qq - oy2 * Wout;
          const long long j = fo + (long long)(ty0 + oy2) * W + (tx0 + ox2);
          const float d = acc[2 * hh] + b4;
          if (MODE == 0) {
            reinterpret_cast<float*>(out)[j] = d;
          } else {
            float2 wv = reinterpret_cast<const float2*>(in)[j];
            wv.x += d * sc;
            reinterpret_cast<float2*>(out)[j] = wv;
          }
        }
      }
    }
  }
}

}  // namespace vsav
