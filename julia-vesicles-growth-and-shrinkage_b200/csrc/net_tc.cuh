// Inference of the learned psi-preconditioner network on the fifth-generation
// tensor cores (tcgen05.mma, BF16 operands from shared memory, FP32
// accumulators in tensor memory), all five layers fused per 32x32 output tile.
//
// Each layer is an implicit GEMM per M-tile of 128 output positions:
// D[128 x 16] = sum over the 9 taps of A_tap[128 x 16] B_tap[16 x 16], with
// A_tap the 16 input channels of the pixels under the tap and B_tap the tap's
// weights (out x in).  The activations live in shared memory in the
// descriptor's canonical K-major no-swizzle layout: two planes (channels 0-7
// and 8-15), 16 bytes per pixel, pixels at a common pitch of 42 (the input
// tile's width).  Output position q = y * 42 + x reads input pixel
// q + dy * 42 + dx under tap (dy, dx), so the A operand of every tap is the
// same layout started dy * 42 + dx pixels later: one descriptor per tap, no
// im2col copy.  Positions with x beyond the layer's width are computed and
// never read by a valid output (a GEMM row depends only on its own A row).
// Layer 0 (2 input channels) reads a packed input plane whose pixel holds the
// two channels of the pixel and of its two right neighbours (8 BF16 values),
// so K = 16 covers two tap rows: two MMAs per M-tile.  Layer 4 (one output
// channel) is an N = 16 MMA of which column 0 is live.
//
// Warp roles (288 threads): warp 0 allocates 256 tensor-memory columns (one
// 16-column accumulator per M-tile of a layer, at most 14) and one of its
// lanes issues the MMAs; warps 1-8 form two epilogue groups of four warps
// (a warp reads the tensor-memory lanes 32 (warp % 4) .. + 31, so each group
// covers the 128 rows of an accumulator).  Group g takes the M-tiles j with
// j % 2 == g: it waits for the tile's MMAs (tcgen05.commit -> mbarrier
// full[j]), loads the accumulator row of its thread (tcgen05.ld), adds the
// bias, applies ReLU, rounds to BF16 and stores the pixel's 32 bytes into the
// next activation buffer, then arrives on done[j].  The MMAs of layer l + 1 on
// a group of M-tiles start once the done barriers of layer l under the group's
// taps (86 positions ahead) are complete.  Every wait is bounded (a timeout sets
// VSAV_ERR_PIPELINE in the error word and the block stops).
//
// Measured on a B200: back-to-back tcgen05.mma of M 128, K 16 cost about 45
// cycles each at N 16 against 129 at N 256 (full rate), so with 16 channels
// the instruction stream of one issuing thread, not the tensor core, bounds
// the layer (the tensor pipe is ~5% active); the mma.sync kernel, whose eight
// warps issue in parallel, is 3.4x faster and stays the default.
//
// The arithmetic is that of k_net_apply (BF16 inputs, weights and
// activations, FP32 accumulation); only the summation order differs.
#pragma once
#include "net_apply.cuh"
#include "tma.cuh"

namespace vsav {

constexpr int NT_T = 32;                     // output tile
constexpr int NT_PW = NT_T + 10;             // pixel pitch of every buffer (input tile width)
constexpr int NT_NPX = 1792;                 // pixels per activation plane (14 M-tiles)
constexpr int NT_XPX = 1920;                 // pixels of the packed input plane
constexpr int NT_PLANE = NT_NPX * 16;        // bytes per channel-half plane
constexpr int NT_ACT = 2 * NT_PLANE;         // bytes per activation buffer
constexpr int NT_WBLK = 512;                 // one 16 x 16 BF16 B operand
constexpr int NT_NWB = 2 + 27 + 9;           // B operands: layer 0 (2), hidden (3 x 9 taps), layer 4 (9 taps)
constexpr int NT_WBYTES = NT_NWB * NT_WBLK;
constexpr int NT_THREADS = 288;
constexpr int NT_TMEM_COLS = 256;
constexpr int NG = 14;                       // M-tiles per MMA group (a whole layer)
// shared-memory map (bytes from a 1024-aligned base)
constexpr int NT_OFF_A = 0, NT_OFF_B = NT_ACT, NT_OFF_X = 2 * NT_ACT;
constexpr int NT_OFF_W = NT_OFF_X + NT_XPX * 16;
constexpr int NT_OFF_BIAS = NT_OFF_W + NT_WBYTES;
constexpr int NT_OFF_BAR = NT_OFF_BIAS + 80 * 4;   // full[16], done[16], fin
constexpr int NT_OFF_MISC = NT_OFF_BAR + 33 * 8;   // tensor-memory base, abort flag
constexpr int NT_SMEM = 1024 + NT_OFF_MISC + 16;

// M-tiles of layer l: the layer's output rows at the common pitch
__host__ __device__ constexpr int nt_tiles(int l) { return ((NT_T + 8 - 2 * l) * NT_PW + 127) / 128; }
static_assert(nt_tiles(0) == 14 && nt_tiles(4) == 11, "tile counts");
static_assert(nt_tiles(0) * 128 <= NT_NPX && 16 * nt_tiles(0) <= NT_TMEM_COLS, "buffer sizes");
// the reads of the last M-tile of each layer stay inside its input buffer
static_assert(nt_tiles(1) * 128 - 1 + 2 * NT_PW + 2 < NT_NPX, "hidden-layer reads");
static_assert(nt_tiles(0) * 128 - 1 + 3 * NT_PW < NT_XPX && NT_PW * NT_PW <= NT_XPX, "layer-0 reads");
static_assert(NT_SMEM <= 227 * 1024, "shared memory");

// byte offset of element (n, k) in a 16 x 16 K-major B operand: core matrices
// of 8 rows x 16 bytes, n-groups 128 bytes apart (SBO), k-halves 256 apart (LBO)
inline int nt_boff(int n, int k) { return (n >> 3) * 128 + (k >> 3) * 256 + (n & 7) * 16 + (k & 7) * 2; }

// wb: BF16-rounded weights + biases in the theta layout (host) -> the B
// operands as an image of shared memory (BF16 bits; NT_WBYTES / 2 values)
inline void net_pack_tc(const float* wb, uint16_t* img) {
  auto W = [&](int l, int o, int i, int tap) { return wb[net_woff(l) + (o * net_cin(l) + i) * 9 + tap]; };
  auto put = [&](int blk, int n, int k, float v) { img[(blk * NT_WBLK + nt_boff(n, k)) / 2] = (uint16_t)bf16_bits_host(v); };
  for (int i = 0; i < NT_WBYTES / 2; ++i) img[i] = 0;
  // layer 0: block a, k-half h covers tap row dy = 2a + h; k = 2 dx + channel
  for (int a = 0; a < 2; ++a)
    for (int h = 0; h < 2; ++h) {
      const int dy = 2 * a + h;
      if (dy > 2) continue;
      for (int n = 0; n < 16; ++n)
        for (int dx = 0; dx < 3; ++dx)
          for (int c = 0; c < 2; ++c) put(a, n, 8 * h + 2 * dx + c, W(0, n, c, 3 * dy + dx));
    }
  for (int l = 1; l <= 3; ++l)
    for (int tap = 0; tap < 9; ++tap)
      for (int n = 0; n < 16; ++n)
        for (int k = 0; k < 16; ++k) put(2 + 9 * (l - 1) + tap, n, k, W(l, n, k, tap));
  for (int tap = 0; tap < 9; ++tap)
    for (int k = 0; k < 16; ++k) put(29 + tap, 0, k, W(4, 0, k, tap));
}

// ---- tcgen05 / tensor-memory primitives (inline PTX)
__device__ __forceinline__ void tc_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tc_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// D (tensor memory) = A B (+ D when acc != 0); A, B by shared-memory descriptors
__device__ __forceinline__ void tc_mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
// arrive on bar once every MMA this thread issued before has completed
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tc_ld1(uint32_t taddr, uint32_t& r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr) : "memory");
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// shared-memory matrix descriptor, K-major, no swizzle (the canonical
// ((8, m), (8 elements, 2)) layout): start, LBO = byte stride of the two
// 16-byte k-halves, SBO = byte stride of 8-row groups, version 1 (sm_100)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = 16, M = 128
constexpr uint32_t NT_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

// bounded wait on an mbarrier phase that also gives up when another thread of
// the block has flagged an abort
__device__ __forceinline__ bool nt_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* err) {
  const uint32_t a = smem_u32(bar);
  for (unsigned it = 0; it < TMA_WAIT_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 1023u) == 1023u && *abort_flag) return false;
  }
  if (err) atomicOr(err, VSAV_ERR_PIPELINE);
  *abort_flag = 1;
  return false;
}

static_assert(nt_tiles(0) <= nt_tiles(1) + 1 && nt_tiles(1) <= nt_tiles(2) + 1 && nt_tiles(2) <= nt_tiles(3) + 1 &&
                  nt_tiles(3) <= nt_tiles(4) + 1, "each done barrier is waited once per layer");

// MODE, in, aux, inv_s, out, H, W, V as k_net_apply; F fields.  Persistent:
// block b walks the tiles b, b + gridDim.x, ... of the F (H / 32) (W / 32)
// output tiles.  wimg: net_pack_tc's image (NT_WBYTES), bias: net_pack's
// biases, err: the error word (bit VSAV_ERR_PIPELINE on a timed-out wait).
template <int MODE>
__global__ void __launch_bounds__(NT_THREADS, 1) k_net_apply_tc(const void* __restrict__ in, const float* __restrict__ aux,
                                                                const float* __restrict__ inv_s, void* __restrict__ out,
                                                                int H, int W, int V, int F, const uint4* __restrict__ wimg,
                                                                const float* __restrict__ bias, int* err) {
  extern __shared__ unsigned char nt_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(nt_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t s0 = smem_u32(sm);
  float* bs = reinterpret_cast<float*>(sm + NT_OFF_BIAS);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + NT_OFF_BAR);
  uint64_t* done = full + 16;
  uint64_t* fin = full + 32;
  uint32_t* tbase_s = reinterpret_cast<uint32_t*>(sm + NT_OFF_MISC);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + NT_OFF_MISC + 4);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // weights, biases, zeroed buffers, barriers, tensor memory
  for (int k = tid; k < NT_WBYTES / 16; k += NT_THREADS) reinterpret_cast<uint4*>(sm + NT_OFF_W)[k] = wimg[k];
  for (int k = tid; k < NF_BIAS; k += NT_THREADS) bs[k] = bias[k];
  for (int k = tid; k < NT_OFF_W / 16; k += NT_THREADS) reinterpret_cast<uint4*>(sm)[k] = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) {
    for (int j = 0; j < 33; ++j) mbar_init(full + j, (j >= 16 && j < 32) ? 128u : 1u);
    *abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == 0) {
    tc_alloc(tbase_s, NT_TMEM_COLS);
    tc_relinquish();
  }
  fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tbase_s;

  const int tpr = W / NT_T, tpf = (H / NT_T) * tpr;
  const long long ntile = (long long)F * tpf;
  uint32_t phf = 0u, phd = 0u;   // phase bits of full[j] (epilogue threads) and done[j] (the MMA thread)
  for (long long tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const int f = (int)(tile / tpf), tt = (int)(tile - (long long)f * tpf);
    const int ty0 = (tt / tpr) * NT_T, tx0 = (tt % tpr) * NT_T;
    const long long fo = (long long)f * H * W;
    const float is = MODE == 1 ? inv_s[f] : 1.f;
    const float sc = is > 0.f ? 1.f / is : 0.f;
    // input tile with a periodic halo of 5: BF16 channel pairs into buffer A
    // (free until layer 0's epilogue), then the packed triples into X
    uint32_t* tmp = reinterpret_cast<uint32_t*>(sm + NT_OFF_A);
    for (int k = tid; k < NT_PW * NT_PW; k += NT_THREADS) {
      const int yy = k / NT_PW, xx = k - yy * NT_PW;
      const int gy = (ty0 + yy - 5) & (H - 1), gx = (tx0 + xx - 5) & (W - 1);
      const long long j = (long long)gy * W + gx;
      float c0, c1;
      if (MODE == 0) {
        const float* x = reinterpret_cast<const float*>(in) + 2 * fo;
        c0 = x[j];
        c1 = x[(long long)H * W + j];
      } else {
        c0 = reinterpret_cast<const float2*>(in)[fo + j].x * is;
        c1 = (aux[(long long)(f % V) * H * W + j] - 0.075f) * 40.f;
      }
      tmp[k] = pack_bf16x2(c0, c1);
    }
    __syncthreads();
    uint4* X = reinterpret_cast<uint4*>(sm + NT_OFF_X);
    for (int k = tid; k < NT_PW * NT_PW; k += NT_THREADS) {
      const int xx = k % NT_PW;
      X[k] = make_uint4(tmp[k], xx + 1 < NT_PW ? tmp[k + 1] : 0u, xx + 2 < NT_PW ? tmp[k + 2] : 0u, 0u);
    }
    fence_proxy_async();
    __syncthreads();
    if (warp == 0) {
      // ---- MMA issue: layer by layer, in groups of NG M-tiles (tap-major over
      // the group's accumulators; groups of 2 and 4 M-tiles measured 16% and
      // 10% slower)
      if (lane == 0 && !*abort_flag) {
        tc_fence_after();
        bool ok = true;
        for (int l = 0; l < NET_NL && ok; ++l) {
          const int nt = nt_tiles(l);
          const uint32_t ibuf = s0 + (l == 0 ? NT_OFF_X : ((l & 1) ? NT_OFF_A : NT_OFF_B));
          const int wb = l == 0 ? 0 : (l < NET_NL - 1 ? 2 + 9 * (l - 1) : 29);
          int nw = 0;                          // done barriers of the previous layer waited so far
          for (int j0 = 0; j0 < nt && ok; j0 += NG) {
            const int j1 = min(j0 + NG, nt);
            if (l > 0) {
              // the previous layer's rows under the group's taps (its M-tiles up to j1) are written
              const int need = min(j1 + 1, nt_tiles(l - 1));
              for (; nw < need && ok; ++nw) {
                ok = nt_wait(done + nw, (phd >> nw) & 1u, abort_flag, err);
                phd ^= 1u << nw;
              }
              if (!ok) break;
              tc_fence_after();
            }
            if (l == 0) {
              // K halves: tap rows 0 and 1, then 2 and 3 (row 3 has zero weights)
              for (int a = 0; a < 2; ++a)
                for (int j = j0; j < j1; ++j)
                  tc_mma_bf16(tbase + 16u * (uint32_t)j,
                              umma_desc(ibuf + (128u * (uint32_t)j + 2u * a * NT_PW) * 16u, NT_PW * 16u, 128u),
                              umma_desc(s0 + NT_OFF_W + a * NT_WBLK, 256u, 128u), NT_IDESC, (uint32_t)a);
            } else {
              for (int tap = 0; tap < 9; ++tap) {
                const uint32_t off = (uint32_t)((tap / 3) * NT_PW + tap % 3);
                const uint64_t bd = umma_desc(s0 + NT_OFF_W + (wb + tap) * NT_WBLK, 256u, 128u);
                for (int j = j0; j < j1; ++j)
                  tc_mma_bf16(tbase + 16u * (uint32_t)j, umma_desc(ibuf + (128u * (uint32_t)j + off) * 16u, NT_PLANE, 128u),
                              bd, NT_IDESC, (uint32_t)tap);
              }
            }
            for (int j = j0; j < j1; ++j) tc_commit(full + j);
          }
        }
      }
      __syncwarp();
    } else {
      // ---- epilogue groups: bias, ReLU, BF16 into the next buffer (layers 0-3); output (layer 4)
      const int g = (warp - 1) >> 2, qd = warp & 3;
      bool ok = true;
      for (int l = 0; l < NET_NL && ok; ++l) {
        const int nt = nt_tiles(l);
        unsigned char* obuf = sm + ((l & 1) ? NT_OFF_B : NT_OFF_A);
        const float* b = bs + 16 * l;
        for (int j = g; j < nt; j += 2) {
          ok = nt_wait(full + j, (phf >> j) & 1u, abort_flag, err);
          phf ^= 1u << j;
          ok = __all_sync(0xffffffffu, ok);
          if (!ok) break;
          tc_fence_after();
          const uint32_t taddr = tbase + ((uint32_t)(qd * 32) << 16) + 16u * (uint32_t)j;
          const int q = j * 128 + qd * 32 + lane;
          if (l < NET_NL - 1) {
            uint32_t r[16];
            tc_ld16(taddr, r);
            tc_wait_ld();
            uint32_t pk[8];
#pragma unroll
            for (int c = 0; c < 8; ++c)
              pk[c] = pack_bf16x2(fmaxf(__uint_as_float(r[2 * c]) + b[2 * c], 0.f),
                                  fmaxf(__uint_as_float(r[2 * c + 1]) + b[2 * c + 1], 0.f));
            *reinterpret_cast<uint4*>(obuf + q * 16) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            *reinterpret_cast<uint4*>(obuf + NT_PLANE + q * 16) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            fence_proxy_async();        // the next layer's MMAs read these bytes
            tc_fence_before();
            mbar_arrive(done + j);
          } else {
            uint32_t r0;
            tc_ld1(taddr, r0);
            tc_wait_ld();
            tc_fence_before();
            const int y = q / NT_PW, x = q - y * NT_PW;
            if (y < NT_T && x < NT_T) {
              const long long jg = fo + (long long)(ty0 + y) * W + (tx0 + x);
              const float dv = __uint_as_float(r0) + b[0];
              if (MODE == 0) {
                reinterpret_cast<float*>(out)[jg] = dv;
              } else {
                float2 wv = reinterpret_cast<const float2*>(in)[jg];
                wv.x += dv * sc;
                reinterpret_cast<float2*>(out)[jg] = wv;
              }
            }
          }
        }
      }
    }
    __syncthreads();
    if (*abort_flag) break;
  }
  // every MMA complete before the tensor memory is released
  if (warp == 0) {
    if (lane == 0) {
      tc_commit(fin);
      mbar_wait(fin, 0u, err);
    }
    __syncwarp();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tc_dealloc(tbase, NT_TMEM_COLS);
  }
}

// host: the kernel's shared-memory size attribute
template <int MODE>
inline cudaError_t net_tc_attributes() {
  return cudaFuncSetAttribute(k_net_apply_tc<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, NT_SMEM);
}

}  // namespace vsav
