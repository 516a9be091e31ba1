// Learned correction of the psi preconditioner: a small convolutional network
// (five 3x3 convolutions, 2 -> 16 -> 16 -> 16 -> 16 -> 1 channels, ReLU after
// the first four), trained on the GPU by the kernels below and applied inside
// the flexible BiCGSTAB of the psi solve.  The reference has only the
// diagonal spectral preconditioner (src/Solvers.jl:53-75); this part has no
// counterpart there.
//
// Parameters: one FP32 master vector theta, layer by layer W[o][i][ky][kx]
// then b[o] (7409 values).  The convolution weights are used BF16-rounded
// (round to nearest even), the biases in FP32; gradients are taken w.r.t. the
// rounded weights.  Activations: [B][C][H][W] FP32 in the training kernels.
// Convolutions are cross-correlations, periodic (output size = input size) or
// valid (output 2 smaller per dimension).
#pragma once
#include "net_common.cuh"
#include <vector>
#include <cstring>
#include <algorithm>

namespace vsav {

// ---------------------------------------------------------------------------
// forward convolution: 16x16 output tile per block, one output pixel (all O
// channels) per thread.  Weights staged transposed [i][tap][o] so one tap's O
// weights are contiguous (float4 broadcast reads).
// ---------------------------------------------------------------------------
template <int I, int O, bool P>
__global__ void __launch_bounds__(256) k_conv_fwd(const float* __restrict__ in, const float* __restrict__ wb, int H, int W,
                                                  int relu, float* __restrict__ out) {
  constexpr int TS = 16, TI = TS + 2;
  __shared__ float sx[I][TI][TI + 1];
  __shared__ __align__(16) float sw[I * 9 * O];
  __shared__ float sb[O];
  const int Ho = P ? H : H - 2, Wo = P ? W : W - 2;
  const int ntx = (Wo + TS - 1) / TS;
  const int b = blockIdx.y;
  const int oy0 = (blockIdx.x / ntx) * TS, ox0 = (blockIdx.x % ntx) * TS;
  for (int k = threadIdx.x; k < I * 9 * O; k += blockDim.x) {
    int o = k % O, it = k / O;                 // it = i*9 + tap
    int i = it / 9, tap = it % 9;
    sw[k] = wb[(o * I + i) * 9 + tap];
  }
  if (threadIdx.x < O) sb[threadIdx.x] = wb[O * I * 9 + threadIdx.x];
  const float* inb = in + (long long)b * I * H * W;
  for (int k = threadIdx.x; k < I * TI * TI; k += blockDim.x) {
    int i = k / (TI * TI), r = k % (TI * TI), yy = r / TI, xx = r % TI;
    int gy, gx;
    float v = 0.f;
    if (P) {
      gy = ((oy0 + yy - 1) % H + H) % H;
      gx = ((ox0 + xx - 1) % W + W) % W;
      v = inb[((long long)i * H + gy) * W + gx];
    } else {
      gy = oy0 + yy; gx = ox0 + xx;
      if (gy < H && gx < W) v = inb[((long long)i * H + gy) * W + gx];
    }
    sx[i][yy][xx] = v;
  }
  __syncthreads();
  const int ly = threadIdx.x / TS, lx = threadIdx.x % TS;
  const int oy = oy0 + ly, ox = ox0 + lx;
  if (oy >= Ho || ox >= Wo) return;
  float acc[O];
#pragma unroll
  for (int o = 0; o < O; ++o) acc[o] = sb[o];
#pragma unroll 1
  for (int i = 0; i < I; ++i) {
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const float xv = sx[i][ly + tap / 3][lx + tap % 3];
      const float* w = sw + (i * 9 + tap) * O;
      if constexpr (O % 4 == 0) {
#pragma unroll
        for (int o = 0; o < O; o += 4) {
          float4 w4 = *reinterpret_cast<const float4*>(w + o);
          acc[o] = fmaf(w4.x, xv, acc[o]);
          acc[o + 1] = fmaf(w4.y, xv, acc[o + 1]);
          acc[o + 2] = fmaf(w4.z, xv, acc[o + 2]);
          acc[o + 3] = fmaf(w4.w, xv, acc[o + 3]);
        }
      } else {
#pragma unroll
        for (int o = 0; o < O; ++o) acc[o] = fmaf(w[o], xv, acc[o]);
      }
    }
  }
  float* ob = out + (long long)b * O * Ho * Wo;
#pragma unroll
  for (int o = 0; o < O; ++o) {
    float v = acc[o];
    if (relu) v = fmaxf(v, 0.f);
    ob[((long long)o * Ho + oy) * Wo + ox] = v;
  }
}

// ---------------------------------------------------------------------------
// input gradient: gx[i][y][x] = sum_o,tap W[o][i][tap] g[o][y - ky (+1)][x - kx (+1)]
// (valid: terms outside the output are zero), times the ReLU mask of the
// layer's input activation when `act` is given.
// ---------------------------------------------------------------------------
template <int I, int O, bool P>
__global__ void __launch_bounds__(256) k_conv_bwd_x(const float* __restrict__ g, const float* __restrict__ wb, int H, int W,
                                                    const float* __restrict__ act, float* __restrict__ gx) {
  constexpr int TS = 16, TI = TS + 2;
  __shared__ float sg[O][TI][TI + 1];
  __shared__ __align__(16) float sw[O * 9 * I];
  const int Ho = P ? H : H - 2, Wo = P ? W : W - 2;
  const int ntx = (W + TS - 1) / TS;
  const int b = blockIdx.y;
  const int y0 = (blockIdx.x / ntx) * TS, x0 = (blockIdx.x % ntx) * TS;
  for (int k = threadIdx.x; k < O * 9 * I; k += blockDim.x) {
    int i = k % I, ot = k / I;                 // ot = o*9 + tap
    int o = ot / 9, tap = ot % 9;
    sw[k] = wb[(o * I + i) * 9 + tap];
  }
  const float* gb = g + (long long)b * O * Ho * Wo;
  for (int k = threadIdx.x; k < O * TI * TI; k += blockDim.x) {
    int o = k / (TI * TI), r = k % (TI * TI), yy = r / TI, xx = r % TI;
    float v = 0.f;
    if (P) {
      int gy = ((y0 + yy - 1) % H + H) % H, gxx = ((x0 + xx - 1) % W + W) % W;
      v = gb[((long long)o * Ho + gy) * Wo + gxx];
    } else {
      int gy = y0 + yy - 2, gxx = x0 + xx - 2;
      if (gy >= 0 && gy < Ho && gxx >= 0 && gxx < Wo) v = gb[((long long)o * Ho + gy) * Wo + gxx];
    }
    sg[o][yy][xx] = v;
  }
  __syncthreads();
  const int ly = threadIdx.x / TS, lx = threadIdx.x % TS;
  const int y = y0 + ly, x = x0 + lx;
  if (y >= H || x >= W) return;
  float acc[I];
#pragma unroll
  for (int i = 0; i < I; ++i) acc[i] = 0.f;
#pragma unroll 1
  for (int o = 0; o < O; ++o) {
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int ky = tap / 3, kx = tap % 3;
      const float gv = sg[o][ly + 2 - ky][lx + 2 - kx];
      const float* w = sw + (o * 9 + tap) * I;
      if constexpr (I % 4 == 0) {
#pragma unroll
        for (int i = 0; i < I; i += 4) {
          float4 w4 = *reinterpret_cast<const float4*>(w + i);
          acc[i] = fmaf(w4.x, gv, acc[i]);
          acc[i + 1] = fmaf(w4.y, gv, acc[i + 1]);
          acc[i + 2] = fmaf(w4.z, gv, acc[i + 2]);
          acc[i + 3] = fmaf(w4.w, gv, acc[i + 3]);
        }
      } else {
#pragma unroll
        for (int i = 0; i < I; ++i) acc[i] = fmaf(w[i], gv, acc[i]);
      }
    }
  }
  const long long base = (long long)b * I * H * W;
#pragma unroll
  for (int i = 0; i < I; ++i) {
    const long long j = base + ((long long)i * H + y) * W + x;
    float v = acc[i];
    if (act && !(act[j] > 0.f)) v = 0.f;
    gx[j] = v;
  }
}

// ---------------------------------------------------------------------------
// weight gradient, per-block partial sums over a strided set of 16x16 output
// tiles: part[blk][(o*I + i)*9 + tap] and part[blk][O*I*9 + o] (bias)
// ---------------------------------------------------------------------------
template <int I, int O, bool P>
__global__ void __launch_bounds__(256) k_conv_bwd_w(const float* __restrict__ g, const float* __restrict__ x, int B, int H,
                                                    int W, float* __restrict__ part) {
  constexpr int TS = 16, TI = TS + 2, NE = O * I * 9 + O, EPT = (NE + 255) / 256;
  __shared__ float sx[I][TI][TI + 1];
  __shared__ float sg[O][TS * TS];
  const int Ho = P ? H : H - 2, Wo = P ? W : W - 2;
  const int ntx = (Wo + TS - 1) / TS, nty = (Ho + TS - 1) / TS;
  const long long ntiles = (long long)B * ntx * nty;
  float acc[EPT];
  int eo[EPT], ei[EPT], et[EPT];
#pragma unroll
  for (int j = 0; j < EPT; ++j) {
    acc[j] = 0.f;
    int e = threadIdx.x + j * 256;
    if (e < O * I * 9) { eo[j] = e / (I * 9); ei[j] = (e / 9) % I; et[j] = e % 9; }
    else if (e < NE) { eo[j] = e - O * I * 9; ei[j] = -1; et[j] = 0; }
    else { eo[j] = -1; ei[j] = -1; et[j] = 0; }
  }
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int b = (int)(tile / (ntx * nty));
    const int tt = (int)(tile % (ntx * nty));
    const int oy0 = (tt / ntx) * TS, ox0 = (tt % ntx) * TS;
    __syncthreads();
    const float* xb = x + (long long)b * I * H * W;
    for (int k = threadIdx.x; k < I * TI * TI; k += blockDim.x) {
      int i = k / (TI * TI), r = k % (TI * TI), yy = r / TI, xx = r % TI;
      float v = 0.f;
      if (P) {
        int gy = ((oy0 + yy - 1) % H + H) % H, gxx = ((ox0 + xx - 1) % W + W) % W;
        v = xb[((long long)i * H + gy) * W + gxx];
      } else {
        int gy = oy0 + yy, gxx = ox0 + xx;
        if (gy < H && gxx < W) v = xb[((long long)i * H + gy) * W + gxx];
      }
      sx[i][yy][xx] = v;
    }
    const float* gb = g + (long long)b * O * Ho * Wo;
    for (int k = threadIdx.x; k < O * TS * TS; k += blockDim.x) {
      int o = k / (TS * TS), r = k % (TS * TS), yy = r / TS, xx = r % TS;
      int gy = oy0 + yy, gxx = ox0 + xx;
      sg[o][r] = (gy < Ho && gxx < Wo) ? gb[((long long)o * Ho + gy) * Wo + gxx] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < EPT; ++j) {
      if (eo[j] < 0) continue;
      const float* gr = sg[eo[j]];
      float a = 0.f;
      if (ei[j] < 0) {
        for (int p = 0; p < TS * TS; ++p) a += gr[p];
      } else {
        const int ky = et[j] / 3, kx = et[j] % 3;
        const float* xr = &sx[ei[j]][0][0];
        for (int py = 0; py < TS; ++py) {
#pragma unroll 4
          for (int px = 0; px < TS; ++px) a = fmaf(gr[py * TS + px], xr[(py + ky) * (TI + 1) + px + kx], a);
        }
      }
      acc[j] += a;
    }
  }
  float* pb = part + (long long)blockIdx.x * NE;
#pragma unroll
  for (int j = 0; j < EPT; ++j) {
    int e = threadIdx.x + j * 256;
    if (e < NE) pb[e] = acc[j];
  }
}

// grad[off + e] = sum over blocks of part[blk][e]   (fixed order: deterministic)
__global__ void k_sum_parts(const float* __restrict__ part, int nblk, int ne, float* __restrict__ grad) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  double s = 0.0;
  for (int k = 0; k < nblk; ++k) s += part[(long long)k * ne + e];
  grad[e] = (float)s;
}

// partial sums of w (out - t)^2 and w t^2 (FP64); w = wsample[k / per] (1 if NULL)
__global__ void __launch_bounds__(256) k_loss_parts(const float* __restrict__ out, const float* __restrict__ t, long long n,
                                                    const float* __restrict__ wsample, long long per,
                                                    double2* __restrict__ part) {
  __shared__ double smm[2 * 2 * 8];
  KSum acc[2] = {{0, 0}, {0, 0}};
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double w = wsample ? (double)wsample[k / per] : 1.0;
    double d = (double)out[k] - (double)t[k];
    acc[0].add(w * d * d);
    acc[1].add(w * (double)t[k] * (double)t[k]);
  }
  block_reduce_store<2>(acc, part + 2 * blockIdx.x, smm);
}
__global__ void k_loss_fin(const double2* __restrict__ part, int nb, double* __restrict__ lsum) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  KSum a{0, 0}, b{0, 0};
  for (int k = 0; k < nb; ++k) { a.merge(part[2 * k].x, part[2 * k].y); b.merge(part[2 * k + 1].x, part[2 * k + 1].y); }
  lsum[0] = a.val();
  lsum[1] = b.val();
}
// g = scale w (out - t), scale = 2 / sum w t^2 (normalised) or 1 (plain 1/2 sum (out-t)^2)
__global__ void k_loss_grad(const float* __restrict__ out, const float* __restrict__ t, long long n,
                            const float* __restrict__ wsample, long long per, const double* __restrict__ lsum,
                            int normalised, float* __restrict__ g) {
  const float sc = normalised ? (float)(2.0 / fmax(lsum[1], 1e-300)) : 1.f;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    g[k] = sc * (wsample ? wsample[k / per] : 1.f) * (out[k] - t[k]);
}

// ---------------------------------------------------------------------------
// residual-norm loss of valid-convolution crops.  The preconditioner's error
// out - t is weighted by the psi operator in grid units,
//   L u = c0 u - div_h(M grad_h u)
// (conservative 5-point stencil, face coefficient = mean of the two cells,
// M = 0.075 + 0.025 * input channel 1 of the crop at offset 5), evaluated at
// the interior output points: the loss is the residual that the corrected
// preconditioner leaves, sum w |L(out - t)|^2 / sum w |L t|^2.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float crop_M(const float* __restrict__ x, int b, int S, int oy, int ox) {
  return 0.075f + 0.025f * x[((long long)(2 * b + 1) * S + oy + 5) * S + ox + 5];
}
__global__ void __launch_bounds__(256) k_loss_res_parts(const float* __restrict__ out, const float* __restrict__ t,
                                                        const float* __restrict__ x, int B, int S, float c0,
                                                        const float* __restrict__ wsample, float* __restrict__ R,
                                                        double2* __restrict__ part) {
  __shared__ double smm[2 * 2 * 8];
  KSum acc[2] = {{0, 0}, {0, 0}};
  const int Ho = S - 10;
  const long long per = (long long)Ho * Ho, n = (long long)B * per;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(k / per), r = (int)(k - (long long)b * per), oy = r / Ho, ox = r - oy * Ho;
    float res = 0.f;
    if (oy > 0 && oy < Ho - 1 && ox > 0 && ox < Ho - 1) {
      const float mc = crop_M(x, b, S, oy, ox);
      const float me = 0.5f * (mc + crop_M(x, b, S, oy, ox + 1)), mw = 0.5f * (mc + crop_M(x, b, S, oy, ox - 1));
      const float mn = 0.5f * (mc + crop_M(x, b, S, oy + 1, ox)), ms = 0.5f * (mc + crop_M(x, b, S, oy - 1, ox));
      const long long c = k;
      auto Lop = [&](const float* f, bool diff) {
        auto u = [&](long long j) { return diff ? out[j] - t[j] : t[j]; };
        const float uc = u(c);
        return c0 * uc - (me * (u(c + 1) - uc) - mw * (uc - u(c - 1)) + mn * (u(c + Ho) - uc) - ms * (uc - u(c - Ho)));
      };
      res = Lop(out, true);
      const float lt = Lop(t, false);
      const double w = wsample ? (double)wsample[b] : 1.0;
      acc[0].add(w * (double)res * res);
      acc[1].add(w * (double)lt * lt);
    }
    R[k] = res;
  }
  block_reduce_store<2>(acc, part + 2 * blockIdx.x, smm);
}
// g = 2 w L^T R / sum w |L t|^2
__global__ void k_loss_res_grad(const float* __restrict__ R, const float* __restrict__ x, int B, int S, float c0,
                                const float* __restrict__ wsample, const double* __restrict__ lsum, float* __restrict__ g) {
  const int Ho = S - 10;
  const long long per = (long long)Ho * Ho, n = (long long)B * per;
  const float sc = (float)(2.0 / fmax(lsum[1], 1e-300));
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(k / per), r = (int)(k - (long long)b * per), oy = r / Ho, ox = r - oy * Ho;
    const float mc = crop_M(x, b, S, oy, ox);
    float diag = c0, off = 0.f;
    const int dy[4] = {0, 0, 1, -1}, dx[4] = {1, -1, 0, 0};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int ny = oy + dy[q], nx = ox + dx[q];
      if (ny < 0 || ny >= Ho || nx < 0 || nx >= Ho) continue;
      const float m = 0.5f * (mc + crop_M(x, b, S, ny, nx));
      diag += m;
      off += m * R[k + (long long)dy[q] * Ho + dx[q]];
    }
    const float w = wsample ? wsample[b] : 1.f;
    g[k] = sc * w * (diag * R[k] - off);
  }
}

__device__ __forceinline__ bool net_is_weight(int k) {
#pragma unroll
  for (int l = 0; l < NET_NL; ++l)
    if (k < net_woff(l) + net_lsize(l)) return k < net_woff(l) + net_wsize(l);
  return false;
}

// Adam on the FP32 master parameters, then the BF16-rounded working copy
__global__ void k_adam(float* __restrict__ th, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ g,
                       float* __restrict__ wb, float lr, float b1, float b2, float eps, float bc1, float bc2) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= NET_NPARAM) return;
  float gk = g[k];
  float mk_ = b1 * m[k] + (1.f - b1) * gk;
  float vk_ = b2 * v[k] + (1.f - b2) * gk * gk;
  m[k] = mk_;
  v[k] = vk_;
  float t = th[k] - lr * (mk_ / bc1) / (sqrtf(vk_ / bc2) + eps);
  th[k] = t;
  wb[k] = net_is_weight(k) ? bf16_round(t) : t;
}
__global__ void k_round_params(const float* __restrict__ th, float* __restrict__ wb) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= NET_NPARAM) return;
  wb[k] = net_is_weight(k) ? bf16_round(th[k]) : th[k];
}

// crops of a [n][C][Hs][Ws] set into a contiguous batch (index list on the
// device); the first nflip values of crop b are multiplied by sgn[b] (sign
// augmentation; sgn NULL: none)
__global__ void k_gather_crops(const float* __restrict__ src, const int* __restrict__ idx, const float* __restrict__ sgn,
                               int B, long long per, long long nflip, float* __restrict__ dst) {
  long long tot = (long long)B * per;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += (long long)gridDim.x * blockDim.x) {
    long long b = k / per, r = k - b * per;
    float v = src[(long long)idx[b] * per + r];
    if (sgn && r < nflip) v *= sgn[b];
    dst[k] = v;
  }
}
// per-sample values of a batch: dst[b] = src[idx[b]]
__global__ void k_gather_vals(const float* __restrict__ src, const int* __restrict__ idx, int B, float* __restrict__ dst) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < B) dst[b] = src[idx[b]];
}

// ---------------------------------------------------------------------------
// host side: parameters, optimiser state and the per-layer activations
// ---------------------------------------------------------------------------
struct Net {
  float *theta = nullptr, *m = nullptr, *v = nullptr, *wb = nullptr, *grad = nullptr, *part = nullptr;
  float* act[NET_NL + 1] = {};    // act[0] input, act[l+1] output of layer l (post-ReLU for l < 4)
  float *g0 = nullptr, *g1 = nullptr;
  double2* lpart = nullptr;
  double* lsum = nullptr;
  int* idx = nullptr;
  float *sgn = nullptr, *wb_batch = nullptr;
  long long cap_pix = 0;          // max B*H*W of an input batch
  int cap_batch = 0;
  int nblk_w = 0, nblk_loss = 0;
  long long step = 0;
  cudaStream_t st = nullptr;
  bool own_stream = false;
  std::vector<void*> allocs;

  template <typename X> X* alloc(size_t n) {
    void* p = nullptr;
    VSAV_CUDA(cudaMalloc(&p, n * sizeof(X)));
    allocs.push_back(p);
    return (X*)p;
  }
  void init(long long cap_pixels, int cap_b) {
    VSAV_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    own_stream = true;
    cap_pix = cap_pixels;
    cap_batch = std::max(cap_b, 1);
    theta = alloc<float>(NET_NPARAM); m = alloc<float>(NET_NPARAM); v = alloc<float>(NET_NPARAM);
    wb = alloc<float>(NET_NPARAM); grad = alloc<float>(NET_NPARAM);
    nblk_w = 296;
    part = alloc<float>((size_t)nblk_w * (16 * 16 * 9 + 16));
    for (int l = 0; l <= NET_NL; ++l) act[l] = alloc<float>((size_t)cap_pix * (l == 0 ? 2 : (l == NET_NL ? 1 : 16)));
    g0 = alloc<float>((size_t)cap_pix * 16);
    g1 = alloc<float>((size_t)cap_pix * 16);
    nblk_loss = 592;
    lpart = alloc<double2>(2 * nblk_loss);
    lsum = alloc<double>(2);
    idx = alloc<int>(cap_batch);
    sgn = alloc<float>(cap_batch);
    wb_batch = alloc<float>(cap_batch);
    VSAV_CUDA(cudaMemsetAsync(theta, 0, NET_NPARAM * 4, st));
    reset_opt();
    k_round_params<<<(NET_NPARAM + 255) / 256, 256, 0, st>>>(theta, wb); VSAV_COUNT_LAUNCH();
    VSAV_CUDA(cudaStreamSynchronize(st));
  }
  ~Net() {
    if (st) cudaStreamSynchronize(st);
    for (void* p : allocs) cudaFree(p);
    if (own_stream && st) cudaStreamDestroy(st);
  }
  void reset_opt() {
    VSAV_CUDA(cudaMemsetAsync(m, 0, NET_NPARAM * 4, st));
    VSAV_CUDA(cudaMemsetAsync(v, 0, NET_NPARAM * 4, st));
    step = 0;
  }
  void set_params(const double* h) {
    std::vector<float> f(NET_NPARAM);
    for (int k = 0; k < NET_NPARAM; ++k) f[k] = (float)h[k];
    VSAV_CUDA(cudaMemcpyAsync(theta, f.data(), NET_NPARAM * 4, cudaMemcpyHostToDevice, st));
    k_round_params<<<(NET_NPARAM + 255) / 256, 256, 0, st>>>(theta, wb); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
    reset_opt();
    VSAV_CUDA(cudaStreamSynchronize(st));
  }
  void get_params(double* h, int rounded) {
    std::vector<float> f(NET_NPARAM);
    VSAV_CUDA(cudaMemcpyAsync(f.data(), rounded ? wb : theta, NET_NPARAM * 4, cudaMemcpyDeviceToHost, st));
    VSAV_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < NET_NPARAM; ++k) h[k] = f[k];
  }
  static int out_dim(int n, bool P, int l) { return P ? n : n - 2 * (l + 1); }
  void check(int B, int H, int W, bool P) const {
    if (B <= 0 || H <= 0 || W <= 0) throw std::runtime_error("net: empty batch");
    if (!P && (H < 11 || W < 11)) throw std::runtime_error("net: valid convolution needs inputs of at least 11x11");
    if ((long long)B * H * W > cap_pix) throw std::runtime_error("net: batch exceeds the capacity given at creation");
  }

  template <bool P> void layer_fwd(int l, const float* in, float* out, int B, int H, int W) {
    const int Ho = P ? H : H - 2, Wo = P ? W : W - 2;
    dim3 grid(((Wo + 15) / 16) * ((Ho + 15) / 16), B);
    const float* w = wb + net_woff(l);
    const int relu = l < NET_NL - 1;
    if (l == 0) k_conv_fwd<2, 16, P><<<grid, 256, 0, st>>>(in, w, H, W, relu, out);
    else if (l < NET_NL - 1) k_conv_fwd<16, 16, P><<<grid, 256, 0, st>>>(in, w, H, W, relu, out);
    else k_conv_fwd<16, 1, P><<<grid, 256, 0, st>>>(in, w, H, W, relu, out);
    VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }
  // act[0] must hold the input; output in act[NET_NL]
  template <bool P> void forward(int B, int H, int W) {
    int h = H, w = W;
    for (int l = 0; l < NET_NL; ++l) {
      layer_fwd<P>(l, act[l], act[l + 1], B, h, w);
      if (!P) { h -= 2; w -= 2; }
    }
  }
  // gradient of sum(gout * out) w.r.t. theta (into grad) given act[] from forward
  template <bool P> void backward(const float* gout, int B, int H, int W) {
    int hs[NET_NL + 1], ws[NET_NL + 1];
    hs[0] = H; ws[0] = W;
    for (int l = 0; l < NET_NL; ++l) { hs[l + 1] = P ? hs[l] : hs[l] - 2; ws[l + 1] = P ? ws[l] : ws[l] - 2; }
    const float* g = gout;
    float* gbuf[2] = {g0, g1};
    int cur = 0;
    for (int l = NET_NL - 1; l >= 0; --l) {
      const int h = hs[l], w = ws[l];
      const int ne = net_lsize(l);
      const float* wl = wb + net_woff(l);
      if (l == 0) k_conv_bwd_w<2, 16, P><<<nblk_w, 256, 0, st>>>(g, act[0], B, h, w, part);
      else if (l < NET_NL - 1) k_conv_bwd_w<16, 16, P><<<nblk_w, 256, 0, st>>>(g, act[l], B, h, w, part);
      else k_conv_bwd_w<16, 1, P><<<nblk_w, 256, 0, st>>>(g, act[l], B, h, w, part);
      VSAV_COUNT_LAUNCH();
      k_sum_parts<<<(ne + 255) / 256, 256, 0, st>>>(part, nblk_w, ne, grad + net_woff(l)); VSAV_COUNT_LAUNCH();
      VSAV_LAUNCH_CHECK();
      if (l > 0) {
        dim3 grid(((w + 15) / 16) * ((h + 15) / 16), B);
        float* gx = gbuf[cur];
        if (l < NET_NL - 1) k_conv_bwd_x<16, 16, P><<<grid, 256, 0, st>>>(g, wl, h, w, act[l], gx);
        else k_conv_bwd_x<16, 1, P><<<grid, 256, 0, st>>>(g, wl, h, w, act[l], gx);
        VSAV_COUNT_LAUNCH();
        VSAV_LAUNCH_CHECK();
        g = gx;
        cur ^= 1;
      }
    }
  }
  // loss of act[NET_NL] against t (n values, per-sample weights w over `per`
  // values each, or NULL); its output gradient into gl
  void loss(const float* t, long long n, int normalised, float* gl, const float* w = nullptr, long long per = 1) {
    k_loss_parts<<<nblk_loss, 256, 0, st>>>(act[NET_NL], t, n, w, per, lpart); VSAV_COUNT_LAUNCH();
    k_loss_fin<<<1, 32, 0, st>>>(lpart, nblk_loss, lsum); VSAV_COUNT_LAUNCH();
    k_loss_grad<<<nblk_loss, 256, 0, st>>>(act[NET_NL], t, n, w, per, lsum, normalised, gl); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }
  // residual-norm loss (valid crops of size S, inputs in act[0]); R in rbuf
  void loss_res(const float* t, int B, int S, float c0, float* rbuf, float* gl, const float* w = nullptr) {
    k_loss_res_parts<<<nblk_loss, 256, 0, st>>>(act[NET_NL], t, act[0], B, S, c0, w, rbuf, lpart); VSAV_COUNT_LAUNCH();
    k_loss_fin<<<1, 32, 0, st>>>(lpart, nblk_loss, lsum); VSAV_COUNT_LAUNCH();
    k_loss_res_grad<<<nblk_loss, 256, 0, st>>>(rbuf, act[0], B, S, c0, w, lsum, gl); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }
  void adam(float lr, float b1 = 0.9f, float b2 = 0.999f, float eps = 1e-8f) {
    ++step;
    float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
    k_adam<<<(NET_NPARAM + 255) / 256, 256, 0, st>>>(theta, m, v, grad, wb, lr, b1, b2, eps, bc1, bc2); VSAV_COUNT_LAUNCH();
    VSAV_LAUNCH_CHECK();
  }
};

}  // namespace vsav
