// Shape of the learned psi-preconditioner network and BF16 rounding, shared by
// the training kernels (net.cuh) and the fused inference kernel (net_apply.cuh).
#pragma once
#include "vsav_internal.cuh"
#include <cuda_bf16.h>
#include <cstring>

namespace vsav {

constexpr int NET_NL = 5;
__host__ __device__ constexpr int net_cin(int l) { return l == 0 ? 2 : 16; }
__host__ __device__ constexpr int net_cout(int l) { return l == NET_NL - 1 ? 1 : 16; }
__host__ __device__ constexpr int net_wsize(int l) { return net_cout(l) * net_cin(l) * 9; }
__host__ __device__ constexpr int net_lsize(int l) { return net_wsize(l) + net_cout(l); }
__host__ __device__ constexpr int net_woff(int l) { return l == 0 ? 0 : net_woff(l - 1) + net_lsize(l - 1); }
constexpr int NET_NPARAM = net_woff(NET_NL);
static_assert(NET_NPARAM == 7409, "parameter count");

// round to BF16, nearest even, kept as an FP32 value (finite inputs)
__host__ __device__ __forceinline__ float bf16_round(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
  float r;
  memcpy(&r, &u, 4);
  return r;
}

}  // namespace vsav
