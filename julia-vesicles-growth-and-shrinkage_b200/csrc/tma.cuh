// Tensor-memory-accelerator (TMA) tile loads and mbarriers for sm_100a.
//
// The column passes of the psi operator stream tiles of a few whole columns
// through a shared-memory ring: one thread issues a 2D bulk tensor copy per
// box (cp.async.bulk.tensor, the tensor map describing this GPU's own buffer;
// no cluster multicast), the copy engine moves the bytes while the block
// transforms the previous tile, and an mbarrier with an expected byte count
// tells the block when the tile has landed.
//
// Every wait is bounded: after TMA_WAIT_LIMIT polls the wait gives up, sets
// bit VSAV_ERR_PIPELINE in the error word the host reads after the step, and
// returns false (the caller then stops), so a copy that never completes
// cannot hang the GPU.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace vsav {

constexpr int VSAV_ERR_PIPELINE = 16;          // error-word bit: a TMA wait timed out
constexpr unsigned TMA_WAIT_LIMIT = 1u << 26;  // polls before a wait gives up (seconds at the slowest)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// make the initialised barriers visible to the asynchronous (copy-engine) proxy
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// order this thread's earlier generic-proxy shared-memory accesses before later
// asynchronous-proxy writes into the same bytes (a refill of a consumed slot)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// wait for the phase with the given parity to complete; false on timeout (error flagged)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
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
  }
  if (err) atomicOr(err, VSAV_ERR_PIPELINE);
  return false;
}

// one 2D box of a tensor map: global (x = inner, y = outer) -> shared, counted on bar
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_u32(smem_dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// one contiguous block global -> shared (no tensor map), counted on bar; both
// addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gsrc, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(smem_dst)), "l"(reinterpret_cast<uint64_t>(gsrc)), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// one contiguous block shared -> global in this thread's bulk group; both addresses
// 16-byte aligned, bytes a multiple of 16.  The writing threads must have fenced their
// shared-memory stores for the async proxy (fence_proxy_async) before the issue.
__device__ __forceinline__ void bulk_store(void* gdst, const void* smem_src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
               ::"l"(reinterpret_cast<uint64_t>(gdst)), "r"(smem_u32(smem_src)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// until this thread's committed bulk stores have read their shared-memory source
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// until this thread's committed bulk stores are complete
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// ---------------------------------------------------------------------------
// host side: tensor maps of row-major [rows][cols] arrays of 8- or 16-byte
// elements (complex float / complex double), boxes of bw columns x bh rows
// ---------------------------------------------------------------------------
inline PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
      throw std::runtime_error("CUDA error: cuTensorMapEncodeTiled is unavailable");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// elem_bytes 8: complex float as one 8-byte element; 16: complex double as two
inline CUtensorMap make_tile_map(const void* base, int elem_bytes, long long rows, int cols, int bw, int bh) {
  const int per = elem_bytes / 8;                     // 8-byte units per element
  if (((uintptr_t)base & 15) != 0) throw std::runtime_error("tensor map base must be 16-byte aligned");
  if ((long long)cols * elem_bytes % 16 != 0) throw std::runtime_error("tensor map row pitch must be a multiple of 16 bytes");
  if ((long long)bw * elem_bytes % 16 != 0) throw std::runtime_error("tensor map box width must be a multiple of 16 bytes");
  if (bh < 1 || bh > 256 || bw * per > 256) throw std::runtime_error("tensor map box too large");
  CUtensorMap m;
  cuuint64_t dims[2] = {(cuuint64_t)cols * per, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols * elem_bytes};
  cuuint32_t box[2] = {(cuuint32_t)(bw * per), (cuuint32_t)bh};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = tma_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(base), dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw std::runtime_error("CUDA error: cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return m;
}

}  // namespace vsav
