// Tensor Memory Accelerator (TMA) and mbarrier helpers for sm_100a.
//
// Tensor maps are encoded on the host with the driver's cuTensorMapEncodeTiled, reached through
// cudaGetDriverEntryPoint (no link against libcuda); kernels take them as __grid_constant__
// parameters.  Loads are 2-D tiled bulk tensor copies (cp.async.bulk.tensor) into shared
// memory that complete on an mbarrier with a transaction count.  No cluster multicast is used.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sgb {

// ---- host: tensor map encoding ------------------------------------------------------------

// cuTensorMapEncodeTiled from the driver, looked up once per process.
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Row-major matrix of `rows` x `cols` elements (row stride `ld` elements) of `dtype`, read in
// boxes of box_rows x box_cols with the 128-byte swizzle (box_cols x element size must be 128
// bytes).  Returns false if the driver refuses the description (alignment, sizes).
inline bool make_tensor_map_2d(CUtensorMap* map, CUtensorMapDataType dtype, size_t elem_bytes,
                               const void* base, uint64_t rows, uint64_t cols, uint64_t ld,
                               uint32_t box_rows, uint32_t box_cols) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || ((ld * elem_bytes) & 15) ||
      box_cols * elem_bytes != 128 || box_rows > 256)
    return false;
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {ld * elem_bytes};
  const cuuint32_t box[2] = {box_cols, box_rows};
  const cuuint32_t estride[2] = {1, 1};
  return enc(map, dtype, 2, const_cast<void*>(base), dims, strides, box, estride,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// ---- device: mbarriers ----------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for the phase of `parity` to complete, at most `spins` polls (each try_wait may also
// suspend the thread for a short hardware-defined time); false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long spins) {
  for (long long s = 0; s < spins; ++s) {
    if (mbar_test(bar, parity)) return true;
    if (s > 64) __nanosleep(32);
  }
  return false;
}

// ---- device: TMA ------------------------------------------------------------------------------

// Box at (x = innermost coordinate, y = row) of the tensor map into shared memory at dst,
// completing `bytes` of transaction count on bar.  x x element size must be a multiple of 16
// bytes (TMA's alignment rule for the innermost coordinate).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
      "{%2, %3}], [%4];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Orders this thread's earlier generic-proxy global writes before later async-proxy (TMA)
// reads of the same memory by any thread that synchronises with it.
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

}  // namespace sgb
