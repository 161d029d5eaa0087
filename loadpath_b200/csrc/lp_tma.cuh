// TMA (cp.async.bulk.tensor) and mbarrier helpers for sm_100a, single-CTA use only: no
// cluster multicast anywhere in this library.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#define LP_WAIT_LIMIT (1u << 26)   // mbarrier polls before a wait gives up and flags an error

__device__ __forceinline__ uint32_t lp_smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void lp_mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(lp_smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void lp_fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void lp_mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(lp_smem_addr(bar)), "r"(bytes)
               : "memory");
}

// true when the phase with the given parity has completed
__device__ __forceinline__ bool lp_mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(lp_smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait: false after LP_WAIT_LIMIT polls
__device__ __forceinline__ bool lp_mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < LP_WAIT_LIMIT; ++i)
    if (lp_mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void lp_tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                               uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(lp_smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2),
      "r"(lp_smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void lp_tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                               uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(lp_smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(lp_smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void lp_tma_store_4d(const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                                const void* src) {
  asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(lp_smem_addr(src))
               : "memory");
}

__device__ __forceinline__ void lp_bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void lp_bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void lp_bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// generic-proxy writes to shared memory made visible to the async (TMA) proxy
__device__ __forceinline__ void lp_fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// byte offset within a 32-byte-swizzled TMA destination (1024-byte aligned): the 16-byte chunk
// bit (4) flipped by bit 7
__device__ __forceinline__ uint32_t lp_swz32(uint32_t off) { return off ^ (((off >> 7) & 1u) << 4); }
// byte offset (from a 1024-byte aligned base) of a 128-byte-swizzled TMA destination
__device__ __forceinline__ uint32_t lp_swz128(uint32_t off) { return off ^ (((off >> 7) & 7u) << 4); }

// ---- host: tensor-map encoding through the runtime's driver entry point ------------------
static inline PFN_cuTensorMapEncodeTiled_v12000 lp_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// rank-r tiled map over a dense C-order array; dims/box innermost first; elem 4 or 8 bytes;
// swizzle: 0, or 32 (box rows of exactly 32 bytes; in shared memory byte address bit 4 is XORed
// with bit 7, see lp_swz32) or 128 (box rows of exactly 128 bytes; bits 4-6 XORed with bits
// 7-9, see lp_swz128), destinations then 1024-byte aligned
static inline bool lp_make_map(CUtensorMap* map, const void* base, int rank, const uint64_t* dims,
                               const uint32_t* box, int elem_bytes, int swizzle = 0) {
  auto fn = lp_encode_fn();
  if (!fn) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  cuuint64_t gd[5], gs[4];
  cuuint32_t bx[5], es[5];
  uint64_t stride = (uint64_t)elem_bytes;
  for (int i = 0; i < rank; ++i) {
    gd[i] = dims[i];
    bx[i] = box[i];
    es[i] = 1;
    if (i > 0) {
      gs[i - 1] = stride;
      if (stride % 16) return false;
    }
    stride *= dims[i];
  }
  if ((box[0] * (uint32_t)elem_bytes) % 16) return false;
  if (swizzle && box[0] * (uint32_t)elem_bytes != (uint32_t)swizzle) return false;
  if (swizzle != 0 && swizzle != 32 && swizzle != 128) return false;
  CUtensorMapDataType dt = elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  CUresult r = fn(map, dt, (cuuint32_t)rank, const_cast<void*>(base), gd, gs, bx, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE,
                  swizzle == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                                 : (swizzle == 32 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_NONE),
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}
