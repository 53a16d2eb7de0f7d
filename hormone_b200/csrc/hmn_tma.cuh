// hmn_tma.cuh -- Tensor Memory Accelerator staging of the stencil region.
//
// The primitive planes of one state are one 4-D tensor (x, y, z, plane) of
// doubles.  A 3-D tile's stencil region is five boxes of it per plane: the
// x-extended rows (TX+4, TY, TZ) and the low/high y halos (TX, 2, TZ) and z
// halos (TX, TY, 2); each box lands in its own contiguous part of the
// region's shared-memory layout (Tile::pidx).  One thread issues the 5 x 10
// bulk tensor copies on one mbarrier; cells outside the grid arrive as
// zeros and are overwritten from the boundary codes afterwards.  Loads
// only, never multicast.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace hmn {

// tensor maps of the primitive planes of one state, one per box shape
struct TmaMaps {
  CUtensorMap box[3];  // 0: x-extended rows, 1: y halos, 2: z halos
};

// time limit of the wait for the region's copies (ns of the global timer);
// on expiry the kernel records HMN_ETIMEOUT and goes on
constexpr unsigned long long kTmaWaitNs = 1000000000ull;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// make the initialised barrier visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// one box of a 4-D tensor into shared memory, completion counted on `bar`
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}

}  // namespace hmn
