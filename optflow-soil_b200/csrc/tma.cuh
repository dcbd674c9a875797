// tma.cuh -- tiled tensor-memory-accelerator copies (cp.async.bulk.tensor) into shared memory, completed on
// mbarriers: tensor-map encoding on the host and the device-side barrier and copy helpers. Copies are plain
// single-CTA loads of this GPU's own memory (no cluster sharing). Every wait is bounded: a caller that gives up
// records it and takes its global-memory path.
#pragma once
#include <cuda.h>

#include "common.cuh"

namespace ofc {

// a float32 tensor of rank 2 or 3 (dims[0] innermost, in elements; strides of the outer dimensions in bytes) with
// box `box` (elements per dimension), no swizzle, out-of-range elements read as zero. false where the driver entry
// point is missing or the driver refuses the map (base not 16-byte aligned, a stride not a multiple of 16 bytes, a box
// dimension above 256 or an inner box extent that is not a multiple of 16 bytes).
bool tma_map_f32(CUtensorMap* m, const void* base, int rank, const uint64_t* dims, const uint64_t* strides_bytes,
                 const uint32_t* box);

constexpr unsigned TMA_WAIT_LIMIT = 1u << 22;  // polls of an mbarrier before a wait gives up

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// makes mbarrier initialisations visible to the asynchronous proxy (call once after the inits, before a barrier)
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// the issuing thread's arrival, announcing `bytes` of copies that complete this phase
__device__ __forceinline__ void mbar_expect(uint32_t bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// waits for the phase of parity `parity` to complete, at most TMA_WAIT_LIMIT polls; false when it gave up
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (unsigned it = 0; it < TMA_WAIT_LIMIT; it++)
    if (mbar_try(bar, parity)) return true;
  return false;
}

// box of a rank-2 / rank-3 tensor map at element coordinates (c0 innermost) into shared memory at dst
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* m, int c0, int c1, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(c0), "r"(c1), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* m, int c0, int c1, int c2, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}

}  // namespace ofc
