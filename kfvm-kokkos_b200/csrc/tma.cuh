// tma.cuh -- tiled TMA loads (cp.async.bulk.tensor, no multicast) into shared
// memory, completed on an mbarrier, and the host-side encoding of their tensor
// maps through the driver's cuTensorMapEncodeTiled (fetched from the runtime's
// driver entry point, so the library does not link libcuda).
//
// Alignment rules the callers keep: the global base is 16-byte aligned, every
// global stride a multiple of 16 bytes, the box's inner extent a multiple of 16
// bytes, and the innermost start coordinate times the element size a multiple of
// 16 bytes (the hardware does not check the last one before the copy runs).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "tcgen05.cuh"

namespace kfvm {

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// arrive on the barrier and add `bytes` to the transaction count of its phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// untiled bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
               : "memory");
}

// box at (x, y, z) of a 3D map into shared memory at dst; completes on bar
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int x, int y, int z,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

// box at (x, y, z, w) of a 4D map
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, int x, int y, int z, int w,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(bar)
      : "memory");
}

// Host: encode a tiled map of 8-byte elements over a row-major array of rank
// `rank` (dims[0] fastest); strides in bytes for dims 1.., box extents per dim.
// Out-of-range elements of a box read as zero.  Returns 0 on success.
int encode_tensor_map_8b(CUtensorMap *map, const void *base, int rank, const uint64_t *dims,
                         const uint64_t *strides_bytes, const uint32_t *box);

} // namespace kfvm
