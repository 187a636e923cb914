// tcgen05.cuh -- inline-PTX helpers for the tcgen05 tensor-core kernels (sm_100a):
// shared-memory matrix descriptors, instruction descriptors, MMA issue and
// commit, bounded mbarrier waits and tensor-memory loads.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace kfvm {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// shared-memory matrix descriptor: start, leading (K) and stride (8-row group)
// byte offsets, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: D f32, A and B tf32, both K-major, M = 128, N = NP
template <int NP>
__host__ __device__ constexpr uint32_t tf32_idesc() {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(NP >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// the same rounding (to nearest, ties away from zero, on the magnitude) with
// integer operations: add half a unit of the last kept bit, drop the 13 low bits
__device__ __forceinline__ uint32_t tf32_rna_bits(float x) {
  return (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u;
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, const uint32_t (&v)[4]) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v[0]), "r"(v[1]), "r"(v[2]),
               "r"(v[3])
               : "memory");
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, int acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// bounded wait for the completion of the mbarrier phase with the given parity: an
// iteration cap and a time limit, the clock read first after 64 polls (a wait
// that completes quickly never reads the global timer)
constexpr uint64_t kTcWaitNs = 1000000000ull;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint64_t limit_ns = kTcWaitNs) {
  uint64_t t0 = 0;
  for (uint32_t it = 0; it < (1u << 26); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 63u) == 63u) {
      const uint64_t now = global_ns();
      if (it == 63u) t0 = now;
      else if (now - t0 > limit_ns) return false;
    }
  }
  return false;
}

// 2 consecutive TMEM columns (an even column) of this warp's 32 lanes, waited for
// in the same asm statement
__device__ __forceinline__ void tmem_ld2(uint32_t taddr, float &r0, float &r1) {
  uint32_t x0, x1;
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(x0), "=r"(x1)
      : "r"(taddr)
      : "memory");
  r0 = __uint_as_float(x0);
  r1 = __uint_as_float(x1);
}

// A column pair (an even column) of each of NV accumulators that lie `stride`
// columns apart, with one wait for all of them: the loads are issued back to back
// and the wait names every destination register, so no use can move above it.
template <int NV>
__device__ __forceinline__ void tmem_ld2_n(uint32_t taddr, uint32_t stride, float (&a0)[NV], float (&a1)[NV]) {
  static_assert(NV == 5 || NV == 9, "Euler / Navier-Stokes or GLM-MHD variable counts");
  uint32_t x[2 * NV];
#pragma unroll
  for (int v = 0; v < NV; v++)
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];"
                 : "=r"(x[2 * v]), "=r"(x[2 * v + 1])
                 : "r"(taddr + (uint32_t)v * stride)
                 : "memory");
  if constexpr (NV == 5) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]), "+r"(x[7]),
                   "+r"(x[8]), "+r"(x[9])
                 :
                 : "memory");
  } else {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]), "+r"(x[7]),
                   "+r"(x[8]), "+r"(x[9]), "+r"(x[10]), "+r"(x[11]), "+r"(x[12]), "+r"(x[13]), "+r"(x[14]),
                   "+r"(x[15]), "+r"(x[16]), "+r"(x[17])
                 :
                 : "memory");
  }
#pragma unroll
  for (int v = 0; v < NV; v++) {
    a0[v] = __uint_as_float(x[2 * v]);
    a1[v] = __uint_as_float(x[2 * v + 1]);
  }
}

// 8 consecutive TMEM columns of this warp's 32 lanes, waited for in the same asm
// statement so no use of the registers can move above the wait
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&r)[8]) {
  uint32_t x0, x1, x2, x3, x4, x5, x6, x7;
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(x0), "=r"(x1), "=r"(x2), "=r"(x3), "=r"(x4), "=r"(x5), "=r"(x6), "=r"(x7)
      : "r"(taddr)
      : "memory");
  r[0] = __uint_as_float(x0);
  r[1] = __uint_as_float(x1);
  r[2] = __uint_as_float(x2);
  r[3] = __uint_as_float(x3);
  r[4] = __uint_as_float(x4);
  r[5] = __uint_as_float(x5);
  r[6] = __uint_as_float(x6);
  r[7] = __uint_as_float(x7);
}

// instruction descriptor: D f32, A and B bf16, both K-major, M = 128, N = NP
template <int NP>
__host__ __device__ constexpr uint32_t bf16_idesc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NP >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, int acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z)
      : "memory");
}

} // namespace kfvm
