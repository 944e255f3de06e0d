// heom_umma.cuh -- the 5th-generation tensor-core pieces of the 24-site
// tile kernel: tcgen05.mma kind::tf32 with both operands K-major in shared
// memory (no swizzle) and the accumulator in tensor memory (TMEM), issued by
// one thread; the split-TF32 product hi*hi + lo*hi + hi*lo keeps the FP32
// accuracy of the CUDA-core products (each operand x = hi + lo, hi = x with
// its low 13 mantissa bits cleared, lo = x - hi exact).
//
// Operand layout (PTX ISA, tcgen05 shared-memory matrix descriptors, the
// canonical K-major layout without swizzle): 8-row x 16-byte core matrices
// stored as 128 contiguous bytes; core matrices adjacent along K are
// kUmmaLbo bytes apart, 8-row groups kUmmaSbo(K) bytes apart.  A K-step of
// the tf32 MMA covers 8 elements = two core matrices along K.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace phi {
namespace umma {

constexpr int kLbo = 128;
template <int K>
constexpr int kSbo = (K / 4) * 128;

// Byte offset of element (row r, k) of a K-major operand with K columns.
template <int K>
__device__ __forceinline__ int core_offset(int r, int k) {
  return (r >> 3) * kSbo<K> + (k >> 2) * kLbo + (r & 7) * 16 + (k & 3) * 4;
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address, leading (K) and stride
// (8-row group) byte offsets in 16-byte units, version 1, no swizzle.
template <int K>
__device__ __forceinline__ uint64_t smem_desc(const void *base) {
  const uint64_t a = smem_addr(base);
  uint64_t d = (a >> 4) & 0x3FFFull;
  d |= (uint64_t)((kLbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((kSbo<K> >> 4) & 0x3FFF) << 32;
  d |= 1ull << 46;
  return d;
}

// Instruction descriptor: D in F32, A and B in TF32, both K-major, M x N.
__host__ __device__ constexpr uint32_t instr_desc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

// Warp-wide: allocate `ncols` TMEM columns (a power of two >= 32), address
// written to *slot; the permit is released at once (one allocation per CTA).
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, int ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// One thread: D (+)= A * B^T for one K-step.
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate ? 1u : 0u)
      : "memory");
}
// One thread: the mbarrier at bar completes a phase once every MMA this
// thread issued before has finished.
__device__ __forceinline__ void commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes become visible to the tensor cores.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Warp-wide: 16 / 8 consecutive 32-bit columns of the warp's 32 TMEM lanes
// (lane l of the warp gets row 32 * (warp % 4) + l).
__device__ __forceinline__ void ld_x16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
__device__ __forceinline__ void ld_x8(uint32_t taddr, uint32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
}
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace umma
}  // namespace phi
