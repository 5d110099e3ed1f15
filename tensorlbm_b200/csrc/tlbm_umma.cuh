// Blackwell (sm_100a) tensor-core helpers: tcgen05.mma with operands in shared
// memory, accumulators in tensor memory (TMEM), completion through an mbarrier.
//
// Operand layout used throughout: K-major, 128-byte swizzle ("SW128"), bf16.
// A tile of R rows x 64 bf16 (128 bytes per row) is stored as groups of 8 rows
// (1024 bytes, 1024-byte aligned); inside a group row r sits at r*128 and its
// 16-byte chunk c at chunk c ^ r.  The smem matrix descriptor for it is
//   start>>4 | LBO 1 (16 B, unused for swizzled K-major) | SBO 1024>>4 |
//   version 1 | layout SWIZZLE_128B (2)
// and the K-slices of 16 elements (32 bytes) of one MMA are selected by
// advancing the start address by 32 bytes.
#pragma once

#include <cstdint>

namespace tlbm {
namespace umma {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (row, k) of an SW128 K-major bf16 tile (64 columns)
__host__ __device__ __forceinline__ uint32_t sw128_offset(uint32_t row, uint32_t k) {
  return (row >> 3) * 1024u + (row & 7u) * 128u + ((((k >> 3) ^ (row & 7u)) & 7u) << 4) + (k & 7u) * 2u;
}

__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>(1u) << 16;             // leading byte offset (16 B units)
  d |= static_cast<uint64_t>(1024u >> 4) << 32;     // stride byte offset: 8-row group
  d |= static_cast<uint64_t>(1u) << 46;             // descriptor version (sm100)
  d |= static_cast<uint64_t>(2u) << 61;             // SWIZZLE_128B
  return d;
}

// instruction descriptor, kind::f16: D f32, A and B bf16, both K-major
template <int M, int N>
struct IdescBf16 {
  static_assert(M == 128 && N % 16 == 0 && N >= 16 && N <= 256, "M=128, N multiple of 16");
  static constexpr uint32_t value = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) |
                                    (uint32_t(M >> 4) << 24);
};

// D[tmem] (+)= A[smem] * B[smem]^T for one K=16 slice; issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrive once on the mbarrier when every tcgen05.mma issued so far by this thread completes
__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// make this thread's generic-proxy shared-memory writes visible to the tensor cores
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// TMEM allocation: one full warp; the base address is written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t slot_saddr, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_saddr), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive fp32 columns of this warp's 32 TMEM lanes (one lane per thread)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait for the phase with the given parity; false if it gave up
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t max_tries) {
  for (uint32_t i = 0; i < max_tries; ++i)
    if (mbar_try_wait(mbar, parity)) return true;
  return false;
}

// try_wait that may suspend the thread for up to hint_ns nanoseconds (it
// resumes when the phase completes): a waiting warp then sleeps through a
// tensor-core round trip instead of spinning on the barrier
__device__ __forceinline__ bool mbar_try_wait_sleep(uint32_t mbar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

// bounded wait of at most about max_tries * hint_ns nanoseconds
__device__ __forceinline__ bool mbar_wait_sleep(uint32_t mbar, uint32_t parity, uint32_t max_tries, uint32_t hint_ns) {
  for (uint32_t i = 0; i < max_tries; ++i)
    if (mbar_try_wait_sleep(mbar, parity, hint_ns)) return true;
  return false;
}

}  // namespace umma
}  // namespace tlbm
