// Shared-memory barriers, shared-memory matrix descriptors and the int8 tensor-core instructions
// of sm_100a (tcgen05), as inline PTX, for the kernels that run on the 5th-generation tensor
// cores (hash_tc.cu, witness_tc.cu).  Every wait is bounded: it gives up after a clock budget
// (or when another role of the CTA has flagged a failure) instead of spinning for good.
#pragma once
#include <cstdint>

namespace lgs {
namespace tc {

constexpr long long DRAIN_CYCLES = 4000000000LL;  // ~2 s at 1.9 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
// A waiting thread sleeps in try_wait until the phase completes or this many nanoseconds pass
// (then the wait loops below check their budget and the failure flag), so waiting roles leave
// the issue slots to the working ones.
constexpr uint32_t SUSPEND_NS = 100000;

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity), "r"(SUSPEND_NS)
      : "memory");
  return done != 0;
}
// Bounded wait for the phase with the given parity to complete.  false after `budget` clock
// cycles, or once another role has flagged a failure (*fail != 0; seen within one suspension).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* fail,
                                          long long budget) {
  const long long t0 = clock64();
  while (true) {
    if (mbar_test(bar, parity)) return true;
    if (*fail) return false;
    if (clock64() - t0 > budget) return false;
  }
}
// Bounded wait that ignores the failure flag (draining work already issued).
__device__ __forceinline__ bool mbar_wait_drain(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_test(bar, parity))
    if (clock64() - t0 > DRAIN_CYCLES) return false;
  return true;
}
__device__ __forceinline__ void flag_failure(volatile int* fail, int* err, int code) {
  *fail = 1;
  atomicExch(err, code);
}
// Descriptor of a K-major operand tile in shared memory with the 128-byte swizzle: rows of 128
// bytes (K) at a 128-byte pitch, 8-row atoms 1024 bytes apart, the 16-byte chunk index of row r
// XORed with r mod 8; the tile base 1024-byte aligned.  Advancing K by 32 bytes inside the atom
// adds 32 to the start address.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);  // start address
  d |= (uint64_t)1 << 16;                          // leading byte offset (unused: K fits the atom)
  d |= (uint64_t)(1024 >> 4) << 32;                // stride byte offset: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                          // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                          // SWIZZLE_128B
  return d;
}
// Byte offset of (row, k byte) in such a tile.
__host__ __device__ constexpr uint32_t sw128_off(uint32_t row, uint32_t kb) {
  return row * 128 + ((((kb >> 4) ^ row) & 7) << 4) + (kb & 15);
}
// Instruction descriptor of tcgen05.mma.kind::i8 with unsigned 8-bit A and B, both K-major, and
// a signed 32-bit accumulator: D = S32 (2 << 4), formats 0 (U8), N / 8 at bit 17, M / 16 at 24.
__host__ __device__ constexpr uint32_t idesc_u8(uint32_t M, uint32_t N) {
  return (2u << 4) | ((N >> 3) << 17) | ((M >> 4) << 24);
}
__device__ __forceinline__ void mma_i8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrives once on the barrier when every MMA this thread issued before it has completed.
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}
// 16 consecutive 32-bit accumulator columns of this warp's 32 TMEM lanes (one lane per thread).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
// 8 consecutive 32-bit accumulator columns of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
// 4 consecutive 32-bit accumulator columns of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
}
// One 32-bit accumulator column of this warp's 32 TMEM lanes.
__device__ __forceinline__ uint32_t tmem_ld1(uint32_t taddr) {
  uint32_t r;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];\n" : "=r"(r) : "r"(taddr));
  return r;
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace tc
}  // namespace lgs
