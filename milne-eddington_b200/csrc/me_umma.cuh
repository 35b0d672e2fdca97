// me_umma.cuh -- sm_100a building blocks of the learned initialiser's GEMM:
// mbarriers with bounded waits, 2-D TMA tile loads, and the tcgen05 tensor-core
// instructions (tensor-memory allocation, BF16 x BF16 -> FP32 MMA issued by one
// thread, commit to an mbarrier, tensor-memory loads for the epilogue).
//
// Operand tiles are K-major with the 128-byte swizzle that TMA writes: each row
// of a tile is 64 BF16 values (128 bytes), groups of 8 rows are 1024 bytes
// apart, and tile bases are 1024-byte aligned.  One MMA of K = 16 reads a
// 32-byte column slice of every row, so the k-th slice of a stage starts at the
// stage base + 32 k.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace me {
namespace umma {

constexpr int kBM = 128;     // rows of A per CTA: one tensor-memory lane per row
constexpr int kBK = 64;      // K values per stage: one 128-byte swizzle row
constexpr int kMaxBN = 256;  // widest accumulator (256 FP32 tensor-memory columns)
constexpr int kStages = 2;
constexpr int kStageA = kBM * kBK * 2;  // 16 KB; a B stage is bn x 128 bytes
// full[kStages], empty[kStages], done mbarriers, then the tensor-memory base
// address and the CTA's abort flag
constexpr int kBarBytes = 8 * (2 * kStages + 1) + 8;
constexpr int kSmPerSm = 233472;  // shared memory of an SM (228 KB)
constexpr int kSmPerCta = 1024;   // reserved by the system per resident CTA

// Tensor-memory columns of a bn-wide accumulator: a power of two >= 32.
__host__ __device__ constexpr uint32_t tmem_cols(int bn) {
  return bn <= 32 ? 32u : bn <= 64 ? 64u : bn <= 128 ? 128u : 256u;
}

// Dynamic shared memory of a CTA with a bn-wide tile: 1 KB of alignment
// slack, the two stages, the barriers -- and at least enough that no more
// CTAs fit on an SM than its 512 tensor-memory columns can serve, so that
// tcgen05.alloc never has to wait for another CTA to exit.
__host__ __device__ constexpr int smem_bytes(int bn) {
  return (1024 + kStages * (kStageA + bn * kBK * 2) + kBarBytes) >
                 (kSmPerSm / (512 / (int)tmem_cols(bn) + 1) - kSmPerCta + 1)
             ? (1024 + kStages * (kStageA + bn * kBK * 2) + kBarBytes)
             : (kSmPerSm / (512 / (int)tmem_cols(bn) + 1) - kSmPerCta + 1);
}
constexpr int kSmemMax = smem_bytes(kMaxBN);
// give up a wait after 2 s of device time (or 2^26 polls)
constexpr unsigned long long kWaitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the completion of the phase of parity `parity`; false when it has
// not completed within kWaitNs (the caller records an error and stops).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = now_ns();
  for (uint32_t it = 1; it < (1u << 26); it++) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 63) == 0 && now_ns() - t0 > kWaitNs) return false;
  }
  return false;
}

// One box of a 2-D tensor map into shared memory; completion is counted in
// bytes on `bar`.  x (the contiguous coordinate) is a multiple of kBK, so its
// byte offset is a multiple of 128.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

// Tensor memory: allocate / free `ncols` columns (a power of two >= 32) for
// the CTA; executed by one whole warp.  The base address is written to
// shared memory at `dst`.
__device__ __forceinline__ void tmem_alloc(uint32_t dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled operand
// slice starting at `saddr`: start address >> 4 (bits 0-13), leading byte
// offset 16 B (unused by swizzled K-major layouts), stride byte offset 1024 B
// between 8-row groups (bits 32-45), descriptor version 1 (bit 46), base
// offset 0 (tiles are 1024-byte aligned), swizzle mode 2 = 128 B (bits 61-63).
__device__ __forceinline__ uint64_t sw128_kmajor_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(16 >> 4) << 16) |
         ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 D, both
// operands K-major, dense: D format (bits 4-5) = 1, A format (7-9) = 1,
// B format (10-12) = 1, N >> 3 (17-22), M >> 4 (24-28).
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

// D[tmem] (+)= A[adesc] * B[bdesc]^T for one K = 16 slice; issued by one thread
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrives once on `bar` when every MMA this thread issued before has completed
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

// 16 consecutive FP32 columns of the warp's 32 tensor-memory lanes (lane i of
// the warp gets lane base + i); called by the whole warp, which it first
// reconverges; the wait names the registers so that no use is scheduled
// before the data arrive.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  __syncwarp();
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace me
