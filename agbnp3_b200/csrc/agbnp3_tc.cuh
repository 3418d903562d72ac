/*
 * 5th-generation tensor-core (tcgen05) building blocks for sm_100a: shared-
 * memory operand descriptors, the BF16 x BF16 -> FP32 MMA with its
 * accumulator in tensor memory (TMEM), commit to an mbarrier, bounded
 * waits, TMEM allocation and row loads.
 *
 * Operand layout in shared memory (K-major, no swizzle): a tile of R rows
 * x K bf16 is stored as 8-row x 8-element "core matrices" of 128 bytes;
 * element (r, k) sits at byte
 *     (k / 8) * 128 + (r / 8) * (K / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
 * so the two 8-element halves of one 16-wide K step are 128 bytes apart
 * (the descriptor's leading offset) and consecutive 8-row groups are
 * K * 16 bytes apart (its stride offset).  The MMA of the k-th K step
 * starts at byte k * 256 of both operands.
 *
 * The accumulator D (M = 128 rows x N fp32) lives in TMEM: row i in lane
 * i, column n in TMEM column n.  Warp w of a 128-thread block reads lanes
 * 32 w .. 32 w + 31.
 */
#ifndef AGBNP3_TC_CUH
#define AGBNP3_TC_CUH

#include <cuda_bf16.h>
#include <stdint.h>

__device__ __forceinline__ uint32_t tc_smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

/* byte offset of element (r, k) of a K-major R x K bf16 tile */
__device__ __forceinline__ uint32_t tc_off(int r, int k, int K) {
  return (uint32_t)((k >> 3) * 128 + (r >> 3) * (K >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

/* shared-memory matrix descriptor: K-major, no swizzle, sm_100 version */
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

/* instruction descriptor: A, B bf16 (K-major), D fp32, M x N */
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

/* D (+)= A * B^T for one 16-wide K step; issued by one thread */
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

/* the mbarrier completes once every MMA issued so far by this thread is done */
__device__ __forceinline__ void tc_commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
      tc_smem_u32(mbar)));
}

__device__ __forceinline__ void tc_mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(mbar)), "r"(count));
}

/* waits for the given phase parity, at most max_iter polls; false: gave up */
__device__ __forceinline__ bool tc_mbar_wait(uint64_t *mbar, uint32_t parity, int max_iter) {
  const uint32_t a = tc_smem_u32(mbar);
  for (int i = 0; i < max_iter; i++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

/* generic-proxy shared-memory writes become visible to the MMA (async proxy) */
__device__ __forceinline__ void tc_fence_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

/* allocation by one whole warp; the TMEM address is written to *slot */
__device__ __forceinline__ void tc_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(slot)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

/* 16 consecutive fp32 columns of this thread's TMEM lane */
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

#endif
