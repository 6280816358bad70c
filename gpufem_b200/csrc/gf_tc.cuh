// tcgen05 (5th-generation tensor core) building blocks for sm_100a: shared-memory matrix
// descriptors, the instruction descriptor of kind::tf32, MMA issue, commit to an mbarrier,
// bounded waits, TMEM allocation and 32-lane loads.  Operands are K-major without swizzle:
// canonical core matrices of 8 rows x 16 bytes, so element (r, k) of an R-row FP32 tile sits
// at byte (k / 4) * R * 16 + r * 16 + (k % 4) * 4 and a K step of 8 spans two core-matrix
// columns (leading byte offset R * 16, stride byte offset 128 between 8-row groups).
#pragma once

#include <algorithm>
#include <cstdint>

__device__ __forceinline__ uint32_t tc_smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: K-major, no swizzle; lbo = bytes between core matrices
// adjacent in K, sbo = bytes between 8-row groups.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version of sm_100
  return d;
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both K-major.
constexpr uint32_t tc_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// D (TMEM) (+)= A B^T; issued by one thread.
__device__ __forceinline__ void tc_mma_tf32(uint32_t tmem, uint64_t da, uint64_t db,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accumulate) : "memory");
}

// Arrive on the mbarrier when every MMA this thread issued so far has completed.
__device__ __forceinline__ void tc_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(tc_smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void tc_mbar_init(uint64_t* mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(tc_smem_u32(mbar)), "r"(1));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the completion of the given phase of the mbarrier; false on timeout.
__device__ __forceinline__ bool tc_mbar_wait(uint64_t* mbar, uint32_t phase, int max_iters) {
  uint32_t done = 0;
  for (int it = 0; it < max_iters && !done; ++it)
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done) : "r"(tc_smem_u32(mbar)), "r"(phase) : "memory");
  return done != 0;
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes made visible to the tensor cores' async proxy
__device__ __forceinline__ void tc_fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Warp-wide: allocate ncols TMEM columns (a power of two >= 32), address to *slot.
__device__ __forceinline__ void tc_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :: "r"(tc_smem_u32(slot)), "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tc_dealloc(uint32_t tmem, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(ncols));
}

// Warp-wide: 32 consecutive FP32 columns of this warp's 32 TMEM lanes (lane = thread).
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}
// Warp-wide: 16 consecutive FP32 columns.
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}
__device__ __forceinline__ void tc_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t tc_tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// Resident CTAs per SM of a kernel with `threads` threads, `smem` bytes of dynamic shared
// memory and `tmem_cols` TMEM columns per CTA, from its register count and the SM's limits
// (65,536 registers, 2,048 threads, 233,472 bytes of shared memory less 1 KB reserved per
// CTA, 512 TMEM columns).
template <typename K>
inline int tc_ctas_per_sm(K kernel, int threads, size_t smem, int tmem_cols) {
  cudaFuncAttributes a{};
  if (cudaFuncGetAttributes(&a, kernel) != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  const int regs = ((a.numRegs * 32 + 255) / 256 * 256) * (threads / 32);  // per-warp granule
  int n = regs > 0 ? 65536 / regs : 16;
  n = std::min(n, 2048 / threads);
  n = std::min(n, (int)(233472 / (smem + a.sharedSizeBytes + 1024)));
  n = std::min(n, 512 / tmem_cols);
  return n < 1 ? 1 : n;
}

