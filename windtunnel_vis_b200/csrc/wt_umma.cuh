// wt_umma.cuh — the few tcgen05 (5th-generation tensor core) operations the learned closure uses:
// tensor-memory allocation, BF16 x BF16 -> F32 MMAs with both operands in shared memory, commit to
// an mbarrier, bounded waits, and tensor-memory loads. sm_100a only.
//
// Operand layout: "K-major, no swizzle". An operand of R rows (M for A, N for B) and K bf16
// columns is stored as 8 x 8 core matrices of 128 contiguous bytes (row r of a core at r * 16 B);
// core (row group g, column group c) starts at g * SBO + c * LBO. Every operand here uses
// LBO = 128 (the two 8-column halves of one K = 16 step are adjacent) and SBO = K / 8 * 128, so a
// tile is dense: element (r, k) of an R x K tile sits at byte kmaj_off(r, k, K).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace wt {
namespace umma {

// byte offset of element (r, k) in a K-major no-swizzle tile with K columns (K % 16 == 0)
__host__ __device__ __forceinline__ uint32_t kmaj_off(uint32_t r, uint32_t k, uint32_t K) {
  return (r >> 3) * (K * 16u) + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: start >> 4 in bits 0-13, LBO >> 4 in 16-29, SBO >> 4 in 32-45,
// descriptor version 1 in bits 46-47 (sm_100), base offset 0, layout type 0 (no swizzle) in 61-63
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16 with BF16 A and B, F32 accumulator, both K-major, dense:
// c_format = 1 (bits 4-5), a_format = 1 (bits 7-9), b_format = 1 (bits 10-12), N >> 3 (bits
// 17-22), M >> 4 (bits 24-28)
template <int M, int N>
__device__ __forceinline__ constexpr uint32_t idesc_bf16() {
  static_assert(M == 64 || M == 128, "M");
  static_assert(N % 16 == 0 && N >= 16 && N <= 256, "N");
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, one K = 16 step; issued by a single thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, bool acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"((uint32_t)acc));
}

// arrive on `mbar` once every tcgen05 operation this thread issued so far has completed
__device__ __forceinline__ void commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// waits for the phase of parity `parity` to complete; false after `limit` polls. Called by whole
// warps, which leave it converged (the tensor-memory loads that follow are warp-collective).
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_u32(mbar);
  uint32_t done = 0;
  for (uint32_t it = 0; it < limit && !done; it++) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
  }
  __syncwarp();
  return done != 0;
}

// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// warp-wide: allocate `ncols` tensor-memory columns (power of two >= 32); the address lands in *slot
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  __syncwarp();
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  __syncwarp();
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// warp-wide: 8 consecutive f32 columns of this thread's lane (lane = 32 * (warp % 4) + lane id)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}
// warp-wide: 32 consecutive f32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Called by every thread of the block, with `dbar` initialised (count 1) at the start of the kernel
// and otherwise unused. Where `pending` is set for some thread (a wait on an MMA's commit timed
// out, so MMAs may still be writing tensor memory), thread 0 (the only thread that issues MMAs)
// commits once more, to `dbar`: its phase 0 completes once every tcgen05 operation thread 0 issued
// has completed. The block waits for that phase (bounded by `limit` polls) so that the tensor
// memory is released only after the MMAs are done with it. Returns false if that wait gave up too.
__device__ __forceinline__ bool drain_before_free(uint64_t* dbar, bool pending, uint32_t limit) {
  fence_before_sync();
  if (!__syncthreads_or(pending)) {
    fence_after_sync();
    return true;
  }
  if (threadIdx.x == 0) {
    fence_after_sync();
    commit(dbar);
  }
  const bool done = mbar_wait(dbar, 0, limit);
  fence_after_sync();
  return done;
}

// tensor-memory address of (lane base of this warp, column)
__device__ __forceinline__ uint32_t tmem_lane_addr(uint32_t base, uint32_t warp, uint32_t col) {
  return base + (((warp & 3u) * 32u) << 16) + col;
}


}  // namespace umma
}  // namespace wt
