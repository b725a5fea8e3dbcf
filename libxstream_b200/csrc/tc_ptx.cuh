/* sm_100a building blocks for the tensor-core (tcgen05) kernels: shared-memory mbarriers with
   bounded waits, TMA tile loads, tensor-memory allocation, UMMA descriptors, tcgen05.mma of kind
   i8, commit and tensor-memory loads. Everything is inline PTX.

   Descriptor bit layouts (PTX ISA "tcgen05 matrix descriptors" / "instruction descriptor"):
     shared-memory matrix descriptor (64 bit): start address >> 4 in [0,14), leading byte offset >> 4
       in [16,30), stride byte offset >> 4 in [32,46), version 1 in [46,48), base offset in [49,52),
       layout type in [61,64) (2 = 128-byte swizzle);
     instruction descriptor (32 bit, kind::i8): D format in [4,6) (2 = s32), A format in [7,10)
       and B format in [10,13) (1 = signed 8 bit), A/B major in bits 15/16 (0 = K-major),
       N >> 3 in [17,23), M >> 4 in [24,29).
   A K-major operand tile staged by TMA with 128-byte swizzle is rows of 128 bytes, eight-row
   atoms 1024 bytes apart (stride byte offset 1024); successive K steps of 32 bytes inside the
   128-byte row advance the start address by 32 bytes. */
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace xs_tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

/* ------------------------------------------------------------------------------ mbarriers */

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
    "{\n\t.reg .pred p;\n\t"
    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
    "selp.u32 %0, 1, 0, p;\n\t}"
    : "=r"(ok)
    : "r"(smem_u32(bar)), "r"(parity)
    : "memory");
  return 0 != ok;
}

/* Non-blocking test of the phase with the given parity. */
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
    "{\n\t.reg .pred p;\n\t"
    "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
    "selp.u32 %0, 1, 0, p;\n\t}"
    : "=r"(ok)
    : "r"(smem_u32(bar)), "r"(parity)
    : "memory");
  return 0 != ok;
}

/* Default bound of a pipeline wait in clock cycles (about two seconds at the boost clock); the
   host may set another one per launch (libxstream_b200_set_wait_limit). */
constexpr long long kDefaultWaitLimit = 4000000000ll;

/* Waits for the phase with the given parity to complete. Gives up when *abort becomes non-zero
   (another role failed) or after `limit` clock cycles, then sets bit `code` in *abort and returns
   false; every wait of a kernel is bounded this way, so a protocol error ends the kernel with an
   error status instead of a hang. The first test does not block and the limit is checked right
   after it, so a phase that is still pending when a wait with a limit of a few cycles starts always
   gives up (the wait-limit test relies on that); later tests use the suspending try_wait. */
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned* abort, unsigned code,
  long long limit = kDefaultWaitLimit) {
  const long long t0 = clock64();
  if (mbar_test_wait(bar, parity)) return true;
  if (clock64() - t0 > limit) {
    atomicOr(abort, code);
    return false;
  }
  for (unsigned it = 1;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (0 == (it & 63)) {
      if (0 != *(volatile unsigned*)abort) return false;
      if (clock64() - t0 > limit) {
        atomicOr(abort, code);
        return false;
      }
    }
  }
}

/* ------------------------------------------------------------------------------------ TMA */

/* 3-D tiled load (x innermost, in elements) of one box into shared memory; completion is
   signalled on the mbarrier as transaction bytes. No cluster multicast. */
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
    "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
      smem_u32(dst)),
    "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
    : "memory");
}

/* 1-D bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16), completion as
   transaction bytes on the mbarrier. No cluster multicast. */
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
    "l"(src), "r"(bytes), "r"(smem_u32(bar))
    : "memory");
}

/* 1-D bulk prefetch of global memory into L2 (16-byte aligned address, size a multiple of 16); no
   completion to wait for. */
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)map) : "memory");
}

/* ------------------------------------------------------------------------- tensor memory */

/* Allocates ncols (power of two >= 32) columns; the base address is written to *dst (shared).
   Executed by one whole warp. */
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

/* ----------------------------------------------------------------------------- UMMA (i8) */

/* K-major operand in shared memory, 128-byte swizzle, 8-row atoms 1024 bytes apart. */
__device__ __forceinline__ uint64_t desc_k_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) | ((uint64_t)1u << 46) |
         ((uint64_t)2u << 61);
}

/* K-major operand without swizzle: core matrices of 8 rows x 16 bytes (rows 16 bytes apart), lbo =
   byte distance between core matrices adjacent in K, sbo = between core matrices adjacent in M/N. */
__device__ __forceinline__ uint64_t desc_k_noswz(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
         ((uint64_t)1u << 46);
}

__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

/* D[tmem] (+)= A[smem] * B[smem]^T, s8 x s8 -> s32, issued by one thread. */
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
    "{\n\t.reg .pred p;\n\t"
    "setp.ne.b32 p, %4, 0;\n\t"
    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
    "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
    : "memory");
}

/* Arrives (once) on the mbarrier when all tcgen05.mma issued so far by this thread are done. */
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

/* 32 consecutive 32-bit columns of this thread's tensor-memory lane (warp w reads lanes
   32*(w%4) .. 32*(w%4)+31). */
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
    "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
    "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
      "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
      "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
      "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
    : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]),
      "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
    : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

/* Stores 32 consecutive 32-bit columns of this thread's tensor-memory lane (same lane rule as the
   loads); tmem_st_wait makes them complete before this thread's later tensor-memory accesses. */
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&v)[32]) {
  asm volatile(
    "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
    "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, "
    "%17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
    "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]), "r"(v[10]),
    "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]), "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]),
    "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]), "r"(v[26]), "r"(v[27]), "r"(v[28]), "r"(v[29]), "r"(v[30]),
    "r"(v[31])
    : "memory");
}
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

}  // namespace xs_tc
