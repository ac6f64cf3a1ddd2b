// tcgen05.cuh -- sm_100a primitives for the learned preconditioner's layer
// kernel, as inline PTX: mbarriers, bulk copies from global into this CTA's
// shared memory (no multicast), tensor-memory allocation, the fifth-generation
// tensor-core MMA (tcgen05.mma, kind::f16, one CTA) with shared-memory matrix
// descriptors, and tensor-memory loads.
//
// Operand layout (both A and B "K-major", BF16): a 64-element (128-byte) run
// of K per row, rows 128 bytes apart, 16-byte chunk c of row r stored at
// chunk position c ^ (r & 7) inside each 1024-byte group of eight rows (the
// 128-byte swizzle); a region starts on a 1024-byte boundary.  K = 128 is
// two such regions; an MMA step of K = 16 starts 32 bytes further into the
// rows.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ab2 {
namespace tc {

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// ---- mbarriers
__device__ __forceinline__ void mbar_init(unsigned a, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned a, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
// One arrival (release at CTA scope: this thread's earlier writes are
// visible to threads that observe the phase complete).
__device__ __forceinline__ void mbar_arrive(unsigned a) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned a, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(a), "r"(parity)
      : "memory");
  return done != 0;
}
// The same test, suspending the thread until the phase completes or about
// `ns` nanoseconds have passed: a waiting warp takes no issue slots.
__device__ __forceinline__ bool mbar_try_wait_sleep(unsigned a, unsigned parity, unsigned ns) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(a), "r"(parity), "r"(ns)
      : "memory");
  return done != 0;
}
// Waits for the phase of the given parity for at most `budget` clock cycles;
// false if it gave up (or, with an abort flag, when the flag became nonzero).
static __device__ __noinline__ bool mbar_wait(unsigned a, unsigned parity, long long budget,
                                             const volatile int* abort) {
  if (mbar_try_wait(a, parity)) return true;
  const long long t0 = clock64();
  for (;;) {
    if (mbar_try_wait_sleep(a, parity, 20000u)) return true;
    if (clock64() - t0 > budget || (abort && *abort)) return false;
  }
}

// ---- bulk copies (cp.async.bulk, no multicast): global -> this CTA's shared
// memory, completing `bytes` of transaction count on the mbarrier.  Both
// addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}
// Orders this thread's generic-proxy shared-memory writes before later
// async-proxy (tensor core, bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- tensor memory
// One full warp: allocates ncols (a power of two >= 32) columns x 128 lanes and
// writes the base address to shared memory at dst.
__device__ __forceinline__ void tmem_alloc(unsigned dst, unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---- MMA
// Shared-memory matrix descriptor of a K-major operand with the 128-byte
// swizzle: start address (bits 0-13, 16-byte units), leading-dimension byte
// offset (bits 16-29; not used by swizzled K-major operands whose MMA step
// stays inside one 128-byte run, set to one unit), stride-dimension byte
// offset 1024 (bits 32-45: from one group of eight rows to the next), the
// descriptor version 1 (bits 46-47), base offset 0 (bits 49-51: regions
// start on 1024-byte boundaries), swizzle mode 2 = 128 bytes (bits 61-63).
__device__ __forceinline__ uint64_t sdesc_sw128(unsigned saddr) {
  uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}
// Instruction descriptor of kind::f16: D in FP32 (bits 4-5 = 1), A and B in
// BF16 (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), no negation
// or sparsity, N / 8 in bits 17-22, M / 16 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// D[tmem] (+)= A[smem] B[smem]^T, one thread issues it.
__device__ __forceinline__ void mma_bf16_ss(unsigned d_tmem, uint64_t a, uint64_t b, uint32_t idesc, unsigned acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
// Arrives once on the mbarrier when every MMA this thread issued before it
// has completed (this CTA's own barrier, no multicast).
__device__ __forceinline__ void mma_commit(unsigned mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

// 32 lanes x 16 columns of 32-bit words: lane t of the warp gets tensor-memory
// lane (taddr >> 16) + t, columns (taddr & 0xffff) .. + 15.  A warp may read
// only its own quarter of the lanes (warp % 4).  The wait for the load is in
// the same statement, so no use of the registers can be scheduled before it.
__device__ __forceinline__ void tmem_ld16(unsigned taddr, float (&v)[16]) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 32 columns (as tmem_ld16).
__device__ __forceinline__ void tmem_ld32(unsigned taddr, float (&v)[32]) {
  unsigned r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace ab2
