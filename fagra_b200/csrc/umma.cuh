// Fifth-generation tensor-core (tcgen05) building blocks for sm_100a: shared
// memory matrix descriptors for the 128-byte-swizzled K-major operand layout,
// the kind::f16 instruction descriptor, MMA issue and commit, tensor-memory
// allocation and loads, and a bounded mbarrier wait. The encodings are the
// ones the PTX ISA defines for tcgen05 (matrix descriptor: start address,
// leading / stride byte offsets, version 1, layout type; instruction
// descriptor: D / A / B formats, majors, N >> 3, M >> 4).
#pragma once
#include <cstdint>

namespace fg {

__device__ __forceinline__ uint32_t umma_smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Operand tile layout (K-major, 128-byte swizzle): rows of 64 bf16 (128 B),
// 8-row atoms of 1024 B; the 16-byte chunk j of row r sits at chunk j ^ (r % 8).
// The tile base must be 1024-byte aligned.
__device__ __forceinline__ uint32_t umma_sw128_offset(int row, int k) {
  return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + ((((k >> 3) ^ (row & 7)) & 7) << 4) + (k & 7) * 2);
}

// Matrix descriptor of a SW128 K-major tile starting at shared address saddr
// (advance saddr by 32 bytes per 16-element K step inside the 128-byte row):
// start >> 4 in bits 0-13, leading byte offset 16 B (unused by this layout),
// stride byte offset 1024 B (between 8-row atoms), version 1, layout 2 = SW128.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// kind::f16 instruction descriptor: D f32, A and B bf16, both K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T, issued by one thread.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// The mbarrier at shared address mbar receives one arrival once every MMA this
// thread issued so far has completed.
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

// Tensor memory: allocation by one whole warp (the base address is written to
// shared memory), permit release, deallocation by the allocating warp.
__device__ __forceinline__ void tmem_alloc(uint32_t dst_saddr, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_saddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tcgen05_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tcgen05_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 32 consecutive 32-bit columns of this warp's 32 lanes (lane = thread).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Generic-proxy shared-memory writes made visible to the tensor core.
__device__ __forceinline__ void umma_fence_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void umma_mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void umma_mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool umma_mbar_test(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait until the phase of the given parity has completed: non-blocking polls
// with a growing sleep, at most `limit` of them; false (and *err = 1) when the
// limit ran out.
__device__ __forceinline__ bool umma_wait(uint32_t mbar, uint32_t parity, int* err, uint32_t limit = 1u << 22) {
  uint32_t ns = 32;
  for (uint32_t i = 0; i < limit; ++i) {
    if (umma_mbar_test(mbar, parity)) return true;
    if (i > 16) {
      __nanosleep(ns);
      if (ns < 1024) ns <<= 1;
    }
  }
  if (err) atomicExch(err, 1);
  return false;
}

}  // namespace fg
