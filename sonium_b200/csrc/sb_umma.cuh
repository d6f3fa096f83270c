// sm_100a building blocks for the tensor-core block product (internal): mbarriers, TMA tile
// loads, tcgen05 tensor-memory allocation / MMA / commit / loads, and the UMMA descriptors.
//
// Descriptor encodings follow the PTX ISA (tcgen05 "matrix descriptor" and "instruction
// descriptor" tables); the bit positions are the ones CUTLASS's cute::UMMA::SmemDescriptor and
// cute::UMMA::InstrDescriptor name (cute/arch/mma_sm100_desc.hpp), cross-checked by a CPU test.
// Every wait here is bounded: after kSpinLimit polls the caller gets `false` and must abandon
// the pipeline through its error path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sb {
namespace umma {

constexpr uint32_t kSpinLimit = 1u << 22;

// ---- descriptors (host and device) ----
// Shared-memory matrix descriptor for a K-major operand tile stored as the 128-byte swizzle of a
// TMA SWIZZLE_128B box: rows of 64 bf16 (128 B), 8-row groups 1024 B apart. Start address and
// offsets are in 16-byte units; version 1 (tcgen05); layout type 2 = SWIZZLE_128B.
__host__ __device__ constexpr uint64_t smem_desc_k_sw128(uint32_t smem_addr) {
    return (uint64_t)((smem_addr >> 4) & 0x3FFFu)      // start address, bits [0,14)
           | ((uint64_t)1u << 16)                       // leading byte offset (unused with swizzle), [16,30)
           | ((uint64_t)(1024u >> 4) << 32)             // stride byte offset: 8-row group pitch, [32,46)
           | ((uint64_t)1u << 46)                       // descriptor version, [46,48)
           | ((uint64_t)2u << 61);                      // layout type SWIZZLE_128B, [61,64)
}

// The same for a TMA SWIZZLE_64B box: rows of 32 bf16 (64 B), 8-row groups 512 B apart; layout
// type 4 = SWIZZLE_64B.
__host__ __device__ constexpr uint64_t smem_desc_k_sw64(uint32_t smem_addr) {
    return (uint64_t)((smem_addr >> 4) & 0x3FFFu)      // start address, bits [0,14)
           | ((uint64_t)1u << 16)                       // leading byte offset (unused with swizzle), [16,30)
           | ((uint64_t)(512u >> 4) << 32)              // stride byte offset: 8-row group pitch, [32,46)
           | ((uint64_t)1u << 46)                       // descriptor version, [46,48)
           | ((uint64_t)4u << 61);                      // layout type SWIZZLE_64B, [61,64)
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 accumulator, both K-major, M x N.
__host__ __device__ constexpr uint32_t instr_desc_bf16_f32(int m, int n) {
    return (1u << 4)                    // D format F32, bits [4,6)
           | (1u << 7)                  // A format BF16, bits [7,10)
           | (1u << 10)                 // B format BF16, bits [10,13)
           | ((uint32_t)(n >> 3) << 17) // N / 8, bits [17,23)
           | ((uint32_t)(m >> 4) << 24);// M / 16, bits [24,29)
}

// Instruction descriptor of kind::i8 with signed 8-bit A and B, S32 accumulator, both K-major.
__host__ __device__ constexpr uint32_t instr_desc_s8_s32(int m, int n) {
    return (2u << 4)                    // D format S32, bits [4,6)
           | (1u << 7)                  // A format signed 8-bit, bits [7,10)
           | (1u << 10)                 // B format signed 8-bit, bits [10,13)
           | ((uint32_t)(n >> 3) << 17) // N / 8, bits [17,23)
           | ((uint32_t)(m >> 4) << 24);// M / 16, bits [24,29)
}

#if defined(__CUDA_ARCH__)
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarriers ----
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// One arrival (no transaction bytes).
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
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
// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < kSpinLimit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// ---- TMA ----
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void* tmap, uint32_t bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(dst), "l"(tmap), "r"(bar), "r"(x), "r"(y)
        : "memory");
}
__device__ __forceinline__ void prefetch_tmap(const void* tmap) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(tmap) : "memory");
}

// ---- tensor memory ----
// Allocation by one full warp; the TMEM address is written to shared memory at `dst`.
__device__ __forceinline__ void tmem_alloc(uint32_t dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T with signed 8-bit operands and exact S32 accumulation.
__device__ __forceinline__ void mma_s8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// The mbarrier gets one arrival when every MMA issued so far by this thread has completed.
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// 32 consecutive 32-bit columns of this warp's 32 TMEM lanes (one lane per thread); the load and
// its completion wait are one asm statement, so no use of the registers can move above the wait.
__device__ __forceinline__ void tmem_ld32_raw(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}
// The same, as FP32 values.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    tmem_ld32_raw(taddr, r);
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
#endif

}  // namespace umma
}  // namespace sb
