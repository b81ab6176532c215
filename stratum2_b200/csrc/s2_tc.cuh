// Blackwell tensor-core primitives (sm_100a): tcgen05 MMA with accumulators in tensor memory
// (TMEM), shared-memory matrix descriptors, mbarrier completion and TMEM loads, written as inline
// PTX.  Field layouts follow the PTX ISA's tcgen05 chapter (instruction descriptor for .kind::f16,
// shared-memory descriptor with the sm_100 version bits) as CUTLASS's cute/arch/mma_sm100_desc.hpp
// also spells them out.
//
// Operand layout used throughout: K-major, no swizzle ("interleaved" core matrices).  A core matrix
// is 8 rows x 8 f16 (16 bytes per row, 128 bytes contiguous).  For an R x K operand the core matrix
// holding (row r, column k) starts at (r / 8) * SBO + (k / 8) * LBO with LBO = 128 bytes and
// SBO = K * 16 bytes, so every row's 8-element chunk is one 16-byte store.
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>

#include "s2_math.cuh"

namespace s2 {

S2D uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) of an R x K K-major core-matrix tile
S2D uint32_t kmaj_offset(uint32_t r, uint32_t k, uint32_t K) {
    return (r >> 3) * (K * 16u) + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor: start address, leading byte offset (between the two 8-column
// chunks of one K=16 step) and stride byte offset (between 8-row groups), all >> 4; version 1 at
// bits 46-47; base offset 0, legacy LBO mode, layout type 0 (no swizzle) at bits 61-63.
S2D uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    return d;
}

// Instruction descriptor of tcgen05.mma .kind::f16: D f32 (bits 4-5 = 1), A and B f16 (bits 7-9,
// 10-12 = 0), both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t idesc_f16_f32(uint32_t M, uint32_t N) {
    return (1u << 4) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

S2D void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// makes mbarrier initialisation visible to the async proxy (tensor-core commits)
S2D void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

S2D bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of `bar`: false after `limit` polls (each poll itself blocks
// for a hardware-defined time slice), so a lost arrival cannot hang the GPU.
constexpr uint32_t kMbarWaitLimit = 1u << 22;
S2D bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = kMbarWaitLimit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// TMEM allocation (one full warp): the base address is written to shared memory at `dst`.
S2D void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(ncols)
                 : "memory");
}
S2D void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory"); }
S2D void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

S2D void tc_fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
S2D void tc_fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// make this thread's generic-proxy shared-memory writes visible to the tensor core (async proxy)
S2D void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
S2D void umma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

// Arrive on `bar` once every tcgen05.mma issued so far by this thread has completed.
S2D void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// 16 consecutive f32 columns of this thread's TMEM lane (32x32b shape: warp w reads lanes
// 32*(w%4) .. +31, thread t of the warp lane 32*(w%4)+t).  The wait is inside the same asm block so
// the registers are valid when it returns.
S2D void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Issue the K/16 MMAs of D = A (128 x K) * B (N x K)^T for operands in the K-major layout above.
S2D void umma_gemm(uint32_t d_tmem, uint32_t a_saddr, uint32_t b_saddr, uint32_t K, uint32_t N, bool accumulate) {
    const uint32_t idesc = idesc_f16_f32(128, N);
    for (uint32_t s = 0; s < K / 16; ++s) {
        const uint64_t a = smem_desc(a_saddr + s * 256u, 128u, K * 16u);
        const uint64_t b = smem_desc(b_saddr + s * 256u, 128u, K * 16u);
        umma_f16(d_tmem, a, b, idesc, (accumulate || s > 0) ? 1u : 0u);
    }
}

}  // namespace s2
