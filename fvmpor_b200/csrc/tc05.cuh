// Thin wrappers over the sm_100a tensor-core instructions used by the
// per-node MLP: tcgen05 TMEM allocation, BF16 x BF16 -> FP32 MMA with
// operands in shared memory, commit to an mbarrier, TMEM loads, and the
// fences that order them.  Every wait is bounded and reports failure
// instead of spinning forever.
//
// Shared-memory operand layout (SWIZZLE_NONE, "interleaved" core matrices):
// an R x K BF16 tile is stored as 8-row x 8-element core matrices of 128 B
// (row r, column k at (r/8)*SBO + (k/8)*LBO + (r%8)*16 + (k%8)*2).  As a
// K-major operand the descriptor carries LBO = offset between K-adjacent
// core matrices and SBO = offset between M/N-adjacent ones; the same bytes
// read as an MN-major operand of the transposed matrix use the two offsets
// swapped.  Field positions follow the sm100 UMMA descriptor definitions
// (CUTLASS cute/arch/mma_sm100_desc.hpp: start address [0,14), LBO [16,30),
// SBO [32,46), version = 1 at [46,48), layout type [61,64) = 0 for
// SWIZZLE_NONE; instruction descriptor: C format [4,6), A/B format
// [7,10)/[10,13), A/B major [15]/[16], N>>3 at [17,23), M>>4 at [24,29)).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fvmb {
namespace tc05 {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version for sm100
    return d;                 // base offset 0, SWIZZLE_NONE
}

// kind::f16 instruction descriptor: BF16 A and B, FP32 accumulate
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N, bool a_mn_major, bool b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) |
           ((b_mn_major ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// called by all 32 threads of one warp; writes the TMEM base to *dst
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// D(tmem) (+)= A(smem) x B(smem)^T, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
    uint32_t acc = accumulate ? 1u : 0u;
    uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

// arrive on the mbarrier once all previously issued MMAs of this thread completed
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
        smem_u32(bar)));
}

// bounded wait for the given phase parity; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t max_iter = (1u << 26)) {
    uint32_t addr = smem_u32(bar);
    for (uint32_t it = 0; it < max_iter; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity));
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;"); }
// make generic-proxy shared-memory writes visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;"); }

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w may only
// address lanes 32w .. 32w+31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// byte offset of element (r, k) in an interleaved tile with K columns
__host__ __device__ constexpr uint32_t il_off(uint32_t r, uint32_t k, uint32_t K) {
    return (r >> 3) * (K * 16u) + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

} // namespace tc05
} // namespace fvmb
