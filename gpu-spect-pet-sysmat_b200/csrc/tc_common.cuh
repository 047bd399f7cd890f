// tcgen05 building blocks shared by the BF16 GEMMs (sm_100a): shared-memory
// matrix descriptors for the K-major no-swizzle core-matrix layout, the
// kind::f16 instruction descriptor, mbarriers with bounded waits, MMA issue
// and commit, TMEM allocation and loads.
//
// Operand tile layout in shared memory (K-major, no swizzle): a tile of R rows
// x 64 k (bf16) is stored as 8 x 8 core matrices of 8 rows x 16 bytes; core
// matrix (row / 8, k / 8) starts at ((row / 8) * 8 + k / 8) * 128 bytes, so the
// leading byte offset (next core matrix along k) is 128 and the stride byte
// offset (next 8 rows) is 1024.
#pragma once

#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace smb {
namespace tc {

constexpr int kTileM = 128;
constexpr int kChunkK = 64;
constexpr uint32_t kWaitLimit = 1u << 26;   // mbarrier polls before giving up (seconds at worst)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (tcgen05), no swizzle, K-major.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);              // start address, bits [0, 14)
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;   // leading byte offset, bits [16, 30)
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;   // stride byte offset, bits [32, 46)
    d |= (uint64_t)1 << 46;                              // descriptor version (sm_100)
    return d;                                            // base offset 0, layout type 0 = no swizzle
}

// Instruction descriptor: kind::f16, A = B = BF16, D = F32, both K-major, M = 128.
__host__ __device__ constexpr uint32_t instr_desc(int n_tile) {
    return (1u << 4)                                     // D format F32
           | (1u << 7)                                   // A format BF16
           | (1u << 10)                                  // B format BF16
           | ((uint32_t)(n_tile >> 3) << 17)             // N / 8
           | ((uint32_t)(kTileM >> 4) << 24);            // M / 16
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Polls until the phase completes or `limit` polls have failed (false).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t phase, uint32_t limit = kWaitLimit) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Element offset of (row, k) inside a staged tile (k < 64).
__device__ __forceinline__ int core_offset(int row, int kc) {
    return (((row >> 3) * 8 + kc) * 8 + (row & 7)) * 8;
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t tmem, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols));
}

// Four 128 x n_tile x 16 MMAs over one staged 64-k chunk, then a commit to `bar`.
// Called by one thread.
__device__ __forceinline__ void mma_chunk(uint32_t tmem, const __nv_bfloat16* a, const __nv_bfloat16* b,
                                          uint32_t idesc, bool first, unsigned long long* bar) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t a_addr = smem_u32(a), b_addr = smem_u32(b);
#pragma unroll
    for (int j = 0; j < kChunkK / 16; ++j) {
        const uint64_t da = smem_desc(a_addr + 256u * j, 128u, 1024u);
        const uint64_t db = smem_desc(b_addr + 256u * j, 128u, 1024u);
        const uint32_t accumulate = (!first || j > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            :
            : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 16 consecutive fp32 accumulator columns of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_load16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int e = 0; e < 16; ++e) v[e] = __uint_as_float(r[e]);
}

}  // namespace tc
}  // namespace smb
