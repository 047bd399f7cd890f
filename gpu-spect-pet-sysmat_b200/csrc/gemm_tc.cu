// BF16 GEMM on the sm_100a tensor cores (tcgen05.mma, accumulators in TMEM),
// for the scatter surrogate: C[M x N] (fp32) = alpha_row[m] * sum_k A[m][k] B[n][k]
// (+ bias[n]) (+ C when accumulating).
//
// A and B are bf16 with arbitrary strides: A[m][k] at a[m * a_ms + k * a_ks],
// B[n][k] at b[n * b_ns + k * b_ks].  When the K stride is 1 (K-major, the
// layout the MMA reads) eight consecutive k load as one 16-byte vector;
// otherwise they are gathered.
//
// One CTA computes a 128 x n_tile block (n_tile 64, 128 or 256): per chunk of
// 64 k the 128 threads stage A (128 x 64) and B (n_tile x 64) into shared
// memory as 8 x 16-byte core matrices (K-major, no swizzle: core matrix
// (row / 8, k / 8) at ((row / 8) * 8 + k / 8) * 128 bytes, so the stride to the
// next core matrix along k is 128 bytes and along rows 1024 bytes), one
// elected thread issues four 128 x n_tile x 16 MMAs into the TMEM accumulator
// and commits them to an mbarrier, and all threads wait for it before the
// buffer is refilled.  The epilogue reads TMEM (warp w owns rows 32w..32w+31)
// and writes each thread's row segment as whole 32-byte sectors.
//
// Every wait is bounded: a wait that runs out sets the error word and the
// CTA skips its epilogue, frees its TMEM and returns.
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "gemm_tc.h"

namespace smb {
namespace {

constexpr int kTileM = 128;
constexpr int kChunkK = 64;
constexpr int kGemmThreads = 128;
constexpr uint32_t kWaitLimit = 1u << 26;   // mbarrier polls before giving up (seconds at worst)

struct __align__(128) GemmSmem {
    __nv_bfloat16 a[kTileM * kChunkK];       // 16 KB
    __nv_bfloat16 b[256 * kChunkK];          // 32 KB (n_tile <= 256)
    unsigned long long mbar;
    uint32_t tmem_base;
    int failed;
};

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

__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t phase) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
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

// Stages rows [r0, r0 + rows) x k [k0, k0 + 64) of a strided bf16 operand into
// the core-matrix layout; rows beyond `rows_total` and k beyond `k_total` are zero.
__device__ __forceinline__ void stage(__nv_bfloat16* dst, int n_rows, const __nv_bfloat16* src, long long rs,
                                      long long ks, int r0, int rows_total, int k0, int k_total) {
    const int vecs = n_rows * (kChunkK / 8);   // 16-byte vectors
    for (int v = threadIdx.x; v < vecs; v += kGemmThreads) {
        const int r = v >> 3, kc = v & 7;      // row, 8-k core column
        const int gr = r0 + r, gk = k0 + kc * 8;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        if (gr < rows_total) {
            const __nv_bfloat16* p = src + (long long)gr * rs + (long long)gk * ks;
            if (ks == 1 && gk + 8 <= k_total && ((reinterpret_cast<uintptr_t>(p) & 15u) == 0)) {
                val = *reinterpret_cast<const uint4*>(p);
            } else {
                __nv_bfloat16 t[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) t[e] = (gk + e < k_total) ? p[(long long)e * ks] : __float2bfloat16(0.0f);
                val = *reinterpret_cast<const uint4*>(t);
            }
        }
        const int off = (((r >> 3) * 8 + kc) * 8 + (r & 7)) * 8;   // elements
        *reinterpret_cast<uint4*>(dst + off) = val;
    }
}

__global__ void __launch_bounds__(kGemmThreads) gemm_bf16_tc_kernel(GemmArgs g) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    GemmSmem& S = *reinterpret_cast<GemmSmem*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * g.n_tile;

    if (threadIdx.x == 0) {
        mbar_init(&S.mbar, 1);
        S.failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                     "r"((uint32_t)g.n_tile));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = S.tmem_base;
    const uint32_t idesc = instr_desc(g.n_tile);

    uint32_t phase = 0;
    bool ok = true;
    const int n_chunks = (g.k + kChunkK - 1) / kChunkK;
    for (int c = 0; c < n_chunks && ok; ++c) {
        const int k0 = c * kChunkK;
        stage(S.a, kTileM, g.a, g.a_ms, g.a_ks, m0, g.m, k0, g.k);
        stage(S.b, g.n_tile, g.b, g.b_ns, g.b_ks, n0, g.n, k0, g.k);
        // generic-proxy stores must be visible to the tensor core's async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a_addr = smem_u32(S.a), b_addr = smem_u32(S.b);
#pragma unroll
            for (int j = 0; j < kChunkK / 16; ++j) {
                const uint64_t da = smem_desc(a_addr + 256u * j, 128u, 1024u);
                const uint64_t db = smem_desc(b_addr + 256u * j, 128u, 1024u);
                const uint32_t accumulate = (c > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    :
                    : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&S.mbar))
                         : "memory");
        }
        // the MMAs must finish reading the buffers before they are refilled
        if (!mbar_wait(&S.mbar, phase)) {
            S.failed = 1;
            ok = false;
        } else {
            phase ^= 1u;
        }
        __syncthreads();
        ok = !S.failed;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");

    if (ok) {
        // epilogue: warp w reads TMEM lanes 32w..32w+31 (rows), 16 columns per load
        const int row = m0 + warp * 32 + lane;
        const float scale = (g.row_scale && row < g.m) ? g.row_scale[row] : g.alpha;
        for (int c0 = 0; c0 < g.n_tile; c0 += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < g.m) {
                float* out = g.c + (long long)row * g.ldc + n0 + c0;
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const int col = n0 + c0 + e;
                    if (col < g.n) {
                        float v = __uint_as_float(r[e]) * scale;
                        if (g.bias) v += g.bias[col];
                        if (g.accumulate) v += out[e];
                        out[e] = v;
                    }
                }
            }
        }
    } else {
        // give MMAs still in flight one more bounded wait before the TMEM is released
        mbar_wait(&S.mbar, phase);
        if (threadIdx.x == 0 && g.error) atomicOr(g.error, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)g.n_tile));
    }
}

}  // namespace

cudaError_t gemm_bf16_tc(const GemmArgs& args, cudaStream_t stream) {
    if (args.m <= 0 || args.n <= 0 || args.k <= 0) return cudaSuccess;
    if (args.n_tile != 64 && args.n_tile != 128 && args.n_tile != 256) return cudaErrorInvalidValue;
    static unsigned long long done = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 64 || !((done >> dev) & 1ULL)) {
        e = cudaFuncSetAttribute(gemm_bf16_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GemmSmem));
        if (e != cudaSuccess) return e;
        if (dev < 64) done |= 1ULL << dev;
    }
    dim3 grid((args.m + kTileM - 1) / kTileM, (args.n + args.n_tile - 1) / args.n_tile);
    gemm_bf16_tc_kernel<<<grid, kGemmThreads, sizeof(GemmSmem), stream>>>(args);
    return cudaGetLastError();
}

}  // namespace smb
