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
// Every wait is bounded (wait_limit polls, set process-wide by
// sm_tc_wait_limit): a wait that runs out sets the error word and the CTA
// skips its epilogue; threads whose wait ran out then wait (bounded by the
// default limit) for their MMAs still in flight, and the CTA frees its TMEM
// and returns.
#include <atomic>
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "gemm_tc.h"
#include "tc_common.cuh"

namespace smb {
namespace {

using namespace tc;
constexpr int kGemmThreads = 128;

struct __align__(128) GemmSmem {
    __nv_bfloat16 a[kTileM * kChunkK];       // 16 KB
    __nv_bfloat16 b[256 * kChunkK];          // 32 KB (n_tile <= 256)
    unsigned long long mbar;
    uint32_t tmem_base;
    int failed;
};

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
        *reinterpret_cast<uint4*>(dst + core_offset(r, kc)) = val;
    }
}

__global__ void __launch_bounds__(kGemmThreads) gemm_bf16_tc_kernel(GemmArgs g, uint32_t wait_limit) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    GemmSmem& S = *reinterpret_cast<GemmSmem*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * g.n_tile;

    if (threadIdx.x == 0) {
        mbar_init(&S.mbar, 1);
        S.failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tmem_alloc(&S.tmem_base, (uint32_t)g.n_tile);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = S.tmem_base;
    const uint32_t idesc = instr_desc(g.n_tile);

    uint32_t phase = 0;
    bool ok = true;
    bool pending = false;   // this thread's wait ran out with MMAs possibly still in flight
    const int n_chunks = (g.k + kChunkK - 1) / kChunkK;
    for (int c = 0; c < n_chunks && ok; ++c) {
        const int k0 = c * kChunkK;
        stage(S.a, kTileM, g.a, g.a_ms, g.a_ks, m0, g.m, k0, g.k);
        stage(S.b, g.n_tile, g.b, g.b_ns, g.b_ks, n0, g.n, k0, g.k);
        // generic-proxy stores must be visible to the tensor core's async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) mma_chunk(tmem, S.a, S.b, idesc, c == 0, &S.mbar);
        // the MMAs must finish reading the buffers before they are refilled
        if (!mbar_wait(&S.mbar, phase, wait_limit)) {
            S.failed = 1;
            ok = false;
            pending = true;
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
            float r[16];
            tmem_load16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
            if (row < g.m) {
                float* out = g.c + (long long)row * g.ldc + n0 + c0;
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const int col = n0 + c0 + e;
                    if (col < g.n) {
                        if (g.epilogue == 1) {
                            out[e] = out[e] * __expf(r[e] * scale);
                        } else {
                            float v = r[e] * scale;
                            if (g.bias) v += g.bias[col];
                            if (g.accumulate) v += out[e];
                            out[e] = v;
                        }
                    }
                }
            }
        }
    } else {
        // MMAs still in flight get one more bounded wait before the TMEM is released
        if (pending) mbar_wait(&S.mbar, phase, kWaitLimit);
        if (threadIdx.x == 0 && g.error) atomicOr(g.error, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, (uint32_t)g.n_tile);
}

std::atomic<uint32_t> g_wait_limit{kWaitLimit};

}  // namespace

uint32_t gemm_wait_limit(int64_t polls) {
    const uint32_t prev = g_wait_limit.load();
    if (polls < 0) g_wait_limit.store(kWaitLimit);
    else g_wait_limit.store(polls > 0xffffffffLL ? 0xffffffffu : (uint32_t)polls);
    return prev;
}

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
    gemm_bf16_tc_kernel<<<grid, kGemmThreads, sizeof(GemmSmem), stream>>>(args, g_wait_limit.load());
    return cudaGetLastError();
}

}  // namespace smb
