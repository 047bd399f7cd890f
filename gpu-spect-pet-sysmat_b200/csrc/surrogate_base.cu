// Physics baseline of the scatter surrogate and the verification helpers (sm_100a).
//
// Crystal scatter of detector d from voxel v is sum_s PE[s][v] K_v[s][d], where
// K_v is the per-unit-PE transfer of source s to detector d for photons
// arriving from v (the scatter terms of the exact kernel; K depends on v only
// through the arrival direction).  The baseline evaluates K at a grid of
// anchors (per anchor and source, at the PE-weighted centroid of the source's
// voxels under the anchor's trilinear weight) and interpolates trilinearly in
// v:  B[d][v] = sum_a w_a(v) sum_s K_a[d][s] PE[s][v].
// Per cell (the voxels between 8 neighbouring anchors) that is one GEMM with
// the corner anchors concatenated along k: A = [K_a0 | ... | K_a7] (rows d),
// B = [w_a0(v) PE[:, v]; ...; w_a7(v) PE[:, v]], run on the tcgen05 tensor
// cores with the weight folded into the B staging.
#include <algorithm>
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "surrogate.h"
#include "tc_common.cuh"

namespace smb {
namespace {

using namespace tc;

constexpr int kBaseThreads = 128;
constexpr int kBaseTileN = 256;

// ---- PE transpose ---------------------------------------------------------------------
__global__ void pe_transpose_kernel(const float* __restrict__ pe, long long ld_pe, int N, long long V,
                                    __nv_bfloat16* __restrict__ pet) {
    __shared__ float tile[32][33];
    const long long v0 = (long long)blockIdx.x * 32;
    const int s0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int s = s0 + i;
        const long long v = v0 + threadIdx.x;
        tile[i][threadIdx.x] = (s < N && v < V) ? pe[(long long)s * ld_pe + v] : 0.0f;
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const long long v = v0 + i;
        const int s = s0 + threadIdx.x;
        if (v < V && s < N) pet[v * N + s] = __float2bfloat16(tile[threadIdx.x][i]);
    }
}

// ---- anchor centroids ------------------------------------------------------------------
// One block per source, one warp per anchor at a time: the warp walks the
// anchor's support box (coordinates where it carries weight) in a fixed order
// and reduces with shuffles, so the result does not depend on scheduling.
// Weight of anchor i at coordinate x of an axis: 1 - t (lo == i, two anchors),
// t (hi == i), 1 (lo == hi == i), else 0.
__device__ __forceinline__ float axis_weight(int i, int lo, int hi, float t) {
    if (lo == i) return hi == i ? 1.0f : 1.0f - t;
    return hi == i ? t : 0.0f;
}

__global__ void anchor_centroid_kernel(const float* __restrict__ pe, long long ld_pe, int N, int nx, int ny, int nz,
                                       const int* __restrict__ lo, const int* __restrict__ hi,
                                       const float* __restrict__ t, const int* __restrict__ box, int kx, int ky, int kz,
                                       float4* __restrict__ vbar) {
    const int A = kx * ky * kz;
    const int s = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, n_warps = blockDim.x >> 5;
    const float* row = pe + (long long)s * ld_pe;
    // box: per axis and anchor, [first, count] of the support (x: 0..kx-1, then y, then z)
    for (int a = warp; a < A; a += n_warps) {
        const int ix = a / (ky * kz), iy = (a / kz) % ky, iz = a % kz;
        const int x0 = box[2 * ix], cx = box[2 * ix + 1];
        const int y0 = box[2 * (kx + iy)], cy = box[2 * (kx + iy) + 1];
        const int z0 = box[2 * (kx + ky + iz)], cz = box[2 * (kx + ky + iz) + 1];
        const int n = cx * cy * cz;
        float sx = 0.f, sy = 0.f, sz = 0.f, sw = 0.f;
        for (int q = lane; q < n; q += 32) {
            const int x = x0 + q % cx, y = y0 + (q / cx) % cy, z = z0 + q / (cx * cy);
            const float p = row[(long long)x + (long long)nx * (y + (long long)ny * z)];
            if (p == 0.0f) continue;
            const float w = axis_weight(ix, lo[x], hi[x], t[x]) * axis_weight(iy, lo[nx + y], hi[nx + y], t[nx + y]) *
                            axis_weight(iz, lo[nx + ny + z], hi[nx + ny + z], t[nx + ny + z]) * p;
            sx += w * (float)x;
            sy += w * (float)y;
            sz += w * (float)z;
            sw += w;
        }
        for (int o = 16; o > 0; o >>= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
            sz += __shfl_xor_sync(0xffffffffu, sz, o);
            sw += __shfl_xor_sync(0xffffffffu, sw, o);
        }
        if (lane == 0)
            vbar[(long long)a * N + s] =
                sw > 0.0f ? make_float4(sx / sw, sy / sw, sz / sw, 1.0f) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// ---- baseline GEMM ------------------------------------------------------------------------
struct __align__(128) BaseSmem {
    __nv_bfloat16 a[2][kTileM * kChunkK];        // 2 x 16 KB
    __nv_bfloat16 b[2][kBaseTileN * kChunkK];    // 2 x 32 KB
    float w[8][kBaseTileN];                      // per segment, per column: trilinear weight
    int vox[kBaseTileN];                         // voxel index per column (-1: none)
    unsigned long long mbar[2];
    uint32_t tmem_base;
    int failed;
};

__global__ void __launch_bounds__(kBaseThreads) baseline_gemm_kernel(
    const __nv_bfloat16* __restrict__ K, const __nv_bfloat16* __restrict__ pet, int N, int NX, int NY,
    const BaseCell* __restrict__ cells, const BaseItem* __restrict__ items, const float* __restrict__ tx,
    const float* __restrict__ ty, const float* __restrict__ tz, const int* __restrict__ row_map, float* __restrict__ dst,
    long long ld, int* __restrict__ error) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    BaseSmem& S = *reinterpret_cast<BaseSmem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kTileM;
    const BaseItem it = items[blockIdx.y];
    const BaseCell C = cells[it.cell];
    const int n_cell = C.nx * C.ny * C.nz;

    for (int j = tid; j < kBaseTileN; j += kBaseThreads) {
        const int l = it.n0 + j;
        int v = -1;
        float tt[3] = {0.f, 0.f, 0.f};
        if (l < n_cell) {
            const int lx = l % C.nx, ly = (l / C.nx) % C.ny, lz = l / (C.nx * C.ny);
            const int x = C.x0 + lx, y = C.y0 + ly, z = C.z0 + lz;
            v = x + NX * (y + NY * z);
            tt[0] = tx[x];
            tt[1] = ty[y];
            tt[2] = tz[z];
        }
        S.vox[j] = v;
        for (int sg = 0; sg < 8; ++sg) {
            float w = 0.0f;
            if (sg < C.n_seg && v >= 0) {
                const int sd = C.side[sg];
                w = 1.0f;
#pragma unroll
                for (int ax = 0; ax < 3; ++ax) {
                    const int bit = (sd >> ax) & 1, dual = (sd >> (ax + 4)) & 1;   // dual: the axis has two anchors
                    if (dual) w *= bit ? tt[ax] : 1.0f - tt[ax];
                }
            }
            S.w[sg][j] = w;
        }
    }
    if (tid == 0) {
        mbar_init(&S.mbar[0], 1);
        mbar_init(&S.mbar[1], 1);
        S.failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tmem_alloc(&S.tmem_base, (uint32_t)kBaseTileN);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = S.tmem_base;
    const uint32_t idesc = instr_desc(kBaseTileN);
    const int kchunks = (N + kChunkK - 1) / kChunkK;
    const int total = C.n_seg * kchunks;
    const bool vec_ok = (N % 8) == 0;

    bool ok = true;
    for (int c = 0; c < total && ok; ++c) {
        const int buf = c & 1;
        if (c >= 2) {
            if (!mbar_wait(&S.mbar[buf], (uint32_t)(((c - 2) >> 1) & 1))) S.failed = 1;
            __syncthreads();
            if (S.failed) { ok = false; break; }
        }
        const int sg = c / kchunks, k0 = (c - sg * kchunks) * kChunkK;
        const __nv_bfloat16* Ka = K + (long long)C.anchor[sg] * N * N;
        // A: detectors m0.. x sources k0..k0+63 of anchor sg
        for (int q = tid; q < kTileM * 8; q += kBaseThreads) {
            const int r = q >> 3, kc = q & 7;
            const int d = m0 + r, k = k0 + kc * 8;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (d < N) {
                const __nv_bfloat16* p = Ka + (long long)d * N + k;
                if (vec_ok && k + 8 <= N) val = *reinterpret_cast<const uint4*>(p);
                else {
                    __nv_bfloat16 tmp[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e) tmp[e] = (k + e < N) ? p[e] : __float2bfloat16(0.0f);
                    val = *reinterpret_cast<const uint4*>(tmp);
                }
            }
            *reinterpret_cast<uint4*>(S.a[buf] + core_offset(r, kc)) = val;
        }
        // B: columns (voxels) x sources, scaled by the segment's weight
        for (int q = tid; q < kBaseTileN * 8; q += kBaseThreads) {
            const int r = q >> 3, kc = q & 7;
            const int v = S.vox[r], k = k0 + kc * 8;
            const float w = S.w[sg][r];
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (v >= 0 && w != 0.0f) {
                const __nv_bfloat16* p = pet + (long long)v * N + k;
                __nv_bfloat16 tmp[8];
                if (vec_ok && k + 8 <= N) *reinterpret_cast<uint4*>(tmp) = *reinterpret_cast<const uint4*>(p);
                else {
#pragma unroll
                    for (int e = 0; e < 8; ++e) tmp[e] = (k + e < N) ? p[e] : __float2bfloat16(0.0f);
                }
                if (w != 1.0f) {
#pragma unroll
                    for (int e = 0; e < 8; ++e) tmp[e] = __float2bfloat16(__bfloat162float(tmp[e]) * w);
                }
                val = *reinterpret_cast<const uint4*>(tmp);
            }
            *reinterpret_cast<uint4*>(S.b[buf] + core_offset(r, kc)) = val;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) mma_chunk(tmem, S.a[buf], S.b[buf], idesc, c == 0, &S.mbar[buf]);
    }
    // the last one or two commits have not been waited for yet, in order per barrier
    if (ok) {
        if (total >= 2 && !mbar_wait(&S.mbar[(total - 2) & 1], (uint32_t)(((total - 2) >> 1) & 1))) ok = false;
        if (ok && !mbar_wait(&S.mbar[(total - 1) & 1], (uint32_t)(((total - 1) >> 1) & 1))) ok = false;
    }
    if (!ok) S.failed = 1;
    __syncthreads();
    ok = !S.failed;
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ok) {
        const int m = m0 + warp * 32 + lane;
        const int d = (m < N && row_map) ? row_map[m] : m;
        for (int c0 = 0; c0 < kBaseTileN; c0 += 16) {
            float r[16];
            tmem_load16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
            if (m < N) {
                float* out = dst + (long long)d * ld;
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const int v = S.vox[c0 + e];
                    if (v >= 0) out[v] = r[e];
                }
            }
        }
    } else if (tid == 0 && error) {
        atomicOr(error, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, (uint32_t)kBaseTileN);
}

// ---- column gather / scatter, per-row error ----------------------------------------------
// Voxel index of column j (= c * ny + y) of a y-column list.
__device__ __forceinline__ long long column_voxel(const int2* cols, long long j, int nx, int ny) {
    const int c = (int)(j / ny), y = (int)(j - (long long)c * ny);
    const int2 xz = cols[c];
    return (long long)xz.x + (long long)nx * (y + (long long)ny * xz.y);
}

// out[r][j] = full[r][voxel of column j]
__global__ void gather_columns_kernel(const float* __restrict__ full, long long ld_full, int N, const int2* __restrict__ cols,
                                      int n_cols, int nx, int ny, float* __restrict__ out, long long ld_out) {
    const long long W = (long long)n_cols * ny;
    const long long total = (long long)N * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / W);
        const long long j = i - (long long)r * W;
        out[(long long)r * ld_out + j] = full[(long long)r * ld_full + column_voxel(cols, j, nx, ny)];
    }
}

// full[r][voxel of column j] = sub[r][j]
__global__ void scatter_columns_kernel(const float* __restrict__ sub, long long ld_sub, int N, const int2* __restrict__ cols,
                                       int n_cols, int nx, int ny, float* __restrict__ full, long long ld_full) {
    const long long W = (long long)n_cols * ny;
    const long long total = (long long)N * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / W);
        const long long j = i - (long long)r * W;
        full[(long long)r * ld_full + column_voxel(cols, j, nx, ny)] = sub[(long long)r * ld_sub + j];
    }
}

__global__ void row_error_kernel(const float* __restrict__ pred, long long ld_pred, const float* __restrict__ ref,
                                 long long ld_ref, int n, double* __restrict__ err2, double* __restrict__ norm2) {
    __shared__ double pe[8], pn[8];
    const int r = blockIdx.x;
    double e = 0.0, q = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double a = pred[(long long)r * ld_pred + j], b = ref[(long long)r * ld_ref + j];
        e += (a - b) * (a - b);
        q += b * b;
    }
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, o);
        q += __shfl_xor_sync(0xffffffffu, q, o);
    }
    if ((threadIdx.x & 31) == 0) {
        pe[threadIdx.x >> 5] = e;
        pn[threadIdx.x >> 5] = q;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double se = 0.0, sq = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            se += pe[w];
            sq += pn[w];
        }
        err2[r] = se;
        norm2[r] = sq;
    }
}

// rho = log(Y / B), wgt = Y^2 / (norm2 / n) where Y > 0 and B > 0, else 0
__global__ void prep_targets_kernel(const float* __restrict__ Y, const float* __restrict__ Bm, long long ld, int N, int n,
                                    const double* __restrict__ norm2, float* __restrict__ rho, float* __restrict__ wgt,
                                    long long ld_out) {
    const long long total = (long long)N * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int d = (int)(i / n), j = (int)(i - (long long)d * n);
        const float y = Y[(long long)d * ld + j], b = Bm[(long long)d * ld + j];
        const double ms = norm2[d] / (double)n;
        const bool ok = y > 0.0f && b > 0.0f && ms > 0.0;
        rho[(long long)d * ld_out + j] = ok ? logf(y / b) : 0.0f;
        wgt[(long long)d * ld_out + j] = ok ? (float)((double)y * (double)y / ms) : 0.0f;
    }
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

// col[j] = fit[h(seed, step, j) mod n_fit], vox[j] = voxel of that column
__global__ void sample_batch_kernel(unsigned long long seed, int step, int B, const int* __restrict__ fit, int n_fit,
                                    const int* __restrict__ col_vox, int* __restrict__ col, int* __restrict__ vox) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= B) return;
    const unsigned long long h = mix64(seed ^ mix64(((unsigned long long)step << 32) | (unsigned)j));
    const int c = fit[(int)(h % (unsigned long long)n_fit)];
    col[j] = c;
    vox[j] = col_vox[c];
}

// out[d][j] = in[d][idx[j]]
__global__ void gather_idx_kernel(const float* __restrict__ in, long long ld_in, int N, const int* __restrict__ idx, int n,
                                  float* __restrict__ out, long long ld_out) {
    const long long total = (long long)N * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int d = (int)(i / n), j = (int)(i - (long long)d * n);
        out[(long long)d * ld_out + j] = in[(long long)d * ld_in + idx[j]];
    }
}

}  // namespace

AxisTable make_axis(int n, int k) {
    AxisTable A;
    A.k = k;
    A.lo.resize(n);
    A.hi.resize(n);
    A.t.resize(n);
    A.slab.resize(n);
    for (int x = 0; x < n; ++x) {
        // slab j: number of centres strictly below x (centres c_i = (i + 0.5) n / k - 0.5)
        int j = 0;
        while (j < k && ((double)j + 0.5) * n / k - 0.5 < (double)x) ++j;
        const int lo = std::max(j - 1, 0), hi = std::min(j, k - 1);
        A.lo[x] = lo;
        A.hi[x] = hi;
        A.slab[x] = j;
        if (lo == hi) A.t[x] = 0.0f;
        else {
            const double cl = ((double)lo + 0.5) * n / k - 0.5, ch = ((double)hi + 0.5) * n / k - 0.5;
            A.t[x] = (float)(((double)x - cl) / (ch - cl));
        }
    }
    A.first.assign(k, -1);
    A.count.assign(k, 0);
    for (int x = 0; x < n; ++x)
        for (int i : {A.lo[x], A.hi[x]}) {
            if (A.first[i] < 0) A.first[i] = x;
            A.count[i] = x - A.first[i] + 1;
        }
    for (int i = 0; i < k; ++i)
        if (A.first[i] < 0) A.first[i] = 0;
    return A;
}

cudaError_t launch_pe_transpose(const float* pe, int64_t ld_pe, int N, int64_t V, __nv_bfloat16* pet, cudaStream_t s) {
    dim3 grid((unsigned)((V + 31) / 32), (unsigned)((N + 31) / 32));
    pe_transpose_kernel<<<grid, dim3(32, 8), 0, s>>>(pe, ld_pe, N, V, pet);
    return cudaGetLastError();
}

cudaError_t launch_anchor_centroids(const float* pe, int64_t ld_pe, int N, int nx, int ny, int nz, const int* d_lo,
                                    const int* d_hi, const float* d_t, const int* d_box, int kx, int ky, int kz,
                                    float4* vbar, cudaStream_t s) {
    anchor_centroid_kernel<<<N, 256, 0, s>>>(pe, ld_pe, N, nx, ny, nz, d_lo, d_hi, d_t, d_box, kx, ky, kz, vbar);
    return cudaGetLastError();
}

cudaError_t launch_baseline_gemm(const __nv_bfloat16* K, const __nv_bfloat16* pet, int N, int nx, int ny,
                                 const BaseCell* cells, const BaseItem* items, int n_items, const float* tx,
                                 const float* ty, const float* tz, const int* row_map, float* dst, int64_t ld,
                                 int* error, cudaStream_t s) {
    if (n_items <= 0 || N <= 0) return cudaSuccess;
    if (n_items > 65535) return cudaErrorInvalidConfiguration;
    const size_t smem = sizeof(BaseSmem);
    cudaError_t e = cudaFuncSetAttribute(baseline_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((N + kTileM - 1) / kTileM, n_items);
    baseline_gemm_kernel<<<grid, kBaseThreads, smem, s>>>(K, pet, N, nx, ny, cells, items, tx, ty, tz, row_map, dst, ld,
                                                          error);
    return cudaGetLastError();
}

cudaError_t launch_gather_columns(const float* full, int64_t ld_full, int N, const int2* cols, int n_cols, int nx,
                                  int ny, float* out, int64_t ld_out, cudaStream_t s) {
    const long long total = (long long)N * n_cols * ny;
    if (total <= 0) return cudaSuccess;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 32);
    gather_columns_kernel<<<blocks, 256, 0, s>>>(full, ld_full, N, cols, n_cols, nx, ny, out, ld_out);
    return cudaGetLastError();
}

cudaError_t launch_scatter_columns(const float* sub, int64_t ld_sub, int N, const int2* cols, int n_cols, int nx,
                                   int ny, float* full, int64_t ld_full, cudaStream_t s) {
    const long long total = (long long)N * n_cols * ny;
    if (total <= 0) return cudaSuccess;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 32);
    scatter_columns_kernel<<<blocks, 256, 0, s>>>(sub, ld_sub, N, cols, n_cols, nx, ny, full, ld_full);
    return cudaGetLastError();
}

cudaError_t launch_row_error(const float* pred, int64_t ld_pred, const float* ref, int64_t ld_ref, int N, int n,
                             double* err2, double* norm2, cudaStream_t s) {
    if (N <= 0) return cudaSuccess;
    row_error_kernel<<<N, 256, 0, s>>>(pred, ld_pred, ref, ld_ref, n, err2, norm2);
    return cudaGetLastError();
}

cudaError_t launch_prep_targets(const float* Y, const float* Bm, int64_t ld, int N, int n, const double* norm2, float* rho,
                                float* wgt, int64_t ld_out, cudaStream_t s) {
    const long long total = (long long)N * n;
    if (total <= 0) return cudaSuccess;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 32);
    prep_targets_kernel<<<blocks, 256, 0, s>>>(Y, Bm, ld, N, n, norm2, rho, wgt, ld_out);
    return cudaGetLastError();
}

cudaError_t launch_sample_batch(uint64_t seed, int step, int B, const int* fit, int n_fit, const int* col_vox, int* col,
                                int* vox, cudaStream_t s) {
    if (B <= 0 || n_fit <= 0) return cudaErrorInvalidValue;
    sample_batch_kernel<<<(B + 255) / 256, 256, 0, s>>>(seed, step, B, fit, n_fit, col_vox, col, vox);
    return cudaGetLastError();
}

cudaError_t launch_gather_idx(const float* in, int64_t ld_in, int N, const int* idx, int n, float* out, int64_t ld_out,
                              cudaStream_t s) {
    const long long total = (long long)N * n;
    if (total <= 0) return cudaSuccess;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 32);
    gather_idx_kernel<<<blocks, 256, 0, s>>>(in, ld_in, N, idx, n, out, ld_out);
    return cudaGetLastError();
}

}  // namespace smb
