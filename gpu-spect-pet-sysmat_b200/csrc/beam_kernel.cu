// Beam masks and multiplexing (MPXI) of a photoelectric sysmat, on the device.
//
// The reference computes these after the fact on the CPU, from a memory-mapped
// .sysmat file (PEGen_RayTracing_CircularHole/extract_beam_prop_masks.py:52-87,
// compute_mpxi_3d.py:45-52): per (rotation, crystal) row the beam mask is
// "entry > 0.05 * row max" (threshold 1.0 for an all-zero row), with the row's
// sum and mask size as beam properties; per rotation, MPXI(voxel) counts the
// rows whose mask holds the voxel.  Here the same quantities come from the
// sysmat where it already lives, in HBM:
//
//  beam_rows_kernel   one CTA per row (grid-stride): pass A reduces max (exact)
//                     and sum (double) with 128-bit loads; pass B re-reads the
//                     row (an L2 hit: a row is at most a few MB and the passes
//                     are back to back) and writes the int8 mask with 32-bit
//                     stores and counts it.  The threshold is the product
//                     frac * max rounded to single precision, as numpy forms
//                     it for a float32 row and a Python float.
//  beam_mpxi_kernel   4 voxels per thread, rows split over gridDim.y; counts
//                     in registers, read from the mask when it was written (1
//                     byte per entry) or else from the sysmat and the row
//                     thresholds; one integer atomicAdd per (thread, voxel) at
//                     the end, so the result is exact and order independent.
//
// Both are HBM-bound streaming kernels: algorithmic traffic is 4 bytes per
// entry read by pass A, 1 byte per entry of mask written and read again (or 4
// bytes of sysmat re-read when no mask is kept).
#include <cstdint>

#include <cuda_runtime.h>

#include "common.h"

namespace smb {
namespace {

constexpr int kBeamThreads = 256;
constexpr int kBeamWarps = kBeamThreads / 32;

struct RowReduce {
    float mx[kBeamWarps];
    double sum[kBeamWarps];
    int cnt[kBeamWarps];
    float thr;
};

__device__ __forceinline__ float row_threshold(float mx, float frac) {
    return mx > 0.0f ? __fmul_rn(frac, mx) : 1.0f;
}

template <bool VEC>
__global__ void __launch_bounds__(kBeamThreads) beam_rows_kernel(const float* __restrict__ A, long long rows,
                                                                  long long V, long long ld, float frac,
                                                                  float* __restrict__ row_max,
                                                                  double* __restrict__ row_sum,
                                                                  int* __restrict__ row_count,
                                                                  signed char* __restrict__ mask, long long ldm) {
    __shared__ RowReduce R;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        const float* row = A + r * ld;
        // ---- pass A: max and sum
        float mx = -INFINITY;
        double s = 0.0;
        long long i0 = 0;
        if (VEC) {
            const float4* row4 = reinterpret_cast<const float4*>(row);
            const long long n4 = V >> 2;
            for (long long i = tid; i < n4; i += kBeamThreads) {
                const float4 v = __ldg(row4 + i);
                mx = fmaxf(fmaxf(mx, fmaxf(v.x, v.y)), fmaxf(v.z, v.w));
                s += ((double)v.x + (double)v.y) + ((double)v.z + (double)v.w);
            }
            i0 = n4 << 2;
        }
        for (long long i = i0 + tid; i < V; i += kBeamThreads) {
            const float v = __ldg(row + i);
            mx = fmaxf(mx, v);
            s += (double)v;
        }
        for (int o = 16; o > 0; o >>= 1) {
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            s += __shfl_xor_sync(0xffffffffu, s, o);
        }
        if (lane == 0) {
            R.mx[warp] = mx;
            R.sum[warp] = s;
        }
        __syncthreads();
        if (tid == 0) {
            float m = R.mx[0];
            double t = R.sum[0];
            for (int w = 1; w < kBeamWarps; ++w) {
                m = fmaxf(m, R.mx[w]);
                t += R.sum[w];
            }
            R.thr = row_threshold(m, frac);
            row_max[r] = m;
            row_sum[r] = t;
        }
        __syncthreads();
        const float thr = R.thr;
        // ---- pass B: mask and its size
        int c = 0;
        signed char* mrow = mask ? mask + r * ldm : nullptr;
        if (VEC) {
            const float4* row4 = reinterpret_cast<const float4*>(row);
            const long long n4 = V >> 2;
            for (long long i = tid; i < n4; i += kBeamThreads) {
                const float4 v = __ldg(row4 + i);
                const int b0 = v.x > thr, b1 = v.y > thr, b2 = v.z > thr, b3 = v.w > thr;
                c += b0 + b1 + b2 + b3;
                if (mrow) reinterpret_cast<char4*>(mrow)[i] = make_char4(b0, b1, b2, b3);
            }
        }
        for (long long i = i0 + tid; i < V; i += kBeamThreads) {
            const int b = __ldg(row + i) > thr;
            c += b;
            if (mrow) mrow[i] = (signed char)b;
        }
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) R.cnt[warp] = c;
        __syncthreads();
        if (tid == 0) {
            int t = 0;
            for (int w = 0; w < kBeamWarps; ++w) t += R.cnt[w];
            row_count[r] = t;
        }
        __syncthreads();
    }
}

// MPXI: thread owns voxels 4t..4t+3; block (x, y) counts rows [y * rpb, (y + 1) * rpb).
template <bool FROM_MASK, bool VEC>
__global__ void __launch_bounds__(kBeamThreads) beam_mpxi_kernel(const float* __restrict__ A, long long ld,
                                                                  const signed char* __restrict__ mask,
                                                                  long long ldm, const float* __restrict__ row_max,
                                                                  float frac, long long rows, long long V,
                                                                  long long rows_per_block,
                                                                  unsigned* __restrict__ mpxi) {
    const long long c0 = 4 * ((long long)blockIdx.x * kBeamThreads + threadIdx.x);
    if (c0 >= V) return;
    const long long r0 = (long long)blockIdx.y * rows_per_block;
    const long long r1 = r0 + rows_per_block < rows ? r0 + rows_per_block : rows;
    const int nc = V - c0 >= 4 ? 4 : (int)(V - c0);
    unsigned u[4] = {0u, 0u, 0u, 0u};
    for (long long r = r0; r < r1; ++r) {
        if (FROM_MASK) {
            const signed char* m = mask + r * ldm + c0;
            if (VEC && nc == 4) {
                const char4 b = *reinterpret_cast<const char4*>(m);
                u[0] += b.x; u[1] += b.y; u[2] += b.z; u[3] += b.w;
            } else {
                for (int k = 0; k < nc; ++k) u[k] += m[k];
            }
        } else {
            const float thr = row_threshold(__ldg(row_max + r), frac);
            const float* a = A + r * ld + c0;
            if (VEC && nc == 4) {
                const float4 v = __ldg(reinterpret_cast<const float4*>(a));
                u[0] += v.x > thr; u[1] += v.y > thr; u[2] += v.z > thr; u[3] += v.w > thr;
            } else {
                for (int k = 0; k < nc; ++k) u[k] += __ldg(a + k) > thr;
            }
        }
    }
    for (int k = 0; k < nc; ++k)
        if (u[k]) atomicAdd(mpxi + c0 + k, u[k]);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
bool aligned4(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 3u) == 0; }

}  // namespace
}  // namespace smb

using namespace smb;

extern "C" int sm_beam_metrics(const float* sysmat, int64_t rows, int64_t voxels, int64_t ld, float frac,
                               float* row_max, double* row_sum, int32_t* row_count, int8_t* mask, int64_t ld_mask,
                               uint32_t* mpxi, void* stream_ptr) {
    if (!sysmat || !row_max || !row_sum || !row_count) return fail(SM_ERR_INVALID, "null argument");
    if (rows < 1 || voxels < 1) return fail(SM_ERR_INVALID, "rows (%lld) and voxels (%lld) must be >= 1",
                                            (long long)rows, (long long)voxels);
    if (ld < voxels) return fail(SM_ERR_INVALID, "ld = %lld is smaller than %lld voxels", (long long)ld, (long long)voxels);
    if (mask && ld_mask < voxels)
        return fail(SM_ERR_INVALID, "ld_mask = %lld is smaller than %lld voxels", (long long)ld_mask, (long long)voxels);
    if (!(frac >= 0.0f) || !(frac < INFINITY)) return fail(SM_ERR_INVALID, "frac = %g must be finite and >= 0", frac);
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    int sms = 148, dev = 0;
    SM_CUDA(cudaGetDevice(&dev));
    SM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const bool vec = (ld % 4 == 0) && aligned16(sysmat) && (!mask || ((ld_mask % 4 == 0) && aligned4(mask)));
    const long long grid1 = rows < (long long)sms * 8 ? rows : (long long)sms * 8;
    signed char* m = reinterpret_cast<signed char*>(mask);
    if (vec)
        beam_rows_kernel<true><<<(unsigned)grid1, kBeamThreads, 0, stream>>>(sysmat, rows, voxels, ld, frac, row_max,
                                                                             row_sum, row_count, m, ld_mask);
    else
        beam_rows_kernel<false><<<(unsigned)grid1, kBeamThreads, 0, stream>>>(sysmat, rows, voxels, ld, frac, row_max,
                                                                              row_sum, row_count, m, ld_mask);
    SM_CUDA(cudaGetLastError());
    if (!mpxi) return SM_OK;
    SM_CUDA(cudaMemsetAsync(mpxi, 0, sizeof(uint32_t) * (size_t)voxels, stream));
    const long long threads = (voxels + 3) / 4;
    const long long gx = (threads + kBeamThreads - 1) / kBeamThreads;
    long long gy = ((long long)sms * 8 + gx - 1) / gx;
    if (gy > rows) gy = rows;
    if (gy > 65535) gy = 65535;
    if (gx > 0x7fffffffLL) return fail(SM_ERR_CAPACITY, "%lld voxels exceed the launch grid", (long long)voxels);
    const long long rpb = (rows + gy - 1) / gy;
    gy = (rows + rpb - 1) / rpb;
    const dim3 grid2((unsigned)gx, (unsigned)gy);
    unsigned* out = reinterpret_cast<unsigned*>(mpxi);
    if (mask) {
        if (vec)
            beam_mpxi_kernel<true, true><<<grid2, kBeamThreads, 0, stream>>>(sysmat, ld, m, ld_mask, row_max, frac, rows,
                                                                            voxels, rpb, out);
        else
            beam_mpxi_kernel<true, false><<<grid2, kBeamThreads, 0, stream>>>(sysmat, ld, m, ld_mask, row_max, frac,
                                                                             rows, voxels, rpb, out);
    } else {
        if (vec)
            beam_mpxi_kernel<false, true><<<grid2, kBeamThreads, 0, stream>>>(sysmat, ld, m, ld_mask, row_max, frac,
                                                                             rows, voxels, rpb, out);
        else
            beam_mpxi_kernel<false, false><<<grid2, kBeamThreads, 0, stream>>>(sysmat, ld, m, ld_mask, row_max, frac,
                                                                              rows, voxels, rpb, out);
    }
    SM_CUDA(cudaGetLastError());
    return SM_OK;
}
