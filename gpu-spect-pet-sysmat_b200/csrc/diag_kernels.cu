// Diagnostic kernel: evaluates the tracer's ray primitives (tracer.cuh) on a
// batch of argument rows, so that tests can compare them with the reference
// primitives bit for bit.  Same device functions as the production kernel.
#include <cuda_runtime.h>

#include "common.h"
#include "tracer.cuh"

namespace smb {
namespace {

__global__ void primitive_kernel(int kind, const float* __restrict__ args, long long n, float* __restrict__ out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (kind == 2) {
        const float* a = args + 11 * i;
        out[i] = chord_hole(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10]);
        return;
    }
    const float* a = args + 12 * i;
    Box3 b{a[6], a[7], a[8], a[9], a[10], a[11]};
    out[i] = kind == 0 ? chord_through(a[0], a[1], a[2], a[3], a[4], a[5], b)
                       : chord_to_end(a[0], a[1], a[2], a[3], a[4], a[5], b);
}

}  // namespace
}  // namespace smb

using namespace smb;

extern "C" int sm_primitive_batch(int kind, const float* args, int64_t n, float* out) {
    if (kind < 0 || kind > 2 || n < 0 || (!args && n) || (!out && n)) return fail(SM_ERR_INVALID, "bad primitive batch");
    if (n == 0) return SM_OK;
    const size_t w = kind == 2 ? 11 : 12;
    float *d_args = nullptr, *d_out = nullptr;
    int rc = check_cuda(cudaMalloc(&d_args, sizeof(float) * w * (size_t)n), "primitive alloc");
    if (rc == SM_OK) rc = check_cuda(cudaMalloc(&d_out, sizeof(float) * (size_t)n), "primitive alloc");
    if (rc == SM_OK) rc = check_cuda(cudaMemcpy(d_args, args, sizeof(float) * w * (size_t)n, cudaMemcpyHostToDevice), "primitive copy");
    if (rc == SM_OK) {
        primitive_kernel<<<(unsigned)((n + 255) / 256), 256>>>(kind, d_args, n, d_out);
        rc = check_cuda(cudaGetLastError(), "primitive launch");
    }
    if (rc == SM_OK) rc = check_cuda(cudaMemcpy(out, d_out, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost), "primitive copy back");
    cudaFree(d_args);
    cudaFree(d_out);
    return rc;
}
