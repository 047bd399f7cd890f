// BF16 tensor-core GEMM (tcgen05, TMEM accumulators) for the scatter surrogate.
#pragma once

#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace smb {

// epilogue 0: C[m][n] = s_m * acc (+ bias[n]) (+ C[m][n] if accumulate)
// epilogue 1: C[m][n] = C[m][n] * exp(s_m * acc)            (multiplicative correction)
// acc = sum_k A[m][k] B[n][k], s_m = row_scale[m] when row_scale is set, else alpha.
struct GemmArgs {
    int m, n, k;
    const __nv_bfloat16* a;
    long long a_ms, a_ks;        // A[m][k] = a[m * a_ms + k * a_ks]
    const __nv_bfloat16* b;
    long long b_ns, b_ks;        // B[n][k] = b[n * b_ns + k * b_ks]
    float* c;
    long long ldc;
    float alpha;
    const float* row_scale;
    const float* bias;
    int accumulate;
    int epilogue;
    int n_tile;                  // 64, 128 or 256 columns per CTA (TMEM columns)
    int* error;                  // set to 1 when a bounded wait runs out (may be null)
};

cudaError_t gemm_bf16_tc(const GemmArgs& args, cudaStream_t stream);

// Sets the mbarrier poll limit of later gemm_bf16_tc launches (polls < 0: the
// default); returns the previous limit.
uint32_t gemm_wait_limit(int64_t polls);

}  // namespace smb
