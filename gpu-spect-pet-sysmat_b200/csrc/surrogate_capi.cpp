// C ABI of the scatter surrogate's building blocks (include/sysmat_b200.h).
#include <cuda_runtime.h>

#include "common.h"
#include "gemm_tc.h"

using namespace smb;

extern "C" int sm_gemm_bf16(int m, int n, int k, const void* a, int64_t a_ms, int64_t a_ks, const void* b, int64_t b_ns,
                            int64_t b_ks, float* c, int64_t ldc, float alpha, const float* row_scale, const float* bias,
                            int accumulate, int n_tile, int* error, void* stream) {
    if (m < 0 || n < 0 || k < 0 || (m > 0 && n > 0 && k > 0 && (!a || !b || !c)))
        return fail(SM_ERR_INVALID, "sm_gemm_bf16: bad sizes or null operand");
    if (n_tile != 64 && n_tile != 128 && n_tile != 256) return fail(SM_ERR_INVALID, "n_tile must be 64, 128 or 256");
    GemmArgs g{};
    g.m = m;
    g.n = n;
    g.k = k;
    g.a = static_cast<const __nv_bfloat16*>(a);
    g.a_ms = a_ms;
    g.a_ks = a_ks;
    g.b = static_cast<const __nv_bfloat16*>(b);
    g.b_ns = b_ns;
    g.b_ks = b_ks;
    g.c = c;
    g.ldc = ldc;
    g.alpha = alpha;
    g.row_scale = row_scale;
    g.bias = bias;
    g.accumulate = accumulate;
    g.n_tile = n_tile;
    g.error = error;
    SM_CUDA(gemm_bf16_tc(g, (cudaStream_t)stream));
    return SM_OK;
}

extern "C" int sm_tc_wait_limit(int64_t polls, int64_t* previous) {
    const uint32_t prev = gemm_wait_limit(polls);
    if (previous) *previous = (int64_t)prev;
    return SM_OK;
}
