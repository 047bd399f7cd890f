// Shared host-side helpers: status codes, thread-local error message, CUDA checks.
#pragma once

#include <cstdarg>
#include <cstdio>
#include <string>

#include <cuda_runtime.h>

#include "sysmat_b200.h"

namespace smb {

// Records `fmt` as the calling thread's last error and returns `code`.
int fail(int code, const char* fmt, ...);
const char* last_error();

struct CudaError {
    int code;
};

// Returns SM_ERR_CUDA with the runtime's message when `e` is not cudaSuccess.
inline int check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return SM_OK;
    if (e == cudaErrorMemoryAllocation)
        return fail(SM_ERR_ALLOC, "%s: %s", what, cudaGetErrorString(e));
    return fail(SM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define SM_TRY(expr)                      \
    do {                                  \
        int sm_try_rc_ = (expr);          \
        if (sm_try_rc_ != SM_OK) return sm_try_rc_; \
    } while (0)

#define SM_CUDA(expr) SM_TRY(::smb::check_cuda((expr), #expr))

// The calling thread's memory pool: the one of the context last bound on this
// thread (context_bind), or null for the device's default pool.
cudaMemPool_t& current_pool();

// Stream-ordered device buffer from the current pool, released on the same
// stream.  A context's pool keeps freed memory mapped (no release threshold),
// so large workspaces freed and allocated again within or across calls do not
// pay for unmapping and mapping at every synchronisation.
struct DevBuf {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    int alloc(size_t bytes, cudaStream_t stream, const char* what) {
        s = stream;
        cudaMemPool_t pool = current_pool();
        if (pool) return check_cuda(cudaMallocFromPoolAsync(&p, bytes ? bytes : 16, pool, stream), what);
        return check_cuda(cudaMallocAsync(&p, bytes ? bytes : 16, stream), what);
    }
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
};


}  // namespace smb
