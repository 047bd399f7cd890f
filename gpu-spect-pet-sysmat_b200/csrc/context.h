// Definitions behind the opaque sm_context / sm_geometry handles.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "geometry.h"
#include "sysmat_b200.h"

struct sm_context {
    int device = 0;
    int sm_count = 0;
    int* d_status = nullptr;                    // device status word (+ counters in the same block)
    unsigned long long* d_counters = nullptr;   // 4 x u64 inside the status block
    bool collect_counters = false;
    int64_t last_counters[4] = {0, 0, 0, 0};
    cudaMemPool_t pool = nullptr;               // device workspaces (DevBuf), kept mapped until trimmed
};

struct sm_geometry {
    sm_context* ctx = nullptr;
    smb::HostGeometry host;
    smb::DeviceGeometryBuffer dev;
};

namespace smb {
int context_bind(sm_context* ctx);
int context_collect_status(sm_context* ctx, cudaStream_t stream);
sm_context* legacy_context(int cuda_id);
int validate_pe(const sm_geometry* geo, const sm_pe_options* opt, int row0, int row1, int z0, int nz);
}  // namespace smb
