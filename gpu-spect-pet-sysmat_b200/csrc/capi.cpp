// C ABI: contexts, geometry objects, the PE entry points and the legacy
// PESysMatGen drop-in (include/sysmat_b200.h).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "context.h"
#include "geometry.h"
#include "pe.h"

namespace smb {

static thread_local char g_err[1024] = "";

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

const char* last_error() { return g_err; }

cudaMemPool_t& current_pool() {
    static thread_local cudaMemPool_t pool = nullptr;
    return pool;
}

int context_bind(sm_context* ctx) {
    if (!ctx) return fail(SM_ERR_INVALID, "null context");
    SM_CUDA(cudaSetDevice(ctx->device));
    current_pool() = ctx->pool;
    return SM_OK;
}

// Reads back and clears the device status word (synchronises `stream`).
int context_collect_status(sm_context* ctx, cudaStream_t stream) {
    int st = 0;
    SM_CUDA(cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    SM_CUDA(cudaStreamSynchronize(stream));
    if (st != 0) {
        SM_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), stream));
        SM_CUDA(cudaStreamSynchronize(stream));
        if (st & kStatusRecordOverflow)
            return fail(SM_ERR_CAPACITY, "a ray hit more than %d holes or %d crystals (hit record capacity)", kRecHoles,
                        kRecCrystals);
        return fail(SM_ERR_CUDA, "device status 0x%x", st);
    }
    return SM_OK;
}

int validate_pe(const sm_geometry* geo, const sm_pe_options* opt, int row0, int row1, int z0, int nz) {
    for (int a = 0; a < 3; ++a) {
        if (opt->sv[a] < 1 || opt->sv[a] > 64) return fail(SM_ERR_INVALID, "sv[%d] = %d must be in 1..64", a, opt->sv[a]);
        if (opt->sc[a] < 1 || opt->sc[a] > kMaxSubcellsPerAxis)
            return fail(SM_ERR_INVALID, "sc[%d] = %d must be in 1..%d", a, opt->sc[a], kMaxSubcellsPerAxis);
        if (opt->tile_voxels[a] < 0) return fail(SM_ERR_INVALID, "tile_voxels[%d] must be >= 0", a);
    }
    if ((int64_t)opt->sv[0] * opt->sv[1] * opt->sv[2] * opt->sc[0] * opt->sc[1] * opt->sc[2] > (1 << 22))
        return fail(SM_ERR_CAPACITY, "more than 2^22 rays per entry");
    if (opt->group < 0 || opt->group > kMaxGroup)
        return fail(SM_ERR_INVALID, "group = %d must be 0 (auto) or 1..%d", opt->group, kMaxGroup);
    const HostGeometry& g = geo->host;
    if ((int64_t)g.nx * opt->sv[0] > (1 << 24) || (int64_t)g.ny * opt->sv[1] > (1 << 24) ||
        (int64_t)g.nz * opt->sv[2] > (1 << 24))
        return fail(SM_ERR_CAPACITY, "fine voxel grid exceeds 2^24 per axis");
    if (row0 < 0 || row1 > g.n_crystals || row0 >= row1)
        return fail(SM_ERR_INVALID, "row range [%d, %d) outside [0, %d)", row0, row1, g.n_crystals);
    if (z0 < 0 || nz < 1 || z0 + nz > g.nz) return fail(SM_ERR_INVALID, "slab z [%d, %d) outside [0, %d)", z0, z0 + nz, g.nz);
    return SM_OK;
}

}  // namespace smb

// ---- legacy drop-in: PEGen_RayTracing_CircularHole/PESysMatGen.h:4-9 ----------
static std::mutex g_legacy_mu;
static sm_context* g_legacy_ctx[64] = {nullptr};

namespace smb {
sm_context* legacy_context(int cuda_id) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) return nullptr;
    if (cuda_id < 0 || cuda_id >= n) cuda_id = 0;   // scatter.cu:2034-2037 falls back to device 0
    if (cuda_id >= 64) return nullptr;
    if (!g_legacy_ctx[cuda_id]) {
        sm_context* c = nullptr;
        if (sm_context_create(cuda_id, &c) != SM_OK) return nullptr;
        g_legacy_ctx[cuda_id] = c;
    }
    return g_legacy_ctx[cuda_id];
}
}  // namespace smb

using namespace smb;

extern "C" {

const char* sm_last_error(void) { return last_error(); }
const char* sm_version(void) { return "sysmat_b200 0.1 (sm_100a)"; }

int sm_context_create(int device, sm_context** out) {
    if (!out) return fail(SM_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int n = 0;
    SM_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return fail(SM_ERR_DEVICE, "device %d not present (%d devices)", device, n);
    cudaDeviceProp prop;
    SM_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return fail(SM_ERR_DEVICE, "device %d is sm_%d%d; this build targets sm_100a", device, prop.major, prop.minor);
    SM_CUDA(cudaSetDevice(device));
    sm_context* ctx = new (std::nothrow) sm_context();
    if (!ctx) return fail(SM_ERR_ALLOC, "host allocation failed");
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    int rc = check_cuda(cudaMalloc(&ctx->d_status, 64), "status word");
    if (rc == SM_OK) rc = check_cuda(cudaMemset(ctx->d_status, 0, 64), "status word");
    if (rc != SM_OK) {
        delete ctx;
        return rc;
    }
    ctx->d_counters = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(ctx->d_status) + 32);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&ctx->pool, &props) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    } else {
        ctx->pool = nullptr;   // fall back to the device's default pool
        cudaGetLastError();
    }
    *out = ctx;
    return SM_OK;
}

int sm_context_destroy(sm_context* ctx) {
    if (!ctx) return SM_OK;
    cudaSetDevice(ctx->device);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->pool) {
        cudaDeviceSynchronize();   // frees still queued on streams reach the pool first
        cudaMemPoolDestroy(ctx->pool);
        if (current_pool() == ctx->pool) current_pool() = nullptr;
    }
    delete ctx;
    return SM_OK;
}

int sm_context_trim(sm_context* ctx) {
    SM_TRY(context_bind(ctx));
    if (ctx->pool) {
        SM_CUDA(cudaDeviceSynchronize());
        SM_CUDA(cudaMemPoolTrimTo(ctx->pool, 0));
    }
    return SM_OK;
}

int sm_context_sync(sm_context* ctx, void* stream) {
    SM_TRY(context_bind(ctx));
    return context_collect_status(ctx, (cudaStream_t)stream);
}

int sm_geometry_create(sm_context* ctx, const float* collimator, size_t n_collimator, const float* detector,
                       size_t n_detector, const float* image, size_t n_image, const float* physics, size_t n_physics,
                       sm_geometry** out) {
    if (!out) return fail(SM_ERR_INVALID, "null output pointer");
    *out = nullptr;
    SM_TRY(context_bind(ctx));
    sm_geometry* geo = new (std::nothrow) sm_geometry();
    if (!geo) return fail(SM_ERR_ALLOC, "host allocation failed");
    geo->ctx = ctx;
    int rc = parse_geometry(collimator, n_collimator, detector, n_detector, image, n_image, physics, n_physics, &geo->host);
    if (rc == SM_OK) rc = upload_geometry(geo->host, &geo->dev);
    if (rc != SM_OK) {
        delete geo;
        return rc;
    }
    *out = geo;
    return SM_OK;
}

int sm_tables_check(const float* collimator, size_t n_collimator, const float* detector, size_t n_detector,
                    const float* image, size_t n_image, const float* physics, size_t n_physics, int64_t out[7]) {
    HostGeometry g;
    SM_TRY(parse_geometry(collimator, n_collimator, detector, n_detector, image, n_image, physics, n_physics, &g));
    if (out) {
        out[0] = g.n_crystals;
        out[1] = g.n_holes;
        out[2] = g.n_plates;
        out[3] = g.nx;
        out[4] = g.ny;
        out[5] = g.nz;
        out[6] = g.n_rotations;
    }
    return SM_OK;
}

int sm_geometry_destroy(sm_geometry* geo) {
    if (!geo) return SM_OK;
    cudaSetDevice(geo->ctx->device);
    free_geometry(&geo->dev);
    delete geo;
    return SM_OK;
}

int sm_geometry_info(const sm_geometry* geo, int64_t out[7]) {
    if (!geo || !out) return fail(SM_ERR_INVALID, "null argument");
    const HostGeometry& g = geo->host;
    out[0] = g.n_crystals;
    out[1] = g.n_holes;
    out[2] = g.n_plates;
    out[3] = g.nx;
    out[4] = g.ny;
    out[5] = g.nz;
    out[6] = g.n_rotations;
    return SM_OK;
}

void sm_pe_options_reference(sm_pe_options* opt) {
    if (!opt) return;
    std::memset(opt, 0, sizeof(*opt));
    opt->sv[0] = opt->sv[1] = opt->sv[2] = 1;
    opt->sc[0] = 8;
    opt->sc[1] = 16;
    opt->sc[2] = 8;
}

int sm_pe_compute(sm_context* ctx, const sm_geometry* geo, const sm_pe_options* opt, int rotation, int row0, int row1,
                  int z0, int nz, float* dst, int64_t ld, int dst_on_device, void* stream_ptr) {
    if (!geo || !opt || !dst) return fail(SM_ERR_INVALID, "null argument");
    SM_TRY(context_bind(ctx));
    SM_TRY(validate_pe(geo, opt, row0, row1, z0, nz));
    const HostGeometry& g = geo->host;
    const int64_t slab = (int64_t)g.nx * g.ny * nz;
    if (ld < slab) return fail(SM_ERR_INVALID, "ld = %lld is smaller than the slab's %lld voxels", (long long)ld, (long long)slab);
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    sm_pe_options tuned = *opt;
    if (opt->flags & SM_PE_AUTOTUNE) SM_TRY(sm_pe_autotune(ctx, geo, opt, rotation, &tuned, nullptr));
    PEParams P;
    pe_plan(g, tuned.sv, tuned.sc, tuned.tile_voxels, tuned.group, rotation, row0, row1, g.nz, z0, nz, &P);
    P.status = ctx->d_status;
    P.counters = ctx->collect_counters ? ctx->d_counters : nullptr;
    if (P.counters) SM_CUDA(cudaMemsetAsync(ctx->d_counters, 0, 4 * sizeof(unsigned long long), stream));
    float* d_out = dst;
    const int64_t rows = row1 - row0;
    if (!dst_on_device) {
        SM_CUDA(cudaMalloc(&d_out, sizeof(float) * (size_t)rows * (size_t)ld));
    }
    P.dst = d_out;
    P.ld = ld;
    int rc = check_cuda(pe_launch(P, geo->dev.view, false, P.n_tiles, stream), "pe_trace_kernel launch");
    if (rc == SM_OK && !dst_on_device) {
        rc = check_cuda(cudaMemcpyAsync(dst, d_out, sizeof(float) * (size_t)rows * (size_t)ld, cudaMemcpyDeviceToHost, stream),
                        "copy sysmat to host");
        if (rc == SM_OK) rc = context_collect_status(ctx, stream);
    }
    if (!dst_on_device) cudaFree(d_out);
    if (rc == SM_OK && P.counters) {
        unsigned long long c[4];
        rc = check_cuda(cudaMemcpyAsync(c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost, stream), "counters");
        if (rc == SM_OK) rc = check_cuda(cudaStreamSynchronize(stream), "counters");
        for (int i = 0; i < 4; ++i) ctx->last_counters[i] = (int64_t)c[i];
    }
    return rc;
}

int sm_pe_set_counters(sm_context* ctx, int enable) {
    if (!ctx) return fail(SM_ERR_INVALID, "null context");
    ctx->collect_counters = enable != 0;
    return SM_OK;
}

int sm_pe_last_counters(sm_context* ctx, int64_t out[4]) {
    if (!ctx || !out) return fail(SM_ERR_INVALID, "null argument");
    for (int i = 0; i < 4; ++i) out[i] = ctx->last_counters[i];
    return SM_OK;
}

int sm_pe_record_hits(sm_context* ctx, const sm_geometry* geo, const sm_pe_options* opt, int rotation,
                      const int64_t* rows, const int64_t* voxels, int64_t n, int32_t* out, int* record_words) {
    if (!geo || !opt || !rows || !voxels || !out) return fail(SM_ERR_INVALID, "null argument");
    if (n < 1 || n > 64) return fail(SM_ERR_INVALID, "record between 1 and 64 entries per call (got %lld)", (long long)n);
    SM_TRY(context_bind(ctx));
    SM_TRY(validate_pe(geo, opt, 0, geo->host.n_crystals, 0, geo->host.nz));
    const HostGeometry& g = geo->host;
    PEParams P;
    pe_plan(g, opt->sv, opt->sc, opt->tile_voxels, opt->group, rotation, 0, g.n_crystals, g.nz, 0, g.nz, &P);
    const int64_t vox_n = (int64_t)g.nx * g.ny * g.nz;
    std::vector<long long> tiles;
    for (int64_t i = 0; i < n; ++i) {
        if (rows[i] < 0 || rows[i] >= g.n_crystals || voxels[i] < 0 || voxels[i] >= vox_n)
            return fail(SM_ERR_INVALID, "entry %lld out of range", (long long)i);
        long long v = voxels[i];
        int ix = (int)(v % g.nx), iy = (int)((v / g.nx) % g.ny), iz = (int)(v / ((long long)g.nx * g.ny));
        long long vt = ((long long)(iz / P.bz) * P.tiles_y + iy / P.by) * P.tiles_x + ix / P.bx;
        long long t = vt * P.n_ctiles + rows[i] / kPeWarps;
        if (std::find(tiles.begin(), tiles.end(), t) == tiles.end()) tiles.push_back(t);
    }
    const int64_t rays = (int64_t)P.n_sv * P.n_sc;
    const size_t out_words = (size_t)n * (size_t)rays * kRecWords;
    long long *d_tiles = nullptr, *d_rows = nullptr, *d_vox = nullptr;
    int* d_out = nullptr;
    int rc = SM_OK;
    rc = check_cuda(cudaMalloc(&d_tiles, sizeof(long long) * tiles.size()), "record alloc");
    if (rc == SM_OK) rc = check_cuda(cudaMalloc(&d_rows, sizeof(long long) * n), "record alloc");
    if (rc == SM_OK) rc = check_cuda(cudaMalloc(&d_vox, sizeof(long long) * n), "record alloc");
    if (rc == SM_OK) rc = check_cuda(cudaMalloc(&d_out, sizeof(int) * out_words), "record alloc");
    if (rc == SM_OK) rc = check_cuda(cudaMemcpy(d_tiles, tiles.data(), sizeof(long long) * tiles.size(), cudaMemcpyHostToDevice), "record copy");
    if (rc == SM_OK) rc = check_cuda(cudaMemcpy(d_rows, rows, sizeof(long long) * n, cudaMemcpyHostToDevice), "record copy");
    if (rc == SM_OK) rc = check_cuda(cudaMemcpy(d_vox, voxels, sizeof(long long) * n, cudaMemcpyHostToDevice), "record copy");
    if (rc == SM_OK) rc = check_cuda(cudaMemset(d_out, 0, sizeof(int) * out_words), "record clear");
    if (rc == SM_OK) {
        P.tile_list = d_tiles;
        P.status = ctx->d_status;
        P.dst = nullptr;
        P.ld = 0;
        P.rec_n = (int)n;
        P.rec_rows = d_rows;
        P.rec_vox = d_vox;
        P.rec_out = d_out;
        rc = check_cuda(pe_launch(P, geo->dev.view, true, (long long)tiles.size(), 0), "record launch");
    }
    if (rc == SM_OK) rc = check_cuda(cudaMemcpy(out, d_out, sizeof(int) * out_words, cudaMemcpyDeviceToHost), "record copy back");
    if (rc == SM_OK) rc = context_collect_status(ctx, 0);
    cudaFree(d_tiles);
    cudaFree(d_rows);
    cudaFree(d_vox);
    cudaFree(d_out);
    if (record_words) *record_words = kRecWords;
    return rc;
}

// ---- legacy drop-in: PEGen_RayTracing_CircularHole/PESysMatGen.h:4-9 ----------
int PESysMatGen(float* parameter_Collimator, float* parameter_Detector, float* parameter_Image, float* dst, int cuda_id) {
    std::lock_guard<std::mutex> lock(g_legacy_mu);
    if (!parameter_Collimator || !parameter_Detector || !parameter_Image || !dst) {
        std::fprintf(stderr, "PESysMatGen: null argument\n");
        return -1;
    }
    sm_context* ctx = legacy_context(cuda_id);
    if (!ctx) {
        std::fprintf(stderr, "PESysMatGen: %s\n", sm_last_error());
        return -1;
    }
    // The tables the reference reads: 80000 / 80000 / 100 floats (PESysMatGen.cu:797-804).
    sm_geometry* geo = nullptr;
    int rc = sm_geometry_create(ctx, parameter_Collimator, 80000, parameter_Detector, 80000, parameter_Image, 100,
                                nullptr, 0, &geo);
    if (rc != SM_OK) {
        std::fprintf(stderr, "PESysMatGen: %s\n", sm_last_error());
        return -1;
    }
    const HostGeometry& g = geo->host;
    // Slab side channel: Image[2] = slab z-planes, Image[30] = full z, Image[31] = z0,
    // Image[20] = rotation (PESysMatGen.cu:390-416).
    const int nz_slab = (int)std::floor(parameter_Image[2]);
    const int nz_full = (int)std::floor(parameter_Image[30]);
    const int z0 = (int)std::floor(parameter_Image[31] + 0.001f);
    const int rotation_index = (int)std::floor(parameter_Image[20] + 0.5f);
    sm_pe_options opt;
    sm_pe_options_reference(&opt);
    PEParams P;
    const int64_t slab = (int64_t)g.nx * g.ny * nz_slab;
    pe_plan(g, opt.sv, opt.sc, opt.tile_voxels, opt.group, rotation_index, 0, g.n_crystals, nz_full, z0, nz_slab, &P);
    // The kernel indexes slab-local columns from z0; a legacy slab is "z0..z0+nz of
    // a volume of nz_full planes", so the slab's own z range is [z0, z0 + nz_slab).
    float angle = parameter_Image[20] * parameter_Image[7];
    P.cos_a = std::cos(angle);
    P.sin_a = std::sin(angle);
    float* d_out = nullptr;
    rc = check_cuda(cudaMalloc(&d_out, sizeof(float) * (size_t)g.n_crystals * (size_t)slab), "PESysMatGen alloc");
    if (rc == SM_OK) {
        P.status = ctx->d_status;
        P.dst = d_out;
        P.ld = slab;
        rc = check_cuda(pe_launch(P, geo->dev.view, false, P.n_tiles, 0), "PESysMatGen launch");
    }
    if (rc == SM_OK)
        rc = check_cuda(cudaMemcpy(dst, d_out, sizeof(float) * (size_t)g.n_crystals * (size_t)slab, cudaMemcpyDeviceToHost),
                        "PESysMatGen copy back");
    if (rc == SM_OK) rc = context_collect_status(ctx, 0);
    if (d_out) cudaFree(d_out);
    sm_geometry_destroy(geo);
    if (rc != SM_OK) {
        std::fprintf(stderr, "PESysMatGen: %s\n", sm_last_error());
        return -1;
    }
    return (int)slab;
}

}  // extern "C"
