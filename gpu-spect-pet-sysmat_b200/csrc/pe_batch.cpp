// Batched photoelectric sysmats (many geometries, one persistent launch
// replayed from a CUDA graph) and the brick-shape autotuner.
//
// The persistent kernel (pe_kernel.cu, pe_batch_kernel) hands out (geometry,
// tile) items from one counter; geometries are ordered by estimated cost,
// largest first, so the dynamic hand-out fills the tail with small items.
// The autotuner times candidate voxel bricks and sub-points per warp pass on
// a geometry (the whole matrix when it is small, else a sample of tiles) and
// caches the fastest per device and geometry class (in memory, and in the
// file named by SYSMAT_B200_TUNE_CACHE when it is set).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "context.h"
#include "geometry.h"
#include "pe.h"

struct sm_pe_batch {
    sm_context* ctx = nullptr;
    std::vector<smb::PeBatchGeom> host;
    void* d_geoms = nullptr;
    unsigned long long* d_counter = nullptr;
    long long total = 0;
    int grid = 0;
    cudaStream_t capture = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    struct Chunk {
        int first, count;
        long long items;
    };
    std::vector<Chunk> chunks;
};

namespace smb {
namespace {

std::mutex g_tune_mu;
std::map<std::string, std::vector<int>> g_tune;   // key -> brick (x, y, z), group
bool g_tune_loaded = false;

void tune_load_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = std::getenv("SYSMAT_B200_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    char key[512];
    int a, b, c;
    int gr;
    while (std::fscanf(f, "%511s %d %d %d %d", key, &a, &b, &c, &gr) == 5) g_tune[key] = {a, b, c, gr};
    std::fclose(f);
}

void tune_store_locked(const std::string& key, const int brick[3], int group) {
    g_tune[key] = {brick[0], brick[1], brick[2], group};
    const char* path = std::getenv("SYSMAT_B200_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "a");
    if (!f) return;
    std::fprintf(f, "%s %d %d %d %d\n", key.c_str(), brick[0], brick[1], brick[2], group);
    std::fclose(f);
}

// Geometry class: what decides which brick is fastest (grid, voxel size,
// sub-sampling, plates, holes and crystals in buckets), plus the device.
std::string tune_key(const sm_context* ctx, const HostGeometry& g, const sm_pe_options* opt) {
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, ctx->device);
    char buf[512];
    auto bucket = [](int n) { int b = 0; while ((1 << b) < n) ++b; return b; };
    std::snprintf(buf, sizeof(buf), "%s|sm%d|g%dx%dx%d|v%.3g|sv%dx%dx%d|sc%dx%dx%d|p%d|h%d|c%d", prop.name,
                  prop.multiProcessorCount, g.nx, g.ny, g.nz, g.voxel[0], opt->sv[0], opt->sv[1], opt->sv[2], opt->sc[0],
                  opt->sc[1], opt->sc[2], g.n_plates, bucket(g.n_holes), bucket(g.n_crystals));
    std::string k(buf);
    for (char& ch : k)
        if (ch == ' ') ch = '_';
    return k;
}

// Estimated work of a geometry: rays x (candidates a ray meets ~ holes and crystals).
double est_cost(const HostGeometry& g, const PEParams& P) {
    const double rays = (double)P.n_sv * P.n_sc * (double)(P.row1 - P.row0) * g.nx * g.ny * P.nzs;
    return rays * (1.0 + 0.02 * std::sqrt((double)g.n_holes) + 0.02 * std::sqrt((double)g.n_crystals));
}

}  // namespace
}  // namespace smb

using namespace smb;

extern "C" {

int sm_pe_autotune(sm_context* ctx, const sm_geometry* geo, const sm_pe_options* opt, int rotation,
                   sm_pe_options* out, double* best_ms_per_tile) {
    if (!geo || !opt || !out) return fail(SM_ERR_INVALID, "null argument");
    SM_TRY(context_bind(ctx));
    const HostGeometry& g = geo->host;
    SM_TRY(validate_pe(geo, opt, 0, g.n_crystals, 0, g.nz));
    *out = *opt;
    const std::string key = tune_key(ctx, g, opt);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        tune_load_locked();
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            for (int a = 0; a < 3; ++a) out->tile_voxels[a] = it->second[a];
            out->group = it->second.size() > 3 ? it->second[3] : 0;
            if (best_ms_per_tile) *best_ms_per_tile = -1.0;
            return SM_OK;
        }
    }
    // Objective: a small matrix (at most kWhole tiles with the default brick)
    // is timed whole, tail and all, which is what its launches cost; a large
    // one on a sample of tiles from a block of rows and a slab of z-planes in
    // the middle of the geometry, per voxel-row processed.
    constexpr long long kWhole = 16384;
    PEParams P0;
    const int zero3[3] = {0, 0, 0};
    pe_plan(g, opt->sv, opt->sc, zero3, 0, rotation, 0, g.n_crystals, g.nz, 0, g.nz, &P0);
    const bool whole = P0.n_tiles <= kWhole;
    const int rows = whole ? g.n_crystals : std::min(g.n_crystals, 512);
    const int row0 = (g.n_crystals - rows) / 2;
    const int nz = whole ? g.nz : std::min(g.nz, 8);
    const int z0 = (g.nz - nz) / 2;
    const int64_t slab = (int64_t)g.nx * g.ny * nz;
    static const int cand[][3] = {{8, 4, 4}, {4, 4, 4}, {8, 8, 2}, {4, 4, 8}, {16, 4, 2}, {4, 8, 4}, {8, 4, 2}, {8, 8, 1},
                                  {4, 4, 2}, {4, 2, 2}};
    // sub-points per group (rays each lane traces per group = group * sub-cells / 32):
    // the automatic value (one column of depth sub-cells per warp pass) and half of it
    std::vector<int> groups = {pe_auto_group(opt->sc[1])};
    if (groups[0] >= 2) groups.push_back(groups[0] / 2);
    float* d_out = nullptr;
    long long* d_tiles = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = check_cuda(cudaMalloc(&d_out, sizeof(float) * (size_t)rows * (size_t)slab), "autotune output");
    if (rc == SM_OK) rc = check_cuda(cudaMalloc(&d_tiles, sizeof(long long) * 4096), "autotune tiles");
    if (rc == SM_OK) rc = check_cuda(cudaEventCreate(&e0), "event");
    if (rc == SM_OK) rc = check_cuda(cudaEventCreate(&e1), "event");
    double best = 1e300, best_ms = 0.0;
    int best_brick[3] = {0, 0, 0}, best_group = 0;
    const int target_tiles = std::min(4096, ctx->sm_count * 2 * 4);
    for (const auto& c : cand) {
        for (int gr : groups) {
            if (rc != SM_OK) break;
            const int brick[3] = {c[0], c[1], c[2]};
            PEParams P;
            pe_plan(g, opt->sv, opt->sc, brick, gr, rotation, row0, row0 + rows, g.nz, z0, nz, &P);
            if (P.bx != brick[0] || P.by != brick[1] || P.bz != brick[2]) continue;   // clipped to the grid
            long long n_launch = P.n_tiles;
            if (!whole) {
                std::vector<long long> tiles;
                const long long k = std::min<long long>(P.n_tiles, target_tiles);
                for (long long i = 0; i < k; ++i) tiles.push_back(i * P.n_tiles / k);
                rc = check_cuda(cudaMemcpy(d_tiles, tiles.data(), sizeof(long long) * tiles.size(),
                                           cudaMemcpyHostToDevice), "autotune tiles");
                if (rc != SM_OK) break;
                P.tile_list = d_tiles;
                n_launch = (long long)tiles.size();
            }
            P.status = ctx->d_status;
            P.dst = d_out;
            P.ld = slab;
            double t_best = 1e300;
            for (int rep = 0; rep < 3 && rc == SM_OK; ++rep) {
                rc = check_cuda(cudaEventRecord(e0, 0), "event");
                if (rc == SM_OK) rc = check_cuda(pe_launch(P, geo->dev.view, false, n_launch, 0), "autotune launch");
                if (rc == SM_OK) rc = check_cuda(cudaEventRecord(e1, 0), "event");
                if (rc == SM_OK) rc = check_cuda(cudaEventSynchronize(e1), "autotune sync");
                float ms = 0.0f;
                if (rc == SM_OK) cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0) t_best = std::min(t_best, (double)ms);   // the first run warms up
            }
            // a launch that reports a device status bit is not a candidate (voxels whose
            // candidates overflow the lists are traced through the tables: slower, not an error)
            int st = 0;
            if (rc == SM_OK) rc = check_cuda(cudaMemcpy(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost), "status");
            if (rc == SM_OK && st != 0) {
                rc = check_cuda(cudaMemset(ctx->d_status, 0, sizeof(int)), "status");
                continue;
            }
            const double score = whole ? t_best : t_best / ((double)n_launch * brick[0] * brick[1] * brick[2]);
            if (score < best) {
                best = score;
                best_ms = t_best / (double)n_launch;
                std::memcpy(best_brick, brick, sizeof(best_brick));
                best_group = gr == groups[0] ? 0 : gr;
            }
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (d_tiles) cudaFree(d_tiles);
    if (d_out) cudaFree(d_out);
    if (rc == SM_OK) rc = context_collect_status(ctx, 0);
    if (rc != SM_OK) return rc;
    if (best_brick[0] == 0) return fail(SM_ERR_INVALID, "no brick candidate fits the grid");
    for (int a = 0; a < 3; ++a) out->tile_voxels[a] = best_brick[a];
    out->group = best_group;
    if (best_ms_per_tile) *best_ms_per_tile = best_ms;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    tune_store_locked(key, best_brick, best_group);
    return SM_OK;
}

int sm_pe_batch_create(sm_context* ctx, int n, const sm_geometry* const* geos, const sm_pe_options* opts,
                       const int* rotations, float* const* dst, const int64_t* ld, sm_pe_batch** out) {
    if (!out || n < 1 || !geos || !opts || !dst || !ld) return fail(SM_ERR_INVALID, "invalid batch arguments");
    *out = nullptr;
    SM_TRY(context_bind(ctx));
    std::vector<std::pair<double, int>> order;
    std::vector<PeBatchGeom> items(n);
    for (int i = 0; i < n; ++i) {
        const sm_geometry* geo = geos[i];
        if (!geo) return fail(SM_ERR_INVALID, "geometry %d is null", i);
        const HostGeometry& g = geo->host;
        sm_pe_options o = opts[i];
        if (o.flags & 1) SM_TRY(sm_pe_autotune(ctx, geo, &opts[i], rotations ? rotations[i] : 0, &o, nullptr));
        SM_TRY(validate_pe(geo, &o, 0, g.n_crystals, 0, g.nz));
        const int64_t vox = (int64_t)g.nx * g.ny * g.nz;
        if (ld[i] < vox) return fail(SM_ERR_INVALID, "geometry %d: ld %lld < %lld voxels", i, (long long)ld[i], (long long)vox);
        if (!dst[i]) return fail(SM_ERR_INVALID, "geometry %d: null output", i);
        PeBatchGeom& b = items[i];
        std::memset(&b, 0, sizeof(b));
        pe_plan(g, o.sv, o.sc, o.tile_voxels, o.group, rotations ? rotations[i] : 0, 0, g.n_crystals, g.nz, 0, g.nz, &b.P);
        b.P.status = ctx->d_status;
        b.P.dst = dst[i];
        b.P.ld = ld[i];
        b.G = geo->dev.view;
        order.push_back({est_cost(g, b.P) / std::max<long long>(1, b.P.n_tiles), i});
    }
    // most expensive tiles first
    std::stable_sort(order.begin(), order.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
        return a.first > b.first;
    });
    sm_pe_batch* B = new (std::nothrow) sm_pe_batch();
    if (!B) return fail(SM_ERR_ALLOC, "host allocation failed");
    B->ctx = ctx;
    long long at = 0;
    for (const auto& o : order) {
        PeBatchGeom b = items[o.second];
        b.tile_begin = at;
        at += b.P.n_tiles;
        B->host.push_back(b);
    }
    B->total = at;
    // chunks of at most kBatchConst geometries, each with items from 0
    for (size_t c0 = 0; c0 < B->host.size(); c0 += kBatchConst) {
        const size_t c1 = std::min(B->host.size(), c0 + (size_t)kBatchConst);
        const long long base = B->host[c0].tile_begin;
        long long end = base;
        for (size_t i = c0; i < c1; ++i) {
            B->host[i].tile_begin -= base;
            end = base + B->host[i].tile_begin + B->host[i].P.n_tiles;
        }
        B->chunks.push_back({(int)c0, (int)(c1 - c0), end - base});
    }
    B->grid = ctx->sm_count * pe_batch_blocks_per_sm();
    int rc = check_cuda(cudaMalloc(&B->d_geoms, sizeof(PeBatchGeom) * B->host.size()), "batch table");
    if (rc == SM_OK) rc = check_cuda(cudaMemcpy(B->d_geoms, B->host.data(), sizeof(PeBatchGeom) * B->host.size(),
                                                cudaMemcpyHostToDevice), "batch table");
    if (rc == SM_OK) rc = check_cuda(cudaMalloc(&B->d_counter, 256), "batch counter");
    if (rc == SM_OK) rc = check_cuda(cudaStreamCreateWithFlags(&B->capture, cudaStreamNonBlocking), "capture stream");
    if (rc != SM_OK) {
        sm_pe_batch_destroy(B);
        return rc;
    }
    *out = B;
    return SM_OK;
}

int sm_pe_batch_info(const sm_pe_batch* b, int64_t out[3]) {
    if (!b || !out) return fail(SM_ERR_INVALID, "null argument");
    out[0] = (int64_t)b->host.size();
    out[1] = b->total;
    out[2] = b->grid;
    return SM_OK;
}

int sm_pe_batch_run(sm_pe_batch* b, void* stream_ptr) {
    if (!b) return fail(SM_ERR_INVALID, "null batch");
    SM_TRY(context_bind(b->ctx));
    if (!b->exec) {
        // counter reset + persistent launch, captured once and replayed
        SM_CUDA(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal));
        cudaError_t e2 = cudaSuccess;
        for (const auto& c : b->chunks) {
            if (e2 == cudaSuccess)
                e2 = pe_batch_launch(static_cast<const PeBatchGeom*>(b->d_geoms) + c.first, c.count, c.items,
                                     b->d_counter, b->grid, b->capture);
        }
        cudaError_t e3 = cudaStreamEndCapture(b->capture, &b->graph);
        SM_CUDA(e2);
        SM_CUDA(e3);
        SM_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    SM_CUDA(cudaGraphLaunch(b->exec, (cudaStream_t)stream_ptr));
    return SM_OK;
}

int sm_pe_batch_destroy(sm_pe_batch* b) {
    if (!b) return SM_OK;
    if (b->ctx) cudaSetDevice(b->ctx->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->capture) cudaStreamDestroy(b->capture);
    if (b->d_geoms) cudaFree(b->d_geoms);
    if (b->d_counter) cudaFree(b->d_counter);
    delete b;
    return SM_OK;
}

}  // extern "C"
