// C ABI of the primary-Compton scatter sysmat (include/sysmat_b200.h):
// sm_scatter_* and the reference's `scatter` drop-in
// (ScatterGen_RayTracing_CircularHole/scatter.h:4-5, body scatter.cu:2013-2378).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "context.h"
#include "geometry.h"
#include "scatter.h"

namespace smb {
namespace {

constexpr size_t kPairBudget = size_t(512) << 20;   // bytes of pair data per detector chunk

int upload_tables(const HostScatterTables& H, int n_crystals, int n_holes0, cudaStream_t s, DevBuf* blob,
                  ScatterTables* T) {
    const size_t b_raw = H.crystal_raw.size() * 4, b_hraw = H.hole_raw.size() * 4, b_hsrc = H.hole_src.size() * 4,
                 b_src = H.crystal_src.size() * 4, b_kn = H.kn.size() * sizeof(KnNode);
    auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
    const size_t o_raw = 0, o_hraw = up(b_raw), o_hsrc = o_hraw + up(b_hraw), o_src = o_hsrc + up(b_hsrc),
                 o_kn = o_src + up(b_src), total = o_kn + up(b_kn);
    std::vector<unsigned char> host(total, 0);
    std::memcpy(host.data() + o_raw, H.crystal_raw.data(), b_raw);
    std::memcpy(host.data() + o_hraw, H.hole_raw.data(), b_hraw);
    std::memcpy(host.data() + o_hsrc, H.hole_src.data(), b_hsrc);
    std::memcpy(host.data() + o_src, H.crystal_src.data(), b_src);
    std::memcpy(host.data() + o_kn, H.kn.data(), b_kn);
    SM_TRY(blob->alloc(total, s, "scatter tables"));
    SM_CUDA(cudaMemcpyAsync(blob->p, host.data(), total, cudaMemcpyHostToDevice, s));
    SM_CUDA(cudaStreamSynchronize(s));   // the staging buffer is released on return
    unsigned char* b = static_cast<unsigned char*>(blob->p);
    T->crystal_raw = reinterpret_cast<const float4*>(b + o_raw);
    T->hole_raw = reinterpret_cast<const float4*>(b + o_hraw);
    T->hole_src = reinterpret_cast<const float4*>(b + o_hsrc);
    T->crystal_src = reinterpret_cast<const float4*>(b + o_src);
    T->kn = reinterpret_cast<const KnNode*>(b + o_kn);
    T->n_crystals = n_crystals;
    T->n_holes0 = n_holes0;
    T->n_points = H.n_points;
    T->kn_inv_norm = H.kn_inv_norm;
    return SM_OK;
}

int holes0_of(const HostGeometry& g) {
    if (g.n_plates < 1) return 0;
    int h0 = (int)std::floor(g.collimator[10] + 0.01f);
    return std::max(0, std::min(h0, g.n_holes));
}

void fill_common(const HostGeometry& g, int rotation_index_unused, float angle, ScatterParams* P) {
    (void)rotation_index_unused;
    P->nx = g.nx;
    P->ny = g.ny;
    P->nz = g.nz;
    P->vx = g.voxel[0];
    P->vy = g.voxel[1];
    P->vz = g.voxel[2];
    P->shx = g.shift[0];
    P->shy = g.shift[1];
    P->shz = g.shift[2];
    P->cos_a = std::cos(angle);
    P->sin_a = std::sin(angle);
    const float* ph = g.physics.data();
    P->e0 = ph[7];
    P->alpha = ph[7] / 511.0f;
    P->use_compton = (int)std::floor(ph[0] + 0.5f);
    P->same_window = (int)std::floor(ph[4] + 0.5f);
    P->win_lo = ph[5];
    P->win_hi = ph[6];
    P->plate_c_over_t = g.n_plates > 0 ? g.collimator[17] / g.collimator[15] : 0.0f;
    P->bricks_x = (g.nx + kScBrickX - 1) / kScBrickX;
    P->bricks_y = (g.ny + kScBrickY - 1) / kScBrickY;
    P->n_bricks = P->bricks_x * P->bricks_y * g.nz;
}

}  // namespace

// Both parts (mask bit 0 crystal, bit 1 collimator) into device dst; rows and
// voxels as `spec` says (see ExactSpec in scatter.h).
int exact_scatter(const sm_geometry* geo, const int sp[3], int parts, float angle, const float* d_pe, int64_t ld_pe,
                  const uint32_t* d_bm_crystal, const uint32_t* d_bm_collimator, const ExactSpec& spec, float* d_dst,
                  int64_t ld, cudaStream_t s) {
    const int row0 = spec.rows ? 0 : spec.row0, row1 = spec.rows ? (int)spec.rows->size() : spec.row1;
    const HostGeometry& g = geo->host;
    const int N = g.n_crystals;
    const int h0 = holes0_of(g);
    HostScatterTables H;
    SM_TRY(build_scatter_tables(g, sp, &H));
    DevBuf tables;
    ScatterTables T;
    SM_TRY(upload_tables(H, N, h0, s, &tables, &T));

    ScatterParams P{};
    fill_common(g, 0, angle, &P);
    const std::vector<int> order = spec.rows ? spatial_order_of(g, *spec.rows) : spatial_order(g, row0, row1);
    // row-list mode: rank r writes the dst row of detector order[r] in the caller's list
    std::vector<int> slot;
    if (spec.rows) {
        std::vector<int> where(N, -1);
        for (size_t i = 0; i < spec.rows->size(); ++i) {
            const int d = (*spec.rows)[i];
            if (d < 0 || d >= N || where[d] >= 0) return fail(SM_ERR_INVALID, "row list: entry %zu (%d) is out of range or repeated", i, d);
            where[d] = (int)i;
        }
        slot.resize(order.size());
        for (size_t r = 0; r < order.size(); ++r) slot[r] = spec.rows_in_place ? order[r] : where[order[r]];
    }
    DevBuf perm;
    SM_TRY(perm.alloc(sizeof(int) * (order.size() + slot.size()), s, "detector order"));
    SM_CUDA(cudaMemcpyAsync(perm.p, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice, s));
    if (!slot.empty())
        SM_CUDA(cudaMemcpyAsync(static_cast<int*>(perm.p) + order.size(), slot.data(), sizeof(int) * slot.size(),
                                cudaMemcpyHostToDevice, s));
    SM_CUDA(cudaStreamSynchronize(s));   // the host vectors are released on return
    P.perm = static_cast<const int*>(perm.p);
    P.slot = slot.empty() ? nullptr : static_cast<const int*>(perm.p) + order.size();
    P.dst_row0 = row0;
    P.dst = d_dst;
    P.ld = ld;
    P.pe = d_pe;
    P.ld_pe = ld_pe;
    if (spec.d_cols) {
        P.cols = spec.d_cols;
        P.n_cols = spec.n_cols;
        P.bricks_x = (spec.n_cols + kScBrickX - 1) / kScBrickX;
        P.bricks_y = (g.ny + kScBrickY - 1) / kScBrickY;
        P.n_bricks = P.bricks_x * P.bricks_y;
    }

    DevBuf bm_c, bm_h, bricks, pairs;
    const uint32_t* bmc = d_bm_crystal;
    const uint32_t* bmh = d_bm_collimator;
    const bool do_crystal = (parts & 1) != 0, do_collimator = (parts & 2) != 0 && h0 > 0;
    if (do_crystal && !bmc && !spec.pairs) {
        const int64_t w = crystal_bitmap_words(N);
        SM_TRY(bm_c.alloc(sizeof(uint32_t) * (size_t)w, s, "crystal bitmap"));
        SM_CUDA(launch_bitmap_crystal(static_cast<uint32_t*>(bm_c.p), w, T, s));
        bmc = static_cast<const uint32_t*>(bm_c.p);
    }
    if (do_collimator && !bmh) {
        const int64_t w = collimator_bitmap_words(N, h0);
        SM_TRY(bm_h.alloc(sizeof(uint32_t) * (size_t)w, s, "collimator bitmap"));
        SM_CUDA(launch_bitmap_collimator(static_cast<uint32_t*>(bm_h.p), w, T, s));
        bmh = static_cast<const uint32_t*>(bm_h.p);
    }
    bool written = false;
    if (do_crystal) {
        P.src_words = (N + 31) / 32;
        const size_t bb = sizeof(uint32_t) * (size_t)P.n_bricks * P.src_words;
        SM_TRY(bricks.alloc(bb, s, "brick sources"));
        SM_CUDA(cudaMemsetAsync(bricks.p, 0, bb, s));
        P.brick_sources = static_cast<const uint32_t*>(bricks.p);
        SM_CUDA(launch_brick_sources(P, T, static_cast<uint32_t*>(bricks.p), s));
    }
    const int kinds[2] = {kScatterCrystal, kScatterCollimator};
    const bool want[2] = {do_crystal, do_collimator};
    DevBuf pcol;
    for (int ki = 0; ki < 2; ++ki) {
        if (!want[ki]) continue;
        const int kind = kinds[ki];
        if (kind == kScatterCrystal && spec.pairs) {
            // shared table: column of rank r is the rank of detector order[r] in the table's order
            const std::vector<int>& all = *spec.pairs_order;
            std::vector<int> where(N, -1), col(order.size());
            for (int r = 0; r < (int)all.size(); ++r) where[all[r]] = r;
            bool ident = true;
            for (size_t r = 0; r < order.size(); ++r) {
                col[r] = where[order[r]];
                ident = ident && col[r] == (int)r;
            }
            ScatterParams Q = P;
            Q.kind = kind;
            Q.rank0 = 0;
            Q.rank1 = row1 - row0;
            Q.pair = spec.pairs;
            Q.pair_r0 = 0;
            Q.pair_ld = N;
            if (!ident) {
                SM_TRY(pcol.alloc(sizeof(int) * col.size(), s, "pair columns"));
                SM_CUDA(cudaMemcpyAsync(pcol.p, col.data(), sizeof(int) * col.size(), cudaMemcpyHostToDevice, s));
                SM_CUDA(cudaStreamSynchronize(s));
                Q.pair_col = static_cast<const int*>(pcol.p);
            }
            Q.accumulate = (written || spec.accumulate) ? 1 : 0;
            SM_CUDA(spec.rows ? launch_scatter_rows(Q, geo->dev.view, T, s) : launch_scatter_main(Q, geo->dev.view, T, s));
            written = true;
            continue;
        }
        const int n_src = kind == kScatterCrystal ? N * T.n_points : h0;
        int chunk = (int)std::max<size_t>(kScTileD, kPairBudget / (sizeof(float4) * (size_t)std::max(1, n_src)));
        chunk = std::max(kScTileD, chunk / kScTileD * kScTileD);
        const int n_rank = row1 - row0;
        const size_t pb = sizeof(float4) * (size_t)n_src * (size_t)std::min(chunk, n_rank);
        DevBuf pair;
        SM_TRY(pair.alloc(pb, s, "scatter pairs"));
        for (int c0 = 0; c0 < n_rank; c0 += chunk) {
            const int c1 = std::min(n_rank, c0 + chunk);
            SM_CUDA(launch_scatter_pairs(kind, geo->dev.view, T, kind == kScatterCrystal ? bmc : bmh, P.perm, c0, c1,
                                         static_cast<float4*>(pair.p), s));
            ScatterParams Q = P;
            Q.kind = kind;
            Q.rank0 = c0;
            Q.rank1 = c1;
            Q.pair = static_cast<const float4*>(pair.p);
            Q.pair_r0 = c0;
            Q.pair_ld = c1 - c0;
            Q.accumulate = (written || spec.accumulate) ? 1 : 0;
            // scattered row lists: voxels on the lanes (same results)
            if (spec.rows && kind == kScatterCrystal) SM_CUDA(launch_scatter_rows(Q, geo->dev.view, T, s));
            else SM_CUDA(launch_scatter_main(Q, geo->dev.view, T, s));
        }
        written = true;
    }
    if (!written && !spec.accumulate) {
        const int64_t vox = spec.d_cols ? (int64_t)spec.n_cols * g.ny : (int64_t)g.nx * g.ny * g.nz;
        if (spec.rows && spec.rows_in_place) {
            for (int d : *spec.rows) SM_CUDA(cudaMemsetAsync(d_dst + (int64_t)d * ld, 0, sizeof(float) * (size_t)vox, s));
        } else {
            SM_CUDA(cudaMemset2DAsync(d_dst, sizeof(float) * (size_t)ld, 0, sizeof(float) * (size_t)vox,
                                      (size_t)(row1 - row0), s));
        }
    }
    return SM_OK;
}

int crystal_pair_table(const sm_geometry* geo, const int sp[3], DevBuf* table, std::vector<int>* order, DevBuf* d_order,
                       cudaStream_t s) {
    const HostGeometry& g = geo->host;
    const int N = g.n_crystals;
    HostScatterTables H;
    SM_TRY(build_scatter_tables(g, sp, &H));
    DevBuf tables;
    ScatterTables T;
    SM_TRY(upload_tables(H, N, holes0_of(g), s, &tables, &T));
    *order = spatial_order(g, 0, N);
    SM_TRY(d_order->alloc(sizeof(int) * (size_t)N, s, "detector order"));
    SM_CUDA(cudaMemcpyAsync(d_order->p, order->data(), sizeof(int) * (size_t)N, cudaMemcpyHostToDevice, s));
    DevBuf bm;
    const int64_t w = crystal_bitmap_words(N);
    SM_TRY(bm.alloc(sizeof(uint32_t) * (size_t)w, s, "crystal bitmap"));
    SM_CUDA(launch_bitmap_crystal(static_cast<uint32_t*>(bm.p), w, T, s));
    const size_t n_src = (size_t)N * T.n_points;
    SM_TRY(table->alloc(sizeof(float4) * n_src * (size_t)N, s, "crystal pair table"));
    SM_CUDA(launch_scatter_pairs(kScatterCrystal, geo->dev.view, T, static_cast<const uint32_t*>(bm.p),
                                 static_cast<const int*>(d_order->p), 0, N, static_cast<float4*>(table->p), s));
    SM_CUDA(cudaStreamSynchronize(s));   // the host tables are released on return
    return SM_OK;
}

int scatter_transfer(const sm_geometry* geo, const int sp[3], float angle, const float4* d_vbar, int n_anchors, void* d_K,
                     int64_t ldk, bool k_bf16, const float4* pairs, const int* d_order, cudaStream_t s) {
    const HostGeometry& g = geo->host;
    const int N = g.n_crystals;
    HostScatterTables H;
    SM_TRY(build_scatter_tables(g, sp, &H));
    DevBuf tables;
    ScatterTables T;
    SM_TRY(upload_tables(H, N, holes0_of(g), s, &tables, &T));
    ScatterParams P{};
    fill_common(g, 0, angle, &P);
    P.kind = kScatterCrystal;
    if (pairs) {
        P.perm = d_order;
        P.rank0 = 0;
        P.rank1 = N;
        P.pair = pairs;
        P.pair_r0 = 0;
        P.pair_ld = N;
        SM_CUDA(launch_scatter_transfer(P, geo->dev.view, T, d_vbar, n_anchors, d_K, k_bf16, ldk, (long long)N * ldk, s));
        SM_CUDA(cudaStreamSynchronize(s));
        return SM_OK;
    }
    std::vector<int> ident(N);
    for (int i = 0; i < N; ++i) ident[i] = i;
    DevBuf perm, bm;
    SM_TRY(perm.alloc(sizeof(int) * (size_t)N, s, "detector order"));
    SM_CUDA(cudaMemcpyAsync(perm.p, ident.data(), sizeof(int) * (size_t)N, cudaMemcpyHostToDevice, s));
    SM_CUDA(cudaStreamSynchronize(s));
    P.perm = static_cast<const int*>(perm.p);
    const int64_t w = crystal_bitmap_words(N);
    SM_TRY(bm.alloc(sizeof(uint32_t) * (size_t)w, s, "crystal bitmap"));
    SM_CUDA(launch_bitmap_crystal(static_cast<uint32_t*>(bm.p), w, T, s));
    const int n_src = N * T.n_points;
    int chunk = (int)std::max<size_t>(128, kPairBudget / (sizeof(float4) * (size_t)std::max(1, n_src)));
    chunk = std::max(128, chunk / 128 * 128);
    DevBuf pair;
    SM_TRY(pair.alloc(sizeof(float4) * (size_t)n_src * (size_t)std::min(chunk, N), s, "scatter pairs"));
    for (int c0 = 0; c0 < N; c0 += chunk) {
        const int c1 = std::min(N, c0 + chunk);
        SM_CUDA(launch_scatter_pairs(kScatterCrystal, geo->dev.view, T, static_cast<const uint32_t*>(bm.p), P.perm, c0, c1,
                                     static_cast<float4*>(pair.p), s));
        ScatterParams Q = P;
        Q.rank0 = c0;
        Q.rank1 = c1;
        Q.pair = static_cast<const float4*>(pair.p);
        Q.pair_r0 = c0;
        Q.pair_ld = c1 - c0;
        void* kc = static_cast<char*>(d_K) + (size_t)c0 * (size_t)ldk * (k_bf16 ? 2 : 4);
        SM_CUDA(launch_scatter_transfer(Q, geo->dev.view, T, d_vbar, n_anchors, kc, k_bf16, ldk, (long long)N * ldk, s));
    }
    SM_CUDA(cudaStreamSynchronize(s));
    return SM_OK;
}

namespace {

int read_words(const char* path, std::vector<uint32_t>* out, int64_t n) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(SM_ERR_IO, "cannot open bitmap file %s", path);
    out->assign((size_t)n, 0u);
    const size_t got = std::fread(out->data(), sizeof(uint32_t), (size_t)n, f);
    std::fclose(f);
    if ((int64_t)got != n) return fail(SM_ERR_IO, "bitmap file %s holds %zu of %lld words", path, got, (long long)n);
    return SM_OK;
}

int write_words(const char* path, const std::vector<uint32_t>& w) {
    FILE* f = std::fopen(path, "wb+");
    if (!f) return fail(SM_ERR_IO, "cannot create bitmap file %s", path);
    const size_t put = std::fwrite(w.data(), sizeof(uint32_t), w.size(), f);
    std::fclose(f);
    if (put != w.size()) return fail(SM_ERR_IO, "short write to %s", path);
    return SM_OK;
}

// ---- geometry hashes of the bitmap files ------------------------------------
// A bitmap file holds no record of the geometry it was computed for, so the
// reference reuses a stale -GeoCrystal / -GeoCollimator file after the tables
// change.  Next to each file this library writes "<file>.geohash": one line
// naming the bitmap kind, its word count and a 64-bit FNV-1a hash of every
// table value the bitmap depends on.  Reading a bitmap whose .geohash names
// another geometry recomputes it (and refreshes both files); a bitmap without
// .geohash (written by the reference) is read as the reference reads it.

uint64_t fnv1a(const void* data, size_t n, uint64_t h) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 0x100000001b3ULL;
    }
    return h;
}

// out[0]: crystal bitmap (detector records and the FOV distance);
// out[1]: collimator bitmap (plate 0's record and holes, detector, FOV distance).
void bitmap_hashes(const HostGeometry& g, uint64_t out[2]) {
    const uint64_t seed = 0xcbf29ce484222325ULL;
    const size_t n_det = 1 + 12 * (size_t)g.n_crystals;
    uint64_t hd = fnv1a("crystal-bitmap-v1", 17, seed);
    hd = fnv1a(g.detector.data(), sizeof(float) * n_det, hd);
    hd = fnv1a(&g.image[11], sizeof(float), hd);
    out[0] = hd;
    const int h0 = holes0_of(g);
    uint64_t hh = fnv1a("collimator-bitmap-v1", 20, seed);
    if (g.collimator.size() >= 18) hh = fnv1a(&g.collimator[10], sizeof(float) * 8, hh);
    hh = fnv1a(&h0, sizeof(h0), hh);
    if (h0 > 0) hh = fnv1a(&g.collimator[100], sizeof(float) * 9 * (size_t)h0, hh);
    hh = fnv1a(g.detector.data(), sizeof(float) * n_det, hh);
    hh = fnv1a(&g.image[11], sizeof(float), hh);
    out[1] = hh;
}

std::string hash_line(const char* kind, int64_t words, uint64_t hash) {
    char buf[128];
    std::snprintf(buf, sizeof(buf), "sysmat_b200-bitmap-v1 %s words=%lld fnv1a64=%016llx\n", kind, (long long)words,
                  (unsigned long long)hash);
    return buf;
}

int write_hash_file(const char* bitmap_path, const std::string& line) {
    const std::string path = std::string(bitmap_path) + ".geohash";
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return fail(SM_ERR_IO, "cannot create %s", path.c_str());
    const bool ok = std::fwrite(line.data(), 1, line.size(), f) == line.size();
    std::fclose(f);
    return ok ? SM_OK : fail(SM_ERR_IO, "short write to %s", path.c_str());
}

// 1: the .geohash file exists and names this geometry; 0: it names another
// one; -1: there is none.
int hash_file_matches(const char* bitmap_path, const std::string& line) {
    const std::string path = std::string(bitmap_path) + ".geohash";
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return -1;
    char buf[256] = {0};
    const size_t got = std::fread(buf, 1, sizeof(buf) - 1, f);
    std::fclose(f);
    return (got == line.size() && std::memcmp(buf, line.data(), got) == 0) ? 1 : 0;
}

int validate_scatter(const sm_geometry* geo, const sm_scatter_options* opt, int row0, int row1) {
    for (int a = 0; a < 3; ++a)
        if (opt->sp[a] < 1 || opt->sp[a] > 16) return fail(SM_ERR_INVALID, "sp[%d] = %d must be in 1..16", a, opt->sp[a]);
    if ((opt->parts & ~3) || !opt->parts) return fail(SM_ERR_INVALID, "parts = %d: use 1 (crystal), 2 (collimator) or 3", opt->parts);
    const HostGeometry& g = geo->host;
    if (row0 < 0 || row1 > g.n_crystals || row0 >= row1)
        return fail(SM_ERR_INVALID, "row range [%d, %d) outside [0, %d)", row0, row1, g.n_crystals);
    if (!(g.physics[7] > 0.0f)) return fail(SM_ERR_INVALID, "Physics[7] (photon energy, keV) must be > 0");
    if ((int64_t)g.n_crystals * opt->sp[0] * opt->sp[1] * opt->sp[2] > (1 << 26))
        return fail(SM_ERR_CAPACITY, "too many scatter points");
    return SM_OK;
}

}  // namespace
}  // namespace smb

using namespace smb;

extern "C" {

int sm_scatter_subset(sm_context* ctx, const sm_geometry* geo, const sm_scatter_options* opt, int rotation,
                      const float* pe, int64_t ld_pe, const int32_t* rows, int n_rows, const int32_t* cols, int n_cols,
                      float* dst, int64_t ld, void* stream_ptr) {
    if (!geo || !opt || !dst || !rows || n_rows <= 0) return fail(SM_ERR_INVALID, "null argument or empty row list");
    SM_TRY(context_bind(ctx));
    SM_TRY(validate_scatter(geo, opt, 0, geo->host.n_crystals));
    const HostGeometry& g = geo->host;
    const int64_t V = (int64_t)g.nx * g.ny * g.nz;
    if ((opt->parts & 1) && (!pe || ld_pe < V)) return fail(SM_ERR_INVALID, "crystal scatter needs the PE sysmat with ld_pe >= %lld", (long long)V);
    const int64_t width = cols ? (int64_t)n_cols * g.ny : V;
    if (cols && n_cols <= 0) return fail(SM_ERR_INVALID, "empty column list");
    if (ld < width) return fail(SM_ERR_INVALID, "ld = %lld is smaller than the %lld output columns", (long long)ld, (long long)width);
    cudaStream_t s = (cudaStream_t)stream_ptr;
    std::vector<int> list(rows, rows + n_rows);
    ExactSpec spec;
    spec.rows = &list;
    DevBuf cb;
    if (cols) {
        for (int c = 0; c < n_cols; ++c)
            if (cols[2 * c] < 0 || cols[2 * c] >= g.nx || cols[2 * c + 1] < 0 || cols[2 * c + 1] >= g.nz)
                return fail(SM_ERR_INVALID, "column %d (%d, %d) is outside the %d x %d grid", c, cols[2 * c], cols[2 * c + 1], g.nx, g.nz);
        SM_TRY(cb.alloc(sizeof(int2) * (size_t)n_cols, s, "column list"));
        SM_CUDA(cudaMemcpyAsync(cb.p, cols, sizeof(int2) * (size_t)n_cols, cudaMemcpyHostToDevice, s));
        spec.d_cols = static_cast<const int2*>(cb.p);
        spec.n_cols = n_cols;
    }
    const float angle = (float)rotation * g.angle_per_rotation;
    return exact_scatter(geo, opt->sp, opt->parts, angle, (opt->parts & 1) ? pe : nullptr, ld_pe, nullptr, nullptr, spec,
                         dst, ld, s);
}

int sm_scatter_transfer(sm_context* ctx, const sm_geometry* geo, const sm_scatter_options* opt, int rotation,
                        const float* vbar, int n_anchors, float* K, int64_t ldk, void* stream) {
    if (!geo || !opt || !vbar || !K || n_anchors <= 0) return fail(SM_ERR_INVALID, "null argument or no anchors");
    SM_TRY(context_bind(ctx));
    SM_TRY(validate_scatter(geo, opt, 0, geo->host.n_crystals));
    if (ldk < geo->host.n_crystals) return fail(SM_ERR_INVALID, "ldk = %lld is smaller than N = %d", (long long)ldk, geo->host.n_crystals);
    const float angle = (float)rotation * geo->host.angle_per_rotation;
    return scatter_transfer(geo, opt->sp, angle, reinterpret_cast<const float4*>(vbar), n_anchors, K, ldk, false, nullptr,
                            nullptr, (cudaStream_t)stream);
}

void sm_scatter_options_reference(sm_scatter_options* opt) {
    if (!opt) return;
    std::memset(opt, 0, sizeof(*opt));
    opt->sp[0] = opt->sp[1] = opt->sp[2] = 1;
    opt->parts = 3;
}

int sm_scatter_bitmap_words(const sm_geometry* geo, int64_t out[2]) {
    if (!geo || !out) return fail(SM_ERR_INVALID, "null argument");
    out[0] = crystal_bitmap_words(geo->host.n_crystals);
    out[1] = collimator_bitmap_words(geo->host.n_crystals, holes0_of(geo->host));
    return SM_OK;
}

int sm_scatter_bitmap_hashes(const sm_geometry* geo, uint64_t out[2]) {
    if (!geo || !out) return fail(SM_ERR_INVALID, "null argument");
    bitmap_hashes(geo->host, out);
    return SM_OK;
}

int sm_scatter_bitmaps(sm_context* ctx, const sm_geometry* geo, uint32_t* crystal, uint32_t* collimator, int on_device,
                       void* stream_ptr) {
    if (!geo) return fail(SM_ERR_INVALID, "null geometry");
    SM_TRY(context_bind(ctx));
    cudaStream_t s = (cudaStream_t)stream_ptr;
    const HostGeometry& g = geo->host;
    const int h0 = holes0_of(g);
    const int sp[3] = {1, 1, 1};
    HostScatterTables H;
    SM_TRY(build_scatter_tables(g, sp, &H));
    DevBuf tables;
    ScatterTables T;
    SM_TRY(upload_tables(H, g.n_crystals, h0, s, &tables, &T));
    const int64_t wc = crystal_bitmap_words(g.n_crystals), wh = collimator_bitmap_words(g.n_crystals, h0);
    if (crystal) {
        DevBuf tmp;
        uint32_t* d = crystal;
        if (!on_device) {
            SM_TRY(tmp.alloc(sizeof(uint32_t) * (size_t)wc, s, "crystal bitmap"));
            d = static_cast<uint32_t*>(tmp.p);
        }
        SM_CUDA(launch_bitmap_crystal(d, wc, T, s));
        if (!on_device) {
            SM_CUDA(cudaMemcpyAsync(crystal, d, sizeof(uint32_t) * (size_t)wc, cudaMemcpyDeviceToHost, s));
            SM_CUDA(cudaStreamSynchronize(s));
        }
    }
    if (collimator && wh > 0) {
        DevBuf tmp;
        uint32_t* d = collimator;
        if (!on_device) {
            SM_TRY(tmp.alloc(sizeof(uint32_t) * (size_t)wh, s, "collimator bitmap"));
            d = static_cast<uint32_t*>(tmp.p);
        }
        SM_CUDA(launch_bitmap_collimator(d, wh, T, s));
        if (!on_device) {
            SM_CUDA(cudaMemcpyAsync(collimator, d, sizeof(uint32_t) * (size_t)wh, cudaMemcpyDeviceToHost, s));
            SM_CUDA(cudaStreamSynchronize(s));
        }
    }
    return SM_OK;
}

int sm_scatter_compute(sm_context* ctx, const sm_geometry* geo, const sm_scatter_options* opt, int rotation,
                       const float* pe, int64_t ld_pe, int pe_on_device, const uint32_t* crystal_bitmap,
                       const uint32_t* collimator_bitmap, int bitmaps_on_device, int row0, int row1, float* dst,
                       int64_t ld, int dst_on_device, void* stream_ptr) {
    if (!geo || !opt || !dst) return fail(SM_ERR_INVALID, "null argument");
    SM_TRY(context_bind(ctx));
    SM_TRY(validate_scatter(geo, opt, row0, row1));
    const HostGeometry& g = geo->host;
    const int N = g.n_crystals;
    const int64_t V = (int64_t)g.nx * g.ny * g.nz;
    if (ld < V) return fail(SM_ERR_INVALID, "ld = %lld is smaller than the %lld voxels", (long long)ld, (long long)V);
    if ((opt->parts & 1) && !pe) return fail(SM_ERR_INVALID, "crystal scatter needs the PE sysmat");
    if ((opt->parts & 1) && ld_pe < V) return fail(SM_ERR_INVALID, "ld_pe = %lld is smaller than the %lld voxels", (long long)ld_pe, (long long)V);
    cudaStream_t s = (cudaStream_t)stream_ptr;
    const float angle = (float)rotation * g.angle_per_rotation;
    const int h0 = holes0_of(g);

    DevBuf pe_buf, bmc_buf, bmh_buf, out_buf;
    const float* d_pe = nullptr;
    if (opt->parts & 1) {
        if (pe_on_device) d_pe = pe;
        else {
            SM_TRY(pe_buf.alloc(sizeof(float) * (size_t)N * (size_t)ld_pe, s, "PE sysmat"));
            SM_CUDA(cudaMemcpyAsync(pe_buf.p, pe, sizeof(float) * (size_t)N * (size_t)ld_pe, cudaMemcpyHostToDevice, s));
            d_pe = static_cast<const float*>(pe_buf.p);
        }
    }
    const uint32_t* d_bmc = nullptr;
    const uint32_t* d_bmh = nullptr;
    if (crystal_bitmap) {
        if (bitmaps_on_device) d_bmc = crystal_bitmap;
        else {
            const size_t b = sizeof(uint32_t) * (size_t)crystal_bitmap_words(N);
            SM_TRY(bmc_buf.alloc(b, s, "crystal bitmap"));
            SM_CUDA(cudaMemcpyAsync(bmc_buf.p, crystal_bitmap, b, cudaMemcpyHostToDevice, s));
            d_bmc = static_cast<const uint32_t*>(bmc_buf.p);
        }
    }
    if (collimator_bitmap && h0 > 0) {
        if (bitmaps_on_device) d_bmh = collimator_bitmap;
        else {
            const size_t b = sizeof(uint32_t) * (size_t)collimator_bitmap_words(N, h0);
            SM_TRY(bmh_buf.alloc(b, s, "collimator bitmap"));
            SM_CUDA(cudaMemcpyAsync(bmh_buf.p, collimator_bitmap, b, cudaMemcpyHostToDevice, s));
            d_bmh = static_cast<const uint32_t*>(bmh_buf.p);
        }
    }
    float* d_dst = dst;
    const int rows = row1 - row0;
    if (!dst_on_device) {
        SM_TRY(out_buf.alloc(sizeof(float) * (size_t)rows * (size_t)ld, s, "scatter output"));
        d_dst = static_cast<float*>(out_buf.p);
    }
    ExactSpec spec;
    spec.row0 = row0;
    spec.row1 = row1;
    SM_TRY(exact_scatter(geo, opt->sp, opt->parts, angle, d_pe, ld_pe, d_bmc, d_bmh, spec, d_dst, ld, s));
    if (!dst_on_device) {
        SM_CUDA(cudaMemcpyAsync(dst, d_dst, sizeof(float) * (size_t)rows * (size_t)ld, cudaMemcpyDeviceToHost, s));
    }
    if (!dst_on_device || !pe_on_device || (crystal_bitmap && !bitmaps_on_device)) SM_CUDA(cudaStreamSynchronize(s));
    return SM_OK;
}

// The reference's three `scatter` entry points in one: parts 3 = both
// (ScatterGen_RayTracing_CircularHole), 1 = crystal only (ScatterGen_Crystal,
// geo_crystal = its FnameGeo), 2 = collimator only (ScatterGen_Collimator,
// geo_collimator = its FnameGeo).  Physics[8] / Physics[9] == 1 compute the
// bitmaps and write the files, otherwise the files are read.
int sm_scatter_legacy(int parts, float* parameter_Collimator, float* parameter_Detector, float* parameter_Image,
                      float* parameter_Physics, float* PE_SysMat, const char* geo_crystal, const char* geo_collimator,
                      float* dst, int cuda_id) {
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    sm_context* ctx = legacy_context(cuda_id);
    if (!ctx) return fail(SM_ERR_DEVICE, "no usable device: %s", sm_last_error());
    std::vector<float> empty_col(100, 0.0f);
    const float* col = parameter_Collimator ? parameter_Collimator : empty_col.data();
    const size_t n_col = parameter_Collimator ? 80000 : 100;
    sm_geometry* geo = nullptr;
    SM_TRY(sm_geometry_create(ctx, col, n_col, parameter_Detector, 80000, parameter_Image, 100, parameter_Physics, 100,
                              &geo));
    struct GeoGuard {
        sm_geometry* g;
        ~GeoGuard() { sm_geometry_destroy(g); }
    } guard{geo};
    const HostGeometry& g = geo->host;
    const int N = g.n_crystals;
    const int64_t V = (int64_t)g.nx * g.ny * g.nz;
    int64_t words[2];
    sm_scatter_bitmap_words(geo, words);
    uint64_t hashes[2];
    bitmap_hashes(g, hashes);
    std::vector<uint32_t> bmc, bmh;
    if (parts & 1) {
        if (!geo_crystal) return fail(SM_ERR_INVALID, "crystal bitmap file name is required");
        const std::string line = hash_line("crystal", words[0], hashes[0]);
        const bool compute = (int)std::floor(parameter_Physics[8]) == 1;
        const int match = compute ? -1 : hash_file_matches(geo_crystal, line);
        if (compute || match == 0) {
            if (match == 0)
                std::fprintf(stderr, "scatter: %s was computed for another geometry (%s.geohash); recomputing it\n",
                             geo_crystal, geo_crystal);
            bmc.assign((size_t)words[0], 0u);
            SM_TRY(sm_scatter_bitmaps(ctx, geo, bmc.data(), nullptr, 0, nullptr));
            SM_TRY(write_words(geo_crystal, bmc));
            SM_TRY(write_hash_file(geo_crystal, line));
        } else {
            SM_TRY(read_words(geo_crystal, &bmc, words[0]));
        }
    }
    if ((parts & 2) && words[1] > 0) {
        if (!geo_collimator) return fail(SM_ERR_INVALID, "collimator bitmap file name is required");
        const std::string line = hash_line("collimator", words[1], hashes[1]);
        const bool compute = (int)std::floor(parameter_Physics[9] + 0.001f) == 1;
        const int match = compute ? -1 : hash_file_matches(geo_collimator, line);
        if (compute || match == 0) {
            if (match == 0)
                std::fprintf(stderr, "scatter: %s was computed for another geometry (%s.geohash); recomputing it\n",
                             geo_collimator, geo_collimator);
            bmh.assign((size_t)words[1], 0u);
            SM_TRY(sm_scatter_bitmaps(ctx, geo, nullptr, bmh.data(), 0, nullptr));
            SM_TRY(write_words(geo_collimator, bmh));
            SM_TRY(write_hash_file(geo_collimator, line));
        } else {
            SM_TRY(read_words(geo_collimator, &bmh, words[1]));
        }
    }
    sm_scatter_options opt;
    sm_scatter_options_reference(&opt);
    opt.parts = parts;
    // The kernels rotate the image by Image[20] * Image[7] (scatter.cu:1107-1110).
    SM_TRY(context_bind(ctx));
    const float angle = parameter_Image[20] * parameter_Image[7];
    std::vector<float> out((size_t)N * (size_t)V, 0.0f);
    {
        DevBuf pe_buf, bmc_buf, bmh_buf, out_buf;
        cudaStream_t s = nullptr;
        SM_TRY(validate_scatter(geo, &opt, 0, N));
        const float* d_pe = nullptr;
        if (parts & 1) {
            SM_TRY(pe_buf.alloc(sizeof(float) * (size_t)N * (size_t)V, s, "PE sysmat"));
            SM_CUDA(cudaMemcpyAsync(pe_buf.p, PE_SysMat, sizeof(float) * (size_t)N * (size_t)V, cudaMemcpyHostToDevice, s));
            d_pe = static_cast<const float*>(pe_buf.p);
        }
        const uint32_t* d_bmc = nullptr;
        const uint32_t* d_bmh = nullptr;
        if (!bmc.empty()) {
            SM_TRY(bmc_buf.alloc(sizeof(uint32_t) * bmc.size(), s, "crystal bitmap"));
            SM_CUDA(cudaMemcpyAsync(bmc_buf.p, bmc.data(), sizeof(uint32_t) * bmc.size(), cudaMemcpyHostToDevice, s));
            d_bmc = static_cast<const uint32_t*>(bmc_buf.p);
        }
        if (!bmh.empty()) {
            SM_TRY(bmh_buf.alloc(sizeof(uint32_t) * bmh.size(), s, "collimator bitmap"));
            SM_CUDA(cudaMemcpyAsync(bmh_buf.p, bmh.data(), sizeof(uint32_t) * bmh.size(), cudaMemcpyHostToDevice, s));
            d_bmh = static_cast<const uint32_t*>(bmh_buf.p);
        }
        SM_TRY(out_buf.alloc(sizeof(float) * (size_t)N * (size_t)V, s, "scatter output"));
        float* d_out = static_cast<float*>(out_buf.p);
        ExactSpec spec;
        spec.row0 = 0;
        spec.row1 = N;
        SM_TRY(exact_scatter(geo, opt.sp, parts, angle, d_pe, V, d_bmc, d_bmh, spec, d_out, V, s));
        SM_CUDA(cudaMemcpyAsync(out.data(), d_out, sizeof(float) * out.size(), cudaMemcpyDeviceToHost, s));
        SM_CUDA(cudaStreamSynchronize(s));
    }
    std::memcpy(dst, out.data(), sizeof(float) * out.size());
    return (int)V;
}

// ScatterGen_RayTracing_CircularHole/scatter.h:4-5.
int scatter(float* parameter_Collimator, float* parameter_Detector, float* parameter_Image, float* parameter_Physics,
            float* PE_SysMat, const char* FnameGeoCrystal, const char* FnameGeoCollimator, float* dst, int cuda_id) {
    if (!parameter_Collimator || !parameter_Detector || !parameter_Image || !parameter_Physics || !PE_SysMat || !dst) {
        std::fprintf(stderr, "scatter: null argument\n");
        return -1;
    }
    const int rc = sm_scatter_legacy(3, parameter_Collimator, parameter_Detector, parameter_Image, parameter_Physics,
                                     PE_SysMat, FnameGeoCrystal, FnameGeoCollimator, dst, cuda_id);
    if (rc < 0) {
        std::fprintf(stderr, "scatter: %s\n", sm_last_error());
        return -1;
    }
    return rc;
}

}  // extern "C"
