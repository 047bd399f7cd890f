// Primary-Compton scatter sysmat: device tables, launch parameters, launchers.
//
// The reference computes every (detector, voxel, scatter source) term in one
// thread and scans all N crystals of a bitmap inside it
// (ScatterGen_RayTracing_CircularHole/scatter.cu:1077-1437, :1544-1936).  Here
// the work is split by what each quantity depends on:
//   * bitmap words (crystal i, j, k / hole i, crystal j, k), one thread per
//     32-bit word, the reference's single-precision test;
//   * per (scatter point, detector): the bitmap-gated attenuation sums
//     sum_k L_k mu_pe_k and sum_k L_k mu_c_k (the path does not depend on the
//     voxel, and mu(E') = mu_pe (E0/E')^3 + mu_c (E0/E') factors out), the
//     path inside the detecting crystal and the absorption chord;
//   * per (detector, voxel, scatter point): the cone angle, the energy
//     window, the azimuth and polar ranges and the Klein-Nishina fraction.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "geometry.h"
#include "common.h"
#include "sysmat_b200.h"

namespace smb {

constexpr int kKnNodes = 512;            // Klein-Nishina table: nodes j * pi / 512, j = 0..512
constexpr int kScTileD = 32;             // detectors per CTA (one per lane)
constexpr int kScBrickX = 8;             // voxel brick: 8 (x) x 32 (y) x 1 (z); one x column per warp
constexpr int kScBrickY = 32;
constexpr int kScWarps = 8;
constexpr int kScThreads = 32 * kScWarps;

// One node of the Klein-Nishina table: the expansion point theta_j (a float),
// F(theta_j) = integral_0^theta_j g as a float pair, and the Taylor
// coefficients of g(theta) = KN(theta) sin(theta) at theta_j.
struct __align__(16) KnNode {
    float theta, f_hi, f_lo, c0;
    float c1, c2, c3, c4;
};

// Device tables of one geometry for the scatter kernels.
struct ScatterTables {
    const float4* crystal_raw;   // x, y (table value, without Image[11]), z, bounding radius R
    const float4* hole_raw;      // layer-0 hole centre x, (y1 + y2) / 2 (table values), z, 0
    const float4* hole_src;      // layer-0 hole scatter point x, (y1 + y2) / 2 + Image[11], z, y2 - y1
    const float4* crystal_src;   // scatter points of every crystal, [crystal][point]: world x, y, z, 0
    const KnNode* kn;            // kKnNodes + 1 nodes
    int n_crystals;
    int n_holes0;                // holes of plate 0 (Collimator[10])
    int n_points;                // scatter points per crystal
    float kn_inv_norm;           // 1 / (rectangle sum of g over [0, pi], as the reference normalises)
};

enum : int { kScatterCrystal = 0, kScatterCollimator = 1 };

struct ScatterParams {
    int kind;
    // image
    int nx, ny, nz;
    float vx, vy, vz, shx, shy, shz, cos_a, sin_a;
    // physics
    float e0, alpha;             // keV, E0 / 511
    int use_compton, same_window;
    float win_lo, win_hi;        // Physics[5], Physics[6]
    // collimator-scatter weight: mu_compton / mu_total of plate 0 (Collimator[17] / Collimator[15])
    float plate_c_over_t;
    // detectors: perm[r] for ranks r in [rank0, rank1); perm orders the requested
    // rows so that 32 consecutive ranks are spatially close (depth layer, then a
    // Morton curve over x, z); dst row of detector d is d - dst_row0
    const int* perm;
    int rank0, rank1;
    int dst_row0;
    // bricks
    int bricks_x, bricks_y, n_bricks;
    // voxel subset: when cols is set, the voxels are the y-columns (x, z) = cols[i]
    // (bricks of 8 columns x 32 y) and output column of (i, y) is i * ny + y
    const int2* cols;
    int n_cols;
    const int* slot;             // when set: dst row of rank r is slot[r] (row-list mode)
    const int* pair_col;         // when set: pair column of rank r is pair_col[r] (shared pair table)
    // inputs
    const float* pe;             // crystal kind: [N][ld_pe] photoelectric sysmat of the rotation
    long long ld_pe;
    const uint32_t* brick_sources;   // crystal kind: [n_bricks][ceil(N/32)] sources with PE != 0 in the brick
    int src_words;
    const float4* pair;          // [source point][pair_ld]: sum L mu_pe, sum L mu_c, self path, absorption chord
    int pair_r0;                 // rank of pair column 0
    long long pair_ld;
    // output
    float* dst;
    long long ld;
    int accumulate;              // 1: dst += result, 0: dst = result
};

// Host-built tables (see scatter_host.cpp).
struct HostScatterTables {
    std::vector<float> crystal_raw, hole_raw, hole_src, crystal_src;
    std::vector<KnNode> kn;
    int n_points = 1;
    int sp[3] = {1, 1, 1};
    float kn_inv_norm = 0.0f;
};

int build_scatter_tables(const HostGeometry& g, const int sp[3], HostScatterTables* out);

// Bitmap sizes in 32-bit words (scatter.cu:2053-2056, :2225-2229).
int64_t crystal_bitmap_words(int n_crystals);
int64_t collimator_bitmap_words(int n_crystals, int n_holes0);

cudaError_t launch_bitmap_crystal(uint32_t* words, int64_t n_words, const ScatterTables& T, cudaStream_t s);
cudaError_t launch_bitmap_collimator(uint32_t* words, int64_t n_words, const ScatterTables& T, cudaStream_t s);
// pair[q][r - r0] for every source point q of `kind` and detectors perm[r], r in [r0, r1).
cudaError_t launch_scatter_pairs(int kind, const DevGeometry& G, const ScatterTables& T, const uint32_t* bitmap,
                                 const int* perm, int r0, int r1, float4* pair, cudaStream_t s);

// Ranks of detectors [row0, row1) (or of the listed ones) in spatial order (see ScatterParams::perm).
std::vector<int> spatial_order(const HostGeometry& g, int row0, int row1);
std::vector<int> spatial_order_of(const HostGeometry& g, const std::vector<int>& ids);

// Which rows and voxels exact_scatter computes:
//  * rows: [row0, row1) with dst row d - row0, or the listed (distinct)
//    detectors with dst row i for detector (*rows)[i];
//  * voxels: all (dst column = voxel index), or the y-columns (x, z) of the
//    device list d_cols (dst column = i * ny + y).
//  * rows_in_place: listed rows write dst row d itself instead of row i;
//  * accumulate: add to dst instead of overwriting it.
struct ExactSpec {
    int row0 = 0, row1 = 0;
    const std::vector<int>* rows = nullptr;
    bool rows_in_place = false;
    bool accumulate = false;
    // crystal pair table computed beforehand (crystal_pair_table) for every
    // detector, columns in spatial_order(0, N); null: computed here
    const float4* pairs = nullptr;
    const std::vector<int>* pairs_order = nullptr;
    const int2* d_cols = nullptr;
    int n_cols = 0;
};

int exact_scatter(const sm_geometry* geo, const int sp[3], int parts, float angle, const float* d_pe, int64_t ld_pe,
                  const uint32_t* d_bm_crystal, const uint32_t* d_bm_collimator, const ExactSpec& spec, float* d_dst,
                  int64_t ld, cudaStream_t s);
// K[a][d][s] (row pitch ldk, anchor pitch N * ldk) = crystal-scatter entry of
// detector d per unit PE of source s with the photon arriving from vbar[a][s]
// (fractional voxel indices in x, y, z; w > 0 marks a source in use), a < n_anchors.
// K is fp32, or bf16 when k_bf16.  With a shared pair table (pairs, its
// device order d_order = spatial_order(0, N)) row r of K is detector d_order[r];
// without one, row d is detector d.
int scatter_transfer(const sm_geometry* geo, const int sp[3], float angle, const float4* d_vbar, int n_anchors, void* d_K,
                     int64_t ldk, bool k_bf16, const float4* pairs, const int* d_order, cudaStream_t s);

// The crystal pair table of every detector: [N * points][N] float4, column r
// for detector (*order)[r], order = spatial_order(0, N) (also uploaded to d_order).
int crystal_pair_table(const sm_geometry* geo, const int sp[3], DevBuf* table, std::vector<int>* order, DevBuf* d_order,
                       cudaStream_t s);
cudaError_t launch_brick_sources(const ScatterParams& P, const ScatterTables& T, uint32_t* brick_sources,
                                 cudaStream_t s);
cudaError_t launch_scatter_transfer(const ScatterParams& P, const DevGeometry& G, const ScatterTables& T,
                                    const float4* vbar, int n_anchors, void* K, bool k_bf16, long long ldk,
                                    long long anchor_stride, cudaStream_t s);
cudaError_t launch_scatter_main(const ScatterParams& P, const DevGeometry& G, const ScatterTables& T,
                                cudaStream_t s);
// Crystal kind only, for row lists of scattered detectors (voxels on the lanes); same results.
cudaError_t launch_scatter_rows(const ScatterParams& P, const DevGeometry& G, const ScatterTables& T, cudaStream_t s);

}  // namespace smb
