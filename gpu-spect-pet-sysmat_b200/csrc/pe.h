// Photoelectric sysmat kernel: launch parameters and host launcher.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "geometry.h"

namespace smb {

constexpr int kPeWarps = 8;            // warps per CTA = crystals per tile
constexpr int kPeThreads = 32 * kPeWarps;
constexpr int kSupC = 1024;            // tile superset capacity, crystals (beyond: the tile's voxels use the tables)
constexpr int kSupH = 384;             // tile superset capacity, holes
constexpr int kMaxGroup = 8;           // voxel sub-points whose candidate masks are live at once
constexpr int kMaxTileVoxels = 128;    // voxels per brick
constexpr int kListC = 512;            // per-voxel candidate list capacity, crystals (beyond: the voxel uses the tables)
constexpr int kListH = 128;            // per-voxel candidate list capacity, holes
constexpr int kMaxSubcellsPerAxis = 64;
constexpr int kRecHoles = 16;          // hit-record capacity per ray
constexpr int kRecCrystals = 40;
constexpr int kRecWords = 3 + kRecHoles + kRecCrystals;

// Bits of the device status word.  (Candidate sets larger than the shared-memory
// lists are not an error: those voxels are traced through the geometry tables.)
enum : int {
    kStatusRecordOverflow = 2,
};

struct PEParams {
    int nx, ny, nz;          // coarse grid (full volume)
    int z0, nzs;             // slab: coarse z range [z0, z0 + nzs)
    int kx, ky, kz;          // voxel sub-samples
    int fnx, fny, fnz;       // fine grid = coarse * k
    float fvx, fvy, fvz;     // fine voxel size = voxel / k (float division)
    float shx, shy, shz;     // FOV shift
    float cos_a, sin_a;      // image rotation about z
    int dX, dY, dZ;          // crystal sub-cells
    int n_sc, n_sv, group;   // sub-cells per crystal, sub-points per voxel, sub-points per mask group
    int pair;                // voxels per group of sub-points (1..8): > 1 when a voxel has at most 16 rays
    float inv_sv;
    // reciprocals for the division-free index decode (exact after one correction step)
    float inv_n_sc, inv_dY, inv_dX, inv_kx, inv_ky, inv_kxky, inv_dXdY;
    int row0, row1;          // crystal rows [row0, row1)
    int bx, by, bz;          // voxel brick
    int tiles_x, tiles_y, tiles_z;
    int n_ctiles;            // crystal tiles
    long long n_tiles;       // total tiles = n_ctiles * tiles_x * tiles_y * tiles_z
    const long long* tile_list;   // optional explicit tile ids (record mode)
    float* dst;
    long long ld;
    int* status;
    unsigned long long* counters; // optional: rays, exact crystal tests, exact hole tests, cone tests
    // record mode
    int rec_n;
    const long long* rec_rows;
    const long long* rec_vox;    // full-volume coarse voxel index
    int* rec_out;
};

// Fills every field of `p` but the output, status and record pointers, for the
// slab [z0, z0 + nz) of a volume of nz_full z-planes and rows [row0, row1).
// group: voxel sub-points whose candidate masks are computed together (0 =
// auto: 32 / depth sub-cells, so that one warp pass traces one column of
// sub-cells from `group` sub-points, at most kMaxGroup).  Within a group the
// rays are ordered (sub-cell column, sub-point, depth sub-cell) and dealt to
// the lanes in order; the group changes which lane sums which ray (the
// rounding of the sums), never a hit decision.
void pe_plan(const HostGeometry& g, const int sv[3], const int sc[3], const int brick[3], int group, int rotation,
             int row0, int row1, int nz_full, int z0, int nz, PEParams* p);
int pe_auto_group(int depth_subcells);

// Launches the trace kernel (RECORD selects the hit-recording instantiation).
cudaError_t pe_launch(const PEParams& p, const DevGeometry& geo, bool record, long long n_tiles, cudaStream_t stream);

size_t pe_smem_bytes();

// One geometry of a batch: its launch parameters, its tables, and the index
// of its first work item; items [tile_begin, tile_begin + P.n_tiles).
struct __align__(16) PeBatchGeom {
    PEParams P;
    DevGeometry G;
    long long tile_begin;
};

constexpr int kBatchConst = 64;   // geometries per persistent launch (constant-memory table)

// One persistent launch over `total` items of n_geoms <= kBatchConst
// geometries (device table `geoms`, ordered by tile_begin, first item 0):
// copies the table to constant memory, zeroes `counter`, launches.
cudaError_t pe_batch_launch(const PeBatchGeom* geoms, int n_geoms, long long total, unsigned long long* counter,
                            int grid, cudaStream_t stream);
int pe_batch_blocks_per_sm();

}  // namespace smb
