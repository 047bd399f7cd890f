// Host planning for the PE kernel: fine grid, rotation, bricks and tiles.
//
// Compiled with -ffp-contract=off: the fine voxel size and the rotation's
// cos/sin must round as the reference's per-thread expressions do.
#include <algorithm>
#include <cmath>

#include "pe.h"

namespace smb {

int pe_auto_group(int depth_subcells) { return std::max(1, std::min(kMaxGroup, 32 / std::max(1, depth_subcells))); }

void pe_plan(const HostGeometry& g, const int sv[3], const int sc[3], const int brick[3], int group, int rotation,
             int row0, int row1, int nz_full, int z0, int nz, PEParams* p) {
    PEParams& P = *p;
    P = PEParams();
    P.nx = g.nx;
    P.ny = g.ny;
    P.nz = nz_full;
    P.z0 = z0;
    P.nzs = nz;
    P.kx = sv[0];
    P.ky = sv[1];
    P.kz = sv[2];
    P.fnx = g.nx * sv[0];
    P.fny = g.ny * sv[1];
    P.fnz = nz_full * sv[2];
    // Fine voxel = voxel / k in single precision: the reference run on the
    // k-times finer grid reads this value from its image table.
    P.fvx = g.voxel[0] / (float)sv[0];
    P.fvy = g.voxel[1] / (float)sv[1];
    P.fvz = g.voxel[2] / (float)sv[2];
    P.shx = g.shift[0];
    P.shy = g.shift[1];
    P.shz = g.shift[2];
    // RotationAngle = Image[20] * Image[7] (PESysMatGen.cu:404-406), then cos/sin.
    float angle = (float)rotation * g.angle_per_rotation;
    P.cos_a = std::cos(angle);
    P.sin_a = std::sin(angle);
    P.dX = sc[0];
    P.dY = sc[1];
    P.dZ = sc[2];
    P.n_sc = sc[0] * sc[1] * sc[2];
    P.n_sv = sv[0] * sv[1] * sv[2];
    P.group = group > 0 ? std::min(group, kMaxGroup) : pe_auto_group(P.dY);
    // Entries of at most 16 rays: VP neighbouring voxels form one group of
    // sub-points (VP * n_sv <= kMaxGroup), so that a warp pass traces one
    // sub-cell column from all of them.  The kernel sums each lane's rays for
    // one voxel, so the lane-to-point map must be the same in every pass: the
    // group's rays fit one pass, or a sub-cell column's rays (cb) divide 32.
    P.pair = 1;
    if (P.n_sv * P.n_sc <= 16) {
        for (int vp = 8; vp >= 2; vp >>= 1) {
            const int g = vp * P.n_sv, cb = g * P.dY;
            if (g <= kMaxGroup && (g * P.n_sc <= 32 || (cb <= 32 && 32 % cb == 0))) {
                P.pair = vp;
                break;
            }
        }
    }
    if (P.pair > 1) P.group = P.pair * P.n_sv;
    P.inv_sv = 1.0f / (float)P.n_sv;
    P.inv_n_sc = 1.0f / (float)P.n_sc;
    P.inv_dY = 1.0f / (float)P.dY;
    P.inv_dX = 1.0f / (float)P.dX;
    P.inv_kx = 1.0f / (float)P.kx;
    P.inv_ky = 1.0f / (float)P.ky;
    P.inv_kxky = 1.0f / (float)(P.kx * P.ky);
    P.inv_dXdY = 1.0f / (float)(P.dX * P.dY);
    P.row0 = row0;
    P.row1 = row1;
    int bx = brick[0] > 0 ? brick[0] : 8;
    int by = brick[1] > 0 ? brick[1] : 4;
    int bz = brick[2] > 0 ? brick[2] : 4;
    bx = std::min(bx, g.nx);
    by = std::min(by, g.ny);
    bz = std::min(bz, std::max(nz, 1));
    while (bx * by * bz > kMaxTileVoxels) {
        if (bz >= by && bz > 1) bz = (bz + 1) / 2;
        else if (by >= bx && by > 1) by = (by + 1) / 2;
        else bx = (bx + 1) / 2;
    }
    P.bx = bx;
    P.by = by;
    P.bz = bz;
    P.tiles_x = (g.nx + bx - 1) / bx;
    P.tiles_y = (g.ny + by - 1) / by;
    P.tiles_z = (nz + bz - 1) / bz;
    P.n_ctiles = (row1 - row0 + kPeWarps - 1) / kPeWarps;
    P.n_tiles = (long long)P.n_ctiles * P.tiles_x * P.tiles_y * P.tiles_z;
}

}  // namespace smb
