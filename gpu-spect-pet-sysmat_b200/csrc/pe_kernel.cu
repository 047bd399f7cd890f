// Photoelectric (PE) system-matrix kernel for sm_100a.
//
// Computes, for every crystal d and voxel v,
//   A[d, v] = 1/Sv * sum over voxel sub-points p and crystal sub-cells q of
//             exp(-sum mu*L along p->q) * Omega(p, q) * absorption(q)
// with the reference's physics and hit decisions
// (PEGen_RayTracing_CircularHole/PESysMatGen.cu:375-764): plate boxes a ray
// does not traverse block it (1e5 penalty), holes and other crystals count
// only when they are among the voxel's bounding-sphere candidates of the
// detecting crystal, the detecting crystal attenuates up to the sub-cell, and
// the sub-cell absorbs (1 - exp(-mu_t L)) mu_pe / mu_t.
//
// Work decomposition (one CTA per tile = 8 crystals x one voxel brick):
//  1. Tile cull: the CTA tests every crystal and hole against the bundle of
//     segments from the brick's sub-point box to each of its 8 crystals
//     (window_hit, conservative) and stages the survivors, ordered by id,
//     in shared memory.
//  2. Each warp owns one crystal and walks the brick's voxels, so its lanes
//     stay on nearby rays with the same candidates.  Per voxel sub-point the
//     warp evaluates the reference's exact cone test on the staged set
//     (after a per-sub-point window test) and keeps the result as ballot
//     bitmasks; lanes then trace one ray (sub-point, sub-cell) each.
//  3. Per ray, a window test against each candidate's box skips the exact
//     slab/cylinder test for candidates the ray cannot reach; the exact
//     tests are the reference's single-precision ones, so hits are
//     identical.  Skipped candidates would have contributed exactly 0.
//  4. Lanes accumulate with Kahan summation; warp shuffles reduce; the CTA
//     stages its 8 x brick results in shared memory and writes them out
//     row by row.
#include <cuda_runtime.h>

#include "pe.h"
#include "tracer.cuh"

namespace smb {

namespace {

constexpr int kMaskC = kSupC / 32;
constexpr int kMaskH = kSupH / 32;
constexpr int kMaskWords = kMaskC + kMaskH;
constexpr float kMargin = 0.01f;   // mm added around every culling box

struct __align__(16) PeSmem {
    float4 c_pos[kSupC];     // cx, cy, cz, mu_total
    float4 c_size[kSupC];    // w, t, h, crit
    float4 c_lo[kSupC];      // inflated world AABB
    float4 c_hi[kSupC];
    float2 c_rot[kSupC];     // cos(-rot), sin(-rot)
    int c_id[kSupC];
    float4 h_a[kSupH];       // x, y1, y2, z
    float4 h_b[kSupH];       // R, mu_total, crit, yc
    int h_id[kSupH];
    int h_plate_begin[kMaxPlates + 1];
    Box3 d_box[kPeWarps];    // inflated AABB of the tile's crystals
    int warp_cnt[kPeWarps];
    int n_c, n_h;
    unsigned int mask[kPeWarps][kMaxGroup][kMaskWords];
    float out[kPeWarps][kMaxTileVoxels];
};

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ Box3 point_box(const Vec3& p) { return Box3{p.x, p.y, p.z, p.x, p.y, p.z}; }

// Voxel sub-point in world coordinates: the reference's voxel centre on the
// fine grid (PESysMatGen.cu:438-449), fine index f = coarse * k + sub.
__device__ __forceinline__ Vec3 subpoint(const PEParams& P, int fx, int fy, int fz) {
    float xI = ((float)fx - (float)P.fnx / 2.0f + 0.5f) * P.fvx;
    float yI = ((float)fy - (float)P.fny / 2.0f + 0.5f) * P.fvy;
    float zI = ((float)fz - (float)P.fnz / 2.0f + 0.5f) * P.fvz;
    xI = xI + P.shx;
    yI = yI + P.shy;
    zI = zI + P.shz;
    Vec3 r;
    r.x = xI * P.cos_a - yI * P.sin_a;
    r.y = xI * P.sin_a + yI * P.cos_a;
    r.z = zI;
    return r;
}

__device__ __forceinline__ void subpoint_index(const PEParams& P, int ix, int iy, int iz, int s, int& fx, int& fy,
                                               int& fz) {
    int sx = s % P.kx;
    int sy = (s / P.kx) % P.ky;
    int sz = s / (P.kx * P.ky);
    fx = ix * P.kx + sx;
    fy = iy * P.ky + sy;
    fz = iz * P.kz + sz;
}

// Per-crystal constants of the warp's detecting crystal.
struct Detecting {
    int id;
    float cx, cy, cz, mu_t, mu_pe;
    float w, t, h, crit;
    float cm, sm, cp, sp;      // cos(-rot), sin(-rot), cos(rot), sin(rot)
    Box3 self_box;             // +-size/2 in its own frame
    Box3 world;                // inflated world AABB
    float area_x, area_z, area_y;   // sub-cell face areas (t*h/dZ/dY, w*t/dX/dY, w*h/dX/dZ)
};

// The reference's bounding-sphere candidate test of crystal k for the voxel
// point p and detecting crystal d (PESysMatGen.cu:506-551), bit-exact.
struct ConeSelf {
    float ux, uy, uz, crit_self;
};

__device__ __forceinline__ ConeSelf cone_self(const Detecting& D, const Vec3& p) {
    ConeSelf c;
    float dist = sqrtf((D.cy - p.y) * (D.cy - p.y) + (D.cx - p.x) * (D.cx - p.x) + (D.cz - p.z) * (D.cz - p.z));
    c.crit_self = D.crit / dist / 2.0f;
    c.ux = (D.cx - p.x) / dist;
    c.uy = (D.cy - p.y) / dist;
    c.uz = (D.cz - p.z) / dist;
    return c;
}

__device__ __forceinline__ bool cone_crystal(const ConeSelf& cs, const Vec3& p, float xk, float yk, float zk,
                                             float crit_k) {
    float dk = sqrtf((p.x - xk) * (p.x - xk) + (p.y - yk) * (p.y - yk) + (p.z - zk) * (p.z - zk));
    float crit = crit_k / dk / 2.0f;
    float ex = (xk - p.x) / dk, ey = (yk - p.y) / dk, ez = (zk - p.z) / dk;
    return sqrtf((ez - cs.uz) * (ez - cs.uz) + (ey - cs.uy) * (ey - cs.uy) + (ex - cs.ux) * (ex - cs.ux)) <=
           crit + cs.crit_self;
}

// Hole candidate test (PESysMatGen.cu:559-585), bit-exact.
__device__ __forceinline__ bool cone_hole(const ConeSelf& cs, const Vec3& p, float hx, float hyc, float hz,
                                          float crit_h) {
    float dh = sqrtf((p.x - hx) * (p.x - hx) + (p.y - hyc) * (p.y - hyc) + (p.z - hz) * (p.z - hz));
    float crit = crit_h / dh;
    float ex = (hx - p.x) / dh, ey = (hyc - p.y) / dh, ez = (hz - p.z) / dh;
    return sqrtf((ez - cs.uz) * (ez - cs.uz) + (ey - cs.uy) * (ey - cs.uy) + (ex - cs.ux) * (ex - cs.ux)) <=
           crit + cs.crit_self;
}

__device__ __forceinline__ Box3 hole_box(const float4& a, const float4& b) {
    return Box3{a.x - b.x - kMargin, a.y - kMargin, a.w - b.x - kMargin,
                a.x + b.x + kMargin, a.z + kMargin, a.w + b.x + kMargin};
}

__device__ __forceinline__ Box3 box_of(const float4& lo, const float4& hi) {
    return Box3{lo.x, lo.y, lo.z, hi.x, hi.y, hi.z};
}

// One ray: voxel sub-point p (world) and its coordinates ps in the detecting
// crystal's frame, sub-cell c.  Returns its contribution; in RECORD mode also
// writes the ray's hit record to rec.
template <bool RECORD>
__device__ float trace_ray(const PEParams& P, const DevGeometry& G, const PeSmem& S, const unsigned* mask,
                           const Detecting& D, const Vec3& p, const Vec3& ps, int c, int* rec, int* status,
                           unsigned long long* n_cry_tests, unsigned long long* n_hole_tests) {
    const int sy = c % P.dY;
    const int sx = (c / P.dY) % P.dX;
    const int sz = c / (P.dY * P.dX);
    // Sub-cell centre, crystal frame then world (PESysMatGen.cu:606-616).
    const float xDs = -D.w / 2.0f + ((float)sx + 0.5f) / (float)P.dX * D.w;
    const float zDs = -D.h / 2.0f + ((float)sz + 0.5f) / (float)P.dZ * D.h;
    const float yDs = -D.t / 2.0f + ((float)sy + 0.5f) / (float)P.dY * D.t;
    Vec3 q;
    q.x = D.cx + (xDs * D.cp - zDs * D.sp);
    q.z = D.cz + (xDs * D.sp + zDs * D.cp);
    q.y = D.cy + yDs;

    const float dsq = (q.y - p.y) * (q.y - p.y) + (q.x - p.x) * (q.x - p.x) + (q.z - p.z) * (q.z - p.z);
    const float r = sqrtf(dsq);
    const float cosang = (q.y - p.y) / r;

    int rec_h = 0, rec_c = 0;
    unsigned plate_miss = 0u;
    // Plates the ray does not traverse block it (PESysMatGen.cu:643-659):
    // exp(-(1e5 + ...)) is exactly 0, so the ray contributes nothing.
    for (int m = 0; m < G.n_plates; ++m) {
        const PlateBox& pb = G.plate[m];
        Box3 b{pb.x1, pb.y1, pb.z1, pb.x2, pb.y2, pb.z2};
        if (chord_through(p.x, p.y, p.z, q.x, q.y, q.z, b) < 0.1f) plate_miss |= 1u << m;
    }
    if (!RECORD && plate_miss) return 0.0f;

    const Box3 q_box = point_box(q);
    const Box3 p_box = point_box(p);
    float att = 0.0f;
    // Plates: holes among the candidates, tungsten for the rest of T / cos(theta)
    // (PESysMatGen.cu:661-685).
    for (int m = 0; m < G.n_plates; ++m) {
        float in_holes = 0.0f;
        const int hb = S.h_plate_begin[m], he = S.h_plate_begin[m + 1];
        for (int wd = hb >> 5; wd <= ((he - 1) >> 5) && he > hb; ++wd) {
            unsigned bits = mask[kMaskC + wd];
            // keep only bits of this plate's range
            int lo = hb - (wd << 5), hi = he - (wd << 5);
            if (lo > 0) bits &= ~0u << lo;
            if (hi < 32) bits &= (1u << hi) - 1u;
            while (bits) {
                int b = __ffs(bits) - 1;
                bits &= bits - 1;
                int k = (wd << 5) + b;
                const float4 ha = S.h_a[k], hbv = S.h_b[k];
                if (!window_hit(p_box, q_box, hole_box(ha, hbv))) continue;
                if (n_hole_tests) ++*n_hole_tests;
                float len = chord_hole(p.x, p.y, p.z, q.x, q.y, q.z, ha.x, ha.y, ha.z, ha.w, hbv.x);
                in_holes += len;
                att += hbv.y * len;
                if (RECORD && len > 0.0f) {
                    if (rec_h < kRecHoles) rec[2 + rec_h] = S.h_id[k];
                    else atomicOr(status, kStatusRecordOverflow);
                    ++rec_h;
                }
            }
        }
        const PlateBox& pb = G.plate[m];
        float through = pb.thickness / cosang;
        if ((through - in_holes) >= 0.00001f) att += pb.mu_total * (through - in_holes);
    }
    // Other crystals among the candidates, each in its own frame (:687-725).
    const int nwc = (S.n_c + 31) >> 5;
    for (int wd = 0; wd < nwc; ++wd) {
        unsigned bits = mask[wd];
        while (bits) {
            int b = __ffs(bits) - 1;
            bits &= bits - 1;
            int k = (wd << 5) + b;
            if (!window_hit(p_box, q_box, box_of(S.c_lo[k], S.c_hi[k]))) continue;
            if (n_cry_tests) ++*n_cry_tests;
            const float4 kp = S.c_pos[k], ks = S.c_size[k];
            const float2 kr = S.c_rot[k];
            float xIa = (p.x - kp.x) * kr.x - (p.z - kp.z) * kr.y;
            float yIa = p.y - kp.y;
            float zIa = (p.x - kp.x) * kr.y + (p.z - kp.z) * kr.x;
            float xDa = (q.x - kp.x) * kr.x - (q.z - kp.z) * kr.y;
            float yDa = q.y - kp.y;
            float zDa = (q.x - kp.x) * kr.y + (q.z - kp.z) * kr.x;
            Box3 kb{-0.5f * ks.x, -0.5f * ks.y, -0.5f * ks.z, 0.5f * ks.x, 0.5f * ks.y, 0.5f * ks.z};
            float len = chord_through(xIa, yIa, zIa, xDa, yDa, zDa, kb);
            att += len * kp.w;
            if (RECORD && len > 0.0f) {
                if (rec_c < kRecCrystals) rec[3 + kRecHoles + rec_c] = S.c_id[k];
                else atomicOr(status, kStatusRecordOverflow);
                ++rec_c;
            }
        }
    }
    if (RECORD) {
        rec[0] = (int)plate_miss;
        rec[1] = rec_h < kRecHoles ? rec_h : kRecHoles;
        rec[2 + kRecHoles] = rec_c < kRecCrystals ? rec_c : kRecCrystals;
        if (plate_miss) return 0.0f;
    }
    // Path inside the detecting crystal up to the sub-cell (:727-746).
    Box3 ub{((float)sx / (float)P.dX - 0.5f) * D.w, ((float)sy / (float)P.dY - 0.5f) * D.t,
            ((float)sz / (float)P.dZ - 0.5f) * D.h, (((float)sx + 1.0f) / (float)P.dX - 0.5f) * D.w,
            (((float)sy + 1.0f) / (float)P.dY - 0.5f) * D.t, (((float)sz + 1.0f) / (float)P.dZ - 0.5f) * D.h};
    float l1 = chord_to_end(ps.x, ps.y, ps.z, xDs, yDs, zDs, D.self_box);
    float l2 = chord_to_end(ps.x, ps.y, ps.z, xDs, yDs, zDs, ub);
    att += (l1 - l2) * D.mu_t;
    const float eff = expf(-att);
    // Absorption in the sub-cell along the ray extended by 1000 mm (:749-759).
    float xt = xDs + 1000.0f * (xDs - ps.x) / r;
    float yt = yDs + 1000.0f * (yDs - ps.y) / r;
    float zt = zDs + 1000.0f * (zDs - ps.z) / r;
    float labs = chord_through(ps.x, ps.y, ps.z, xt, yt, zt, ub);
    float absorb = (1.0f - expf(-labs * D.mu_t)) * D.mu_pe / D.mu_t;
    // Solid angle: the largest of the three projected sub-cell faces (:618-639),
    // A * |cos| / (4 pi d^2), single precision.
    const float k4 = 0.0795774715459476678f / (dsq * r);   // 1 / (4 pi d^3)
    float sa_x = D.area_x * fabsf((q.x - p.x) * D.cp - (q.z - p.z) * D.sp) * k4;
    float sa_z = D.area_z * fabsf((q.x - p.x) * D.sp + (q.z - p.z) * D.cp) * k4;
    float sa_y = D.area_y * fabsf(q.y - p.y) * k4;
    float sa = fmaxf(fmaxf(sa_x, sa_y), sa_z);
    return eff * sa * absorb;
}

template <bool RECORD>
__global__ void __launch_bounds__(kPeThreads, 2) pe_trace_kernel(PEParams P, DevGeometry G) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PeSmem& S = *reinterpret_cast<PeSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    const long long tile = P.tile_list ? P.tile_list[blockIdx.x] : (long long)blockIdx.x;
    const int ct = (int)(tile % P.n_ctiles);
    const long long vt = tile / P.n_ctiles;
    const int bxi = (int)(vt % P.tiles_x);
    const int byi = (int)((vt / P.tiles_x) % P.tiles_y);
    const int bzi = (int)(vt / ((long long)P.tiles_x * P.tiles_y));
    const int ix0 = bxi * P.bx, iy0 = byi * P.by, iz0 = P.z0 + bzi * P.bz;
    const int ix1 = min(ix0 + P.bx, P.nx), iy1 = min(iy0 + P.by, P.ny), iz1 = min(iz0 + P.bz, P.z0 + P.nzs);
    const int d0 = P.row0 + ct * kPeWarps;

    // ---- 1. tile cull -------------------------------------------------------
    // Sub-point box of the brick: extreme fine voxel centres, rotated.
    Box3 A;
    {
        Vec3 c0 = subpoint(P, ix0 * P.kx, iy0 * P.ky, iz0 * P.kz);
        Vec3 c1 = subpoint(P, ix1 * P.kx - 1, iy0 * P.ky, iz0 * P.kz);
        Vec3 c2 = subpoint(P, ix0 * P.kx, iy1 * P.ky - 1, iz0 * P.kz);
        Vec3 c3 = subpoint(P, ix1 * P.kx - 1, iy1 * P.ky - 1, iz0 * P.kz);
        A.x1 = fminf(fminf(c0.x, c1.x), fminf(c2.x, c3.x)) - kMargin;
        A.x2 = fmaxf(fmaxf(c0.x, c1.x), fmaxf(c2.x, c3.x)) + kMargin;
        A.y1 = fminf(fminf(c0.y, c1.y), fminf(c2.y, c3.y)) - kMargin;
        A.y2 = fmaxf(fmaxf(c0.y, c1.y), fmaxf(c2.y, c3.y)) + kMargin;
        Vec3 c4 = subpoint(P, ix0 * P.kx, iy0 * P.ky, iz1 * P.kz - 1);
        A.z1 = fminf(c0.z, c4.z) - kMargin;
        A.z2 = fmaxf(c0.z, c4.z) + kMargin;
    }
    if (tid < kPeWarps) {
        int d = d0 + tid;
        if (d < P.row1) {
            float4 lo = G.c.lo[d], hi = G.c.hi[d];
            S.d_box[tid] = Box3{lo.x - kMargin, lo.y - kMargin, lo.z - kMargin, hi.x + kMargin, hi.y + kMargin, hi.z + kMargin};
        } else {
            S.d_box[tid] = Box3{1e30f, 1e30f, 1e30f, -1e30f, -1e30f, -1e30f};
        }
    }
    __syncthreads();
    const int n_d = min(kPeWarps, P.row1 - d0);

    int base = 0;
    for (int k0 = 0; k0 < G.n_crystals; k0 += kPeThreads) {
        const int k = k0 + tid;
        bool pass = false;
        float4 lo, hi;
        if (k < G.n_crystals) {
            lo = G.c.lo[k];
            hi = G.c.hi[k];
            Box3 K{lo.x - kMargin, lo.y - kMargin, lo.z - kMargin, hi.x + kMargin, hi.y + kMargin, hi.z + kMargin};
            for (int j = 0; j < n_d && !pass; ++j) pass = window_hit(A, S.d_box[j], K);
        }
        unsigned bal = __ballot_sync(0xffffffffu, pass);
        if (lane == 0) S.warp_cnt[warp] = __popc(bal);
        __syncthreads();
        int off = base, total = 0;
        for (int w = 0; w < kPeWarps; ++w) {
            int cnt = S.warp_cnt[w];
            if (w < warp) off += cnt;
            total += cnt;
        }
        off += __popc(bal & lanemask_lt());
        if (pass) {
            if (off < kSupC) {
                S.c_pos[off] = G.c.pos[k];
                S.c_size[off] = G.c.size[k];
                float4 rr = G.c.rot[k];
                S.c_rot[off] = make_float2(rr.x, rr.y);
                S.c_lo[off] = make_float4(lo.x - kMargin, lo.y - kMargin, lo.z - kMargin, 0.0f);
                S.c_hi[off] = make_float4(hi.x + kMargin, hi.y + kMargin, hi.z + kMargin, 0.0f);
                S.c_id[off] = k;
            } else {
                atomicOr(P.status, kStatusSupersetOverflow);
            }
        }
        base += total;
        __syncthreads();
    }
    const int n_c = min(base, kSupC);
    base = 0;
    for (int k0 = 0; k0 < G.n_holes; k0 += kPeThreads) {
        const int k = k0 + tid;
        bool pass = false;
        float4 ha, hb;
        if (k < G.n_holes) {
            ha = G.h.a[k];
            hb = G.h.b[k];
            Box3 K = hole_box(ha, hb);
            for (int j = 0; j < n_d && !pass; ++j) pass = window_hit(A, S.d_box[j], K);
        }
        unsigned bal = __ballot_sync(0xffffffffu, pass);
        if (lane == 0) S.warp_cnt[warp] = __popc(bal);
        __syncthreads();
        int off = base, total = 0;
        for (int w = 0; w < kPeWarps; ++w) {
            int cnt = S.warp_cnt[w];
            if (w < warp) off += cnt;
            total += cnt;
        }
        off += __popc(bal & lanemask_lt());
        if (pass) {
            if (off < kSupH) {
                S.h_a[off] = ha;
                S.h_b[off] = hb;
                S.h_id[off] = k;
            } else {
                atomicOr(P.status, kStatusSupersetOverflow);
            }
        }
        base += total;
        __syncthreads();
    }
    const int n_h = min(base, kSupH);
    if (tid == 0) {
        S.n_c = n_c;
        S.n_h = n_h;
    }
    if (tid <= G.n_plates) {
        // First staged hole whose id is at or beyond plate `tid`'s first hole.
        int first = (tid < G.n_plates) ? G.plate[tid].hole_begin : G.n_holes;
        int cnt = 0;
        for (int i = 0; i < n_h; ++i) cnt += (S.h_id[i] < first) ? 1 : 0;
        S.h_plate_begin[tid] = cnt;
    }
    __syncthreads();

    // ---- 2. per-warp crystal, voxel walk --------------------------------------
    const int tv = P.bx * P.by * P.bz;
    const int d = d0 + warp;
    if (d < P.row1) {
        Detecting D;
        D.id = d;
        {
            float4 pos = G.c.pos[d], sz = G.c.size[d], rt = G.c.rot[d], ph = G.c.phys[d];
            D.cx = pos.x; D.cy = pos.y; D.cz = pos.z; D.mu_t = pos.w; D.mu_pe = ph.x;
            D.w = sz.x; D.t = sz.y; D.h = sz.z; D.crit = sz.w;
            D.cm = rt.x; D.sm = rt.y; D.cp = rt.z; D.sp = rt.w;
            D.self_box = Box3{-D.w / 2.0f, -D.t / 2.0f, -D.h / 2.0f, D.w / 2.0f, D.t / 2.0f, D.h / 2.0f};
            D.world = S.d_box[warp];
            D.area_x = D.t * D.h / (float)P.dZ / (float)P.dY;
            D.area_z = D.w * D.t / (float)P.dX / (float)P.dY;
            D.area_y = D.w * D.h / (float)P.dX / (float)P.dZ;
        }
        const bool absorbing = D.mu_t > 0.01f;   // PESysMatGen.cu:504, :598
        unsigned long long cnt_rays = 0, cnt_cry = 0, cnt_hole = 0, cnt_cone = 0;
        unsigned long long* pc_cry = P.counters ? &cnt_cry : nullptr;
        unsigned long long* pc_hole = P.counters ? &cnt_hole : nullptr;
        for (int vl = 0; vl < tv; ++vl) {
            const int ix = ix0 + vl % P.bx;
            const int iy = iy0 + (vl / P.bx) % P.by;
            const int iz = iz0 + vl / (P.bx * P.by);
            if (ix >= ix1 || iy >= iy1 || iz >= iz1) continue;
            int rec_slot = -1;
            if (RECORD) {
                long long vox = ((long long)iz * P.ny + iy) * P.nx + ix;
                for (int i = 0; i < P.rec_n; ++i)
                    if (P.rec_rows[i] == d && P.rec_vox[i] == vox) rec_slot = i;
                if (rec_slot < 0) continue;
            }
            float acc = 0.0f, comp = 0.0f;
            if (absorbing) {
                for (int s0 = 0; s0 < P.n_sv; s0 += P.group) {
                    const int gn = min(P.group, P.n_sv - s0);
                    // Candidate masks for sub-points s0 .. s0+gn-1.
                    for (int j = 0; j < gn; ++j) {
                        int fx, fy, fz;
                        subpoint_index(P, ix, iy, iz, s0 + j, fx, fy, fz);
                        const Vec3 p = subpoint(P, fx, fy, fz);
                        const ConeSelf cs = cone_self(D, p);
                        const Box3 pb = point_box(p);
                        for (int wd = 0; wd < kMaskC; ++wd) {
                            if ((wd << 5) >= n_c) {
                                if (lane == 0) S.mask[warp][j][wd] = 0u;
                                continue;
                            }
                            const int k = (wd << 5) + lane;
                            bool pass = false;
                            if (k < n_c && S.c_id[k] != d && window_hit(pb, D.world, box_of(S.c_lo[k], S.c_hi[k]))) {
                                const float4 kp = S.c_pos[k];
                                pass = cone_crystal(cs, p, kp.x, kp.y, kp.z, S.c_size[k].w);
                                if (P.counters) ++cnt_cone;
                            }
                            unsigned bal = __ballot_sync(0xffffffffu, pass);
                            if (lane == 0) S.mask[warp][j][wd] = bal;
                        }
                        for (int wd = 0; wd < kMaskH; ++wd) {
                            if ((wd << 5) >= n_h) {
                                if (lane == 0) S.mask[warp][j][kMaskC + wd] = 0u;
                                continue;
                            }
                            const int k = (wd << 5) + lane;
                            bool pass = false;
                            if (k < n_h) {
                                const float4 ha = S.h_a[k], hb = S.h_b[k];
                                if (window_hit(pb, D.world, hole_box(ha, hb))) {
                                    pass = cone_hole(cs, p, ha.x, hb.w, ha.w, hb.z);
                                    if (P.counters) ++cnt_cone;
                                }
                            }
                            unsigned bal = __ballot_sync(0xffffffffu, pass);
                            if (lane == 0) S.mask[warp][j][kMaskC + wd] = bal;
                        }
                    }
                    __syncwarp();
                    const int nr = gn * P.n_sc;
                    for (int q0 = 0; q0 < nr; q0 += 32) {
                        const int q = q0 + lane;
                        if (q < nr) {
                            const int j = q / P.n_sc;
                            const int c = q - j * P.n_sc;
                            int fx, fy, fz;
                            subpoint_index(P, ix, iy, iz, s0 + j, fx, fy, fz);
                            const Vec3 p = subpoint(P, fx, fy, fz);
                            Vec3 ps;
                            ps.x = (p.x - D.cx) * D.cm - (p.z - D.cz) * D.sm;
                            ps.y = p.y - D.cy;
                            ps.z = (p.x - D.cx) * D.sm + (p.z - D.cz) * D.cm;
                            int* rec = nullptr;
                            if (RECORD)
                                rec = P.rec_out + ((long long)rec_slot * P.n_sv * P.n_sc + (long long)(s0 + j) * P.n_sc + c) *
                                                      kRecWords;
                            float v = trace_ray<RECORD>(P, G, S, S.mask[warp][j], D, p, ps, c, rec, P.status, pc_cry, pc_hole);
                            if (P.counters) ++cnt_rays;
                            // Kahan summation of the lane's rays.
                            float y = v - comp;
                            float t = acc + y;
                            comp = (t - acc) - y;
                            acc = t;
                        }
                    }
                    __syncwarp();
                }
            }
            float v = acc - comp;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) S.out[warp][vl] = v * P.inv_sv;
        }
        if (P.counters) {
            for (int o = 16; o > 0; o >>= 1) {
                cnt_rays += __shfl_xor_sync(0xffffffffu, cnt_rays, o);
                cnt_cry += __shfl_xor_sync(0xffffffffu, cnt_cry, o);
                cnt_hole += __shfl_xor_sync(0xffffffffu, cnt_hole, o);
                cnt_cone += __shfl_xor_sync(0xffffffffu, cnt_cone, o);
            }
            if (lane == 0) {
                atomicAdd(&P.counters[0], cnt_rays);
                atomicAdd(&P.counters[1], cnt_cry);
                atomicAdd(&P.counters[2], cnt_hole);
                atomicAdd(&P.counters[3], cnt_cone);
            }
        }
    }
    if (RECORD) return;
    __syncthreads();

    // ---- 4. write the tile: rows of the brick, voxel-contiguous runs ----------
    const int n_out = n_d * tv;
    for (int i = tid; i < n_out; i += kPeThreads) {
        const int w = i / tv, vl = i - w * tv;
        const int ix = ix0 + vl % P.bx;
        const int iy = iy0 + (vl / P.bx) % P.by;
        const int iz = iz0 + vl / (P.bx * P.by);
        if (ix >= ix1 || iy >= iy1 || iz >= iz1) continue;
        const long long col = ((long long)(iz - P.z0) * P.ny + iy) * P.nx + ix;
        P.dst[(long long)(d0 + w - P.row0) * P.ld + col] = S.out[w][vl];
    }
}

}  // namespace

size_t pe_smem_bytes() { return sizeof(PeSmem); }

cudaError_t pe_launch(const PEParams& p, const DevGeometry& geo, bool record, long long n_tiles, cudaStream_t stream) {
    const size_t smem = sizeof(PeSmem);
    if (n_tiles <= 0) return cudaSuccess;
    if (n_tiles > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    if (record) {
        static bool attr_set = false;
        if (!attr_set) {
            cudaError_t e = cudaFuncSetAttribute(pe_trace_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            attr_set = true;
        }
        pe_trace_kernel<true><<<(unsigned)n_tiles, kPeThreads, smem, stream>>>(p, geo);
    } else {
        static bool attr_set = false;
        if (!attr_set) {
            cudaError_t e = cudaFuncSetAttribute(pe_trace_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            attr_set = true;
        }
        pe_trace_kernel<false><<<(unsigned)n_tiles, kPeThreads, smem, stream>>>(p, geo);
    }
    return cudaGetLastError();
}

}  // namespace smb
