// Photoelectric (PE) system-matrix kernel for sm_100a.
//
// Computes, for every crystal d and voxel v,
//   A[d, v] = 1/Sv * sum over voxel sub-points p and crystal sub-cells q of
//             exp(-sum mu*L along p->q) * Omega(p, q) * absorption(q)
// with the reference's physics and hit decisions
// (PEGen_RayTracing_CircularHole/PESysMatGen.cu:375-764): a plate box the ray
// does not traverse blocks it (1e5 penalty), holes and other crystals count
// only when they are among the bounding-sphere candidates of (voxel point,
// detecting crystal), the detecting crystal attenuates up to the sub-cell,
// and the sub-cell absorbs (1 - exp(-mu_t L)) mu_pe / mu_t.
//
// Work decomposition (one CTA per tile = 8 crystals x one voxel brick):
//  1. Tile cull: the CTA tests every crystal and hole against the bundle of
//     segments from the brick's sub-point box to the union of its 8 crystals,
//     then to each crystal (division-free window test, conservative), and
//     stages the survivors, ordered by id, in shared memory.
//  2. Each warp owns one crystal and walks the brick's voxels.  Per voxel it
//     narrows the staged set with the same window test for that voxel's
//     sub-point box and compacts the survivors into a per-warp list.  The
//     reference counts a crystal or hole only when it passes the candidate
//     cone test of (voxel point, detecting crystal); a candidate that the ray
//     does not cross contributes nothing either way, so the cone test is taken
//     per ray and only for candidates with a nonzero chord (a float filter
//     decides clear cases; cases within 1e-5 of the threshold use the
//     reference's exact single-precision expression).  Each sub-point's own
//     cone parameters are computed once per group of sub-points.
//  3. Lanes trace one ray (sub-point, sub-cell) each.  The rays of a group of
//     sub-points are ordered (sub-cell column, sub-point, depth sub-cell) and
//     dealt 32 to a warp pass, so a pass holds rays that run almost together
//     through the plates and the crystals in front (one column of depth
//     cells seen from neighbouring sub-points): the lanes meet the same
//     candidates and take the same branches.  Each pass first narrows the
//     candidates to those its bundle of rays can reach (window test from the
//     voxel's sub-point box to the box of the pass's sub-cell centres).  Per
//     ray a division-free window test skips the exact test for candidates
//     the ray cannot reach; the exact tests are the reference's
//     single-precision ones, so every hit decision is the reference's.
//     Skipped candidates would have contributed exactly 0.  The plates use a
//     fast path that proves "fully traversed" with margins, else the exact
//     test.  Values that are not hit decisions (solid angle, path inside the
//     detecting crystal, absorption chord) use closed forms in single
//     precision.
//  4. Lanes accumulate with Kahan summation; warp shuffles reduce; the CTA
//     stages its 8 x brick results in shared memory and writes them out.
#include <cuda_runtime.h>

#include "pe.h"
#include "tracer.cuh"

namespace smb {

namespace {

constexpr int kLWC = kListC / 32;
constexpr int kLWH = kListH / 32;
constexpr float kMargin = 0.01f;     // mm added around every culling box
constexpr float kConeMargin = 1e-5f; // float-filter band around the cone threshold
constexpr int kPassSlots = 4;        // warp passes per group whose candidate masks are kept

struct WarpLists {
    unsigned short list_c[kListC];    // staged-set indices of the voxel's candidate crystals
    unsigned short list_h[kListH];    // ... and holes (ascending ids)
    unsigned short blist_c[kListC];   // staged-set indices the whole brick can reach for this warp's crystal
    unsigned short blist_h[kListH];   // (per-voxel lists narrow from these when they fit)
    int n_c, n_h;
    int nb_c, nb_h;
    int plate_begin[kMaxPlates + 1];  // list_h index where each plate's holes start
    float4 cs[kMaxGroup];             // per sub-point of the group: the detecting crystal's cone (ConeSelf)
    float4 pt[kMaxGroup];             // ... the sub-point in the world
    float4 pself[kMaxGroup];          // ... and in the detecting crystal's frame
    // Per warp pass: the candidates the pass's bundle of rays can reach.  Slot
    // i holds pass i of a group; full groups of one voxel trace the same
    // sub-cells in the same passes, so later groups reuse the first one's.
    unsigned pass_c[kPassSlots][kLWC];
    unsigned pass_h[kPassSlots][kLWH];
};

struct __align__(16) PeSmem {
    float4 c_pos[kSupC];     // cx, cy, cz, mu_total
    float4 c_size[kSupC];    // w, t, h, crit
    float4 c_lo[kSupC];      // inflated world AABB (lower corner), cos(-rot)
    float4 c_hi[kSupC];      // ... (upper corner), sin(-rot)
    int c_id[kSupC];
    float4 h_a[kSupH];       // x, y1, y2, z
    float4 h_b[kSupH];       // R, mu_total, crit, yc
    int h_id[kSupH];
    float frac[3][kMaxSubcellsPerAxis];   // (s + 0.5) / d per axis, IEEE, as the reference computes it
    Box3 d_box[kPeWarps];    // inflated AABB of the tile's crystals
    int warp_cnt[kPeWarps];
    int n_c, n_h;
    int overflow;            // the tile's candidates exceed the staged capacity: every voxel goes through the tables
    WarpLists wl[kPeWarps];
    float out[kPeWarps][kMaxTileVoxels];
};

// Two CTAs per SM (the kernel's launch bound): an SM holds 228 KB of shared
// memory, of which each CTA also reserves 1 KB.
static_assert(2 * (sizeof(PeSmem) + 1024) <= 228 * 1024, "PeSmem must leave room for two CTAs per SM");

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// floor(n / d) for 0 <= n < 2^22 with inv ~ 1/d: exact after one correction.
__device__ __forceinline__ int fast_div(int n, int d, float inv) {
    int q = __float2int_rz(__fmul_rn((float)n, inv));
    int r = n - q * d;
    if (r < 0) --q;
    else if (r >= d) ++q;
    return q;
}

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

__device__ __forceinline__ Vec3 subpoint_of(const PEParams& P, int ix, int iy, int iz, int s) {
    const int sz = fast_div(s, P.kx * P.ky, P.inv_kxky);
    const int rem = s - sz * P.kx * P.ky;
    const int sy = fast_div(rem, P.kx, P.inv_kx);
    const int sx = rem - sy * P.kx;
    return subpoint(P, ix * P.kx + sx, iy * P.ky + sy, iz * P.kz + sz);
}

// Per-crystal constants of the warp's detecting crystal.
struct Detecting {
    float cx, cy, cz, mu_t, mu_pe;
    float w, t, h, crit;
    float cm, sm, cp, sp;          // cos(-rot), sin(-rot), cos(rot), sin(rot)
    Box3 world;                    // inflated world AABB
    float area_x, area_z, area_y;  // sub-cell face areas (t*h/dZ/dY, w*t/dX/dY, w*h/dX/dZ)
    float hx, hy, hz;              // sub-cell half sizes
};

// ---- candidate cone test (PESysMatGen.cu:506-589) -----------------------------
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

// The reference's crystal test, exactly (IEEE single, no contraction).
__device__ __noinline__ bool cone_crystal_exact(ConeSelf cs, Vec3 p, float xk, float yk, float zk, float crit_k) {
    float dk = sqrtf((p.x - xk) * (p.x - xk) + (p.y - yk) * (p.y - yk) + (p.z - zk) * (p.z - zk));
    float crit = crit_k / dk / 2.0f;
    float ex = (xk - p.x) / dk, ey = (yk - p.y) / dk, ez = (zk - p.z) / dk;
    return sqrtf((ez - cs.uz) * (ez - cs.uz) + (ey - cs.uy) * (ey - cs.uy) + (ex - cs.ux) * (ex - cs.ux)) <=
           crit + cs.crit_self;
}

// The reference's hole test, exactly.
__device__ __noinline__ bool cone_hole_exact(ConeSelf cs, Vec3 p, float hx, float hyc, float hz, float crit_h) {
    float dh = sqrtf((p.x - hx) * (p.x - hx) + (p.y - hyc) * (p.y - hyc) + (p.z - hz) * (p.z - hz));
    float crit = crit_h / dh;
    float ex = (hx - p.x) / dh, ey = (hyc - p.y) / dh, ez = (hz - p.z) / dh;
    return sqrtf((ez - cs.uz) * (ez - cs.uz) + (ey - cs.uy) * (ey - cs.uy) + (ex - cs.ux) * (ex - cs.ux)) <=
           crit + cs.crit_self;
}

// Float filter: the same quantities with fast reciprocal square roots; its
// error is below 1e-6 of the unit-sphere distances compared, so outside a
// band of kConeMargin the answer equals the exact one.  Returns 1 (pass),
// 0 (fail) or -1 (too close to call).
__device__ __forceinline__ int cone_filter(const ConeSelf& cs, const Vec3& p, float xk, float yk, float zk,
                                           float crit_scaled) {
    float dx = xk - p.x, dy = yk - p.y, dz = zk - p.z;
    float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float inv = rsqrtf(d2);
    float ex = fmaf(dx, inv, -cs.ux), ey = fmaf(dy, inv, -cs.uy), ez = fmaf(dz, inv, -cs.uz);
    const float e2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
    const float lhs = e2 > 0.0f ? e2 * rsqrtf(e2) : 0.0f;   // within 1e-6 relative of sqrt(e2)
    float rhs = fmaf(crit_scaled, inv, cs.crit_self);
    float diff = lhs - rhs;
    if (diff < -kConeMargin) return 1;
    if (diff > kConeMargin) return 0;
    return -1;
}

__device__ __forceinline__ Box3 hole_box(const float4& a, const float4& b) {
    return Box3{a.x - b.x - kMargin, a.y - kMargin, a.w - b.x - kMargin,
                a.x + b.x + kMargin, a.z + kMargin, a.w + b.x + kMargin};
}

__device__ __forceinline__ Box3 box_of(const float4& lo, const float4& hi) {
    return Box3{lo.x, lo.y, lo.z, hi.x, hi.y, hi.z};
}

// ---- division-free window test -------------------------------------------------
// window_hit (tracer.cuh) with the bundle source A and target B fixed: the two
// reciprocals are computed once.  Conservative: K carries the 0.01 mm margin,
// far above the error of the approximate reciprocals.
struct Bundle {
    Box3 A, B;
    float inv2;     // 1 / (B.y2 - A.y2)
    float inv1;     // 1 / (B.y1 - A.y1)
    bool ordered;   // A lies entirely before B in depth
};

__device__ __forceinline__ Bundle make_bundle(const Box3& A, const Box3& B) {
    Bundle b;
    b.A = A;
    b.B = B;
    b.ordered = A.y2 < B.y1;
    b.inv2 = __fdividef(1.0f, B.y2 - A.y2);
    b.inv1 = __fdividef(1.0f, B.y1 - A.y1);
    return b;
}

__device__ __forceinline__ bool bundle_hit(const Bundle& b, const Box3& K) {
    if (!b.ordered || !(b.A.y2 < K.y1)) return true;
    if (K.y1 > b.B.y2) return false;              // beyond every segment's end
    const float yhi = fminf(K.y2, b.B.y2);
    const float lmin = fmaxf((K.y1 - b.A.y2) * b.inv2, 0.0f);
    const float lmax = fminf(1.0f, (yhi - b.A.y1) * b.inv1);
    const float xa = fmaf(b.B.x1 - b.A.x1, lmin, b.A.x1), xb = fmaf(b.B.x1 - b.A.x1, lmax, b.A.x1);
    const float xc = fmaf(b.B.x2 - b.A.x2, lmin, b.A.x2), xd = fmaf(b.B.x2 - b.A.x2, lmax, b.A.x2);
    if (fminf(xa, xb) > K.x2 || fmaxf(xc, xd) < K.x1) return false;
    const float za = fmaf(b.B.z1 - b.A.z1, lmin, b.A.z1), zb = fmaf(b.B.z1 - b.A.z1, lmax, b.A.z1);
    const float zc = fmaf(b.B.z2 - b.A.z2, lmin, b.A.z2), zd = fmaf(b.B.z2 - b.A.z2, lmax, b.A.z2);
    if (fminf(za, zb) > K.z2 || fmaxf(zc, zd) < K.z1) return false;
    return true;
}

// Segment p -> q against box K (inflated): the point-to-point bundle.
struct RaySeg {
    Vec3 p, q;
    float inv_dy;
    bool ordered;
};

__device__ __forceinline__ bool ray_may_hit(const RaySeg& r, const Box3& K) {
    if (!r.ordered || !(r.p.y < K.y1)) return true;
    if (K.y1 > r.q.y) return false;               // beyond the segment's end
    const float lmin = (K.y1 - r.p.y) * r.inv_dy;
    const float lmax = fminf(1.0f, (fminf(K.y2, r.q.y) - r.p.y) * r.inv_dy);
    const float dx = r.q.x - r.p.x, dz = r.q.z - r.p.z;
    const float xa = fmaf(dx, lmin, r.p.x), xb = fmaf(dx, lmax, r.p.x);
    if (fminf(xa, xb) > K.x2 || fmaxf(xa, xb) < K.x1) return false;
    const float za = fmaf(dz, lmin, r.p.z), zb = fmaf(dz, lmax, r.p.z);
    if (fminf(za, zb) > K.z2 || fmaxf(za, zb) < K.z1) return false;
    return true;
}

// Exact plate test out of line (rarely needed: see plate_traversed).
__device__ __noinline__ float plate_chord_exact(Vec3 p, Vec3 q, Box3 b) {
    return chord_through(p.x, p.y, p.z, q.x, q.y, q.z, b);
}

// The reference blocks a ray whose chord through a plate box is < 0.1
// (PESysMatGen.cu:656-658).  When the segment starts 0.01 mm before the plate,
// ends 0.01 mm after it, and stays 0.01 mm inside its lateral faces at both
// depth planes, every branch of the exact test returns the y-slab chord
// (>= thickness > 0.11), so the answer "traversed" is certain; otherwise the
// exact test decides.
__device__ __forceinline__ bool plate_traversed(const Vec3& p, const Vec3& q, float inv_dy, const PlateBox& pb) {
    const Box3 b{pb.x1, pb.y1, pb.z1, pb.x2, pb.y2, pb.z2};
    if (p.y < pb.y1 - kMargin && q.y > pb.y2 + kMargin && (pb.y2 - pb.y1) > 0.11f) {
        const float l1 = (pb.y1 - p.y) * inv_dy, l2 = (pb.y2 - p.y) * inv_dy;
        const float dx = q.x - p.x, dz = q.z - p.z;
        const float xa = fmaf(dx, l1, p.x), xb = fmaf(dx, l2, p.x);
        const float za = fmaf(dz, l1, p.z), zb = fmaf(dz, l2, p.z);
        const float lo_x = pb.x1 + kMargin, hi_x = pb.x2 - kMargin, lo_z = pb.z1 + kMargin, hi_z = pb.z2 - kMargin;
        if (fminf(xa, xb) > lo_x && fmaxf(xa, xb) < hi_x && fminf(za, zb) > lo_z && fmaxf(za, zb) < hi_z) return true;
    }
    return !(plate_chord_exact(p, q, b) < 0.1f);
}

__device__ __noinline__ float self_path_exact(Vec3 ps, Vec3 qs, Box3 crystal, Box3 unit, float* absorb_len, float r) {
    float l1 = chord_to_end(ps.x, ps.y, ps.z, qs.x, qs.y, qs.z, crystal);
    float l2 = chord_to_end(ps.x, ps.y, ps.z, qs.x, qs.y, qs.z, unit);
    float xt = qs.x + 1000.0f * (qs.x - ps.x) / r;
    float yt = qs.y + 1000.0f * (qs.y - ps.y) / r;
    float zt = qs.z + 1000.0f * (qs.z - ps.z) / r;
    *absorb_len = chord_through(ps.x, ps.y, ps.z, xt, yt, zt, unit);
    return l1 - l2;
}

// Contribution of one ray once its attenuation outside the detecting crystal
// is known: the path inside the detecting crystal, absorption and solid angle.
__device__ __forceinline__ float ray_value(const Detecting& D, const Vec3& ps, float xDs, float yDs, float zDs,
                                           float att, float r, float inv_r, float dxw, float dy, float dzw) {
    // Path inside the detecting crystal before the sub-cell and the absorption
    // chord (PESysMatGen.cu:727-759), as values: for the line from ps through
    // the sub-cell centre qs (direction u), the sub-cell entry lies at
    // min_i(h_i / |u_i|) before qs and the exit as far after it, and the
    // crystal entry at min_i(g_i / |u_i|) with g_i the distance from qs to the
    // crystal face facing ps.  When ps is not clearly outside the crystal or
    // the ray is nearly parallel to its depth faces, the reference's own
    // functions are used.
    const float vx = xDs - ps.x, vy = yDs - ps.y, vz = zDs - ps.z;
    float self_len, absorb_len;
    const float hw = 0.5f * D.w, ht = 0.5f * D.t, hh = 0.5f * D.h;
    const bool outside = (fabsf(ps.x) > hw + kMargin) || (fabsf(ps.y) > ht + kMargin) || (fabsf(ps.z) > hh + kMargin);
    if (outside && fabsf(vy) > 0.01f) {
        const float ax = fabsf(vx), ay = fabsf(vy), az = fabsf(vz);
        // distances along the line, in units of |v| * (1 / |v_i|)
        const float cell = fminf(fminf(D.hx * __fdividef(1.0f, ax), D.hy * __fdividef(1.0f, ay)),
                                 D.hz * __fdividef(1.0f, az));
        const float gx = (vx > 0.0f) ? (xDs + hw) : (hw - xDs);
        const float gy = (vy > 0.0f) ? (yDs + ht) : (ht - yDs);
        const float gz = (vz > 0.0f) ? (zDs + hh) : (hh - zDs);
        const float crys = fminf(fminf(gx * __fdividef(1.0f, ax), gy * __fdividef(1.0f, ay)), gz * __fdividef(1.0f, az));
        self_len = (crys - cell) * r;
        absorb_len = 2.0f * cell * r;
    } else {
        const Box3 cb{-D.w / 2.0f, -D.t / 2.0f, -D.h / 2.0f, D.w / 2.0f, D.t / 2.0f, D.h / 2.0f};
        const Box3 ub{xDs - D.hx, yDs - D.hy, zDs - D.hz, xDs + D.hx, yDs + D.hy, zDs + D.hz};
        self_len = self_path_exact(ps, Vec3{xDs, yDs, zDs}, cb, ub, &absorb_len, r);
    }
    att = fmaf(self_len, D.mu_t, att);
    const float eff = __expf(-att);
    const float absorb = (1.0f - __expf(-absorb_len * D.mu_t)) * D.mu_pe / D.mu_t;
    // Solid angle: the largest of the three projected sub-cell faces (:618-639),
    // A * |cos| / (4 pi d^2).
    const float k4 = 0.0795774715459476678f * inv_r * inv_r * inv_r;   // 1 / (4 pi d^3)
    const float sa_x = D.area_x * fabsf(dxw * D.cp - dzw * D.sp);
    const float sa_z = D.area_z * fabsf(dxw * D.sp + dzw * D.cp);
    const float sa_y = D.area_y * fabsf(dy);
    const float sa = fmaxf(fmaxf(sa_x, sa_y), sa_z) * k4;
    return eff * sa * absorb;
}

// Sub-cell centre in the detecting crystal's frame (xDs, yDs, zDs) and in the
// world (q), as the reference computes them (PESysMatGen.cu:606-616).
struct SubCell {
    float xDs, yDs, zDs;
    Vec3 q;
};

__device__ __forceinline__ SubCell sub_cell(const Detecting& D, const PeSmem& S, int sx, int sy, int sz) {
    SubCell c;
    c.xDs = -D.w / 2.0f + S.frac[0][sx] * D.w;
    c.zDs = -D.h / 2.0f + S.frac[2][sz] * D.h;
    c.yDs = -D.t / 2.0f + S.frac[1][sy] * D.t;
    c.q.x = D.cx + (c.xDs * D.cp - c.zDs * D.sp);
    c.q.z = D.cz + (c.xDs * D.sp + c.zDs * D.cp);
    c.q.y = D.cy + c.yDs;
    return c;
}

// One ray: sub-point p (world) and ps (detecting crystal frame), sub-cell
// `cell`.  pass_c / pass_h: the candidates the warp pass's bundle of rays
// can reach (a superset of those this ray can reach).  The reference counts a
// crystal or hole only when it is among the sub-point's cone candidates
// (PESysMatGen.cu:506-589); a candidate the ray does not cross adds nothing
// either way, so the cone test (`csp`: the sub-point's ConeSelf) is taken only
// for candidates with a nonzero chord.  Returns the contribution; in RECORD
// mode also the hit record.
template <bool RECORD>
__device__ __forceinline__ float trace_ray(const PEParams& P, const DevGeometry& G, const PeSmem& S,
                                           const WarpLists& L, const unsigned* pass_c, const unsigned* pass_h,
                                           const float4* csp, const Detecting& D, const Vec3& p,
                                           const Vec3& ps, const SubCell& cell, int* rec, int* status,
                                           unsigned long long* n_cry, unsigned long long* n_hole,
                                           unsigned long long* n_cone) {
    const float xDs = cell.xDs, yDs = cell.yDs, zDs = cell.zDs;
    const Vec3 q = cell.q;

    RaySeg seg;
    seg.p = p;
    seg.q = q;
    seg.ordered = p.y < q.y;
    const float dy = q.y - p.y;
    seg.inv_dy = __fdividef(1.0f, dy);

    unsigned plate_miss = 0u;
    for (int m = 0; m < G.n_plates; ++m)
        if (!plate_traversed(p, q, seg.inv_dy, G.plate[m])) plate_miss |= 1u << m;
    if (!RECORD && plate_miss) return 0.0f;   // exp(-(1e5 + ...)) == 0

    const float dxw = q.x - p.x, dzw = q.z - p.z;
    const float dsq = fmaf(dy, dy, fmaf(dxw, dxw, dzw * dzw));
    const float inv_r = rsqrtf(dsq);
    const float r = dsq * inv_r;

    int rec_h = 0, rec_c = 0;
    float att = 0.0f;
    // Plates: holes among the candidates, tungsten for the rest of T / cos(theta)
    // (PESysMatGen.cu:661-685).
    for (int m = 0; m < G.n_plates; ++m) {
        float in_holes = 0.0f;
        const int hb = L.plate_begin[m], he = L.plate_begin[m + 1];
        for (int wd = hb >> 5; wd <= ((he - 1) >> 5) && he > hb; ++wd) {
            unsigned bits = pass_h[wd];
            const int lo = hb - (wd << 5), hi = he - (wd << 5);
            if (lo > 0) bits &= ~0u << lo;
            if (hi < 32) bits &= (1u << hi) - 1u;
            while (bits) {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1;
                const int k = L.list_h[(wd << 5) + b];
                const float4 ha = S.h_a[k], hbv = S.h_b[k];
                if (!ray_may_hit(seg, hole_box(ha, hbv))) continue;
                if (n_hole) ++*n_hole;
                const float len = chord_hole(p.x, p.y, p.z, q.x, q.y, q.z, ha.x, ha.y, ha.z, ha.w, hbv.x);
                if (len == 0.0f) continue;
                if (n_cone) ++*n_cone;
                const float4 c4 = *csp;
                const ConeSelf cs{c4.x, c4.y, c4.z, c4.w};
                int f = cone_filter(cs, p, ha.x, hbv.w, ha.w, hbv.z);
                if (f < 0) f = cone_hole_exact(cs, p, ha.x, hbv.w, ha.w, hbv.z) ? 1 : 0;
                if (!f) continue;
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
        const float through = pb.thickness * r * seg.inv_dy;   // T / cos(theta)
        if ((through - in_holes) >= 0.00001f) att += pb.mu_total * (through - in_holes);
    }
    // Other crystals among the candidates, each in its own frame (:687-725).
    const int nwc = (L.n_c + 31) >> 5;
    for (int wd = 0; wd < nwc; ++wd) {
        unsigned bits = pass_c[wd];
        while (bits) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            const int k = L.list_c[(wd << 5) + b];
            const float4 klo = S.c_lo[k], khi = S.c_hi[k];
            if (!ray_may_hit(seg, box_of(klo, khi))) continue;
            if (n_cry) ++*n_cry;
            const float4 kp = S.c_pos[k], ks = S.c_size[k];
            const float2 kr = make_float2(klo.w, khi.w);
            const float yIa = p.y - kp.y;
            const float yDa = q.y - kp.y;
            float xIa, zIa, xDa, zDa;
            if (kr.x == 1.0f && kr.y == 0.0f) {
                // Unrotated crystal: a * 1 - b * (+-0) and a * (+-0) + b * 1
                // round to a and b exactly.  Only the sign of a zero result
                // can differ, and chord_through never divides by a coordinate:
                // it subtracts them from nonzero box bounds, compares them, and
                // divides only by differences of at least 0.001.
                xIa = p.x - kp.x;
                zIa = p.z - kp.z;
                xDa = q.x - kp.x;
                zDa = q.z - kp.z;
            } else {
                xIa = (p.x - kp.x) * kr.x - (p.z - kp.z) * kr.y;
                zIa = (p.x - kp.x) * kr.y + (p.z - kp.z) * kr.x;
                xDa = (q.x - kp.x) * kr.x - (q.z - kp.z) * kr.y;
                zDa = (q.x - kp.x) * kr.y + (q.z - kp.z) * kr.x;
            }
            const Box3 kb{-0.5f * ks.x, -0.5f * ks.y, -0.5f * ks.z, 0.5f * ks.x, 0.5f * ks.y, 0.5f * ks.z};
            const float len = chord_through(xIa, yIa, zIa, xDa, yDa, zDa, kb);
            if (len == 0.0f) continue;
            if (n_cone) ++*n_cone;
            const float4 c4 = *csp;
            const ConeSelf cs{c4.x, c4.y, c4.z, c4.w};
            int f = cone_filter(cs, p, kp.x, kp.y, kp.z, 0.5f * ks.w);
            if (f < 0) f = cone_crystal_exact(cs, p, kp.x, kp.y, kp.z, ks.w) ? 1 : 0;
            if (!f) continue;
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

    return ray_value(D, ps, xDs, yDs, zDs, att, r, inv_r, dxw, dy, dzw);
}

// One ray with its candidates read straight from the geometry tables: every
// hole and every other crystal, in id order, under the same window test,
// exact chord and cone test as trace_ray.  For voxels whose candidate sets do
// not fit the shared-memory lists (dense hole grids, very large detectors):
// the same decisions and values, without a list.
template <bool RECORD>
__device__ __forceinline__ float trace_ray_global(const DevGeometry& G, const Detecting& D, int d, const Vec3& p,
                                                  const Vec3& ps, const ConeSelf& cs, const SubCell& cell, int* rec,
                                                  int* status) {
    const float xDs = cell.xDs, yDs = cell.yDs, zDs = cell.zDs;
    const Vec3 q = cell.q;
    RaySeg seg;
    seg.p = p;
    seg.q = q;
    seg.ordered = p.y < q.y;
    const float dy = q.y - p.y;
    seg.inv_dy = __fdividef(1.0f, dy);
    unsigned plate_miss = 0u;
    for (int m = 0; m < G.n_plates; ++m)
        if (!plate_traversed(p, q, seg.inv_dy, G.plate[m])) plate_miss |= 1u << m;
    if (!RECORD && plate_miss) return 0.0f;
    const float dxw = q.x - p.x, dzw = q.z - p.z;
    const float dsq = fmaf(dy, dy, fmaf(dxw, dxw, dzw * dzw));
    const float inv_r = rsqrtf(dsq);
    const float r = dsq * inv_r;
    int rec_h = 0, rec_c = 0;
    float att = 0.0f;
    for (int m = 0; m < G.n_plates; ++m) {
        float in_holes = 0.0f;
        const int hb = G.plate[m].hole_begin, he = (m + 1 < G.n_plates) ? G.plate[m + 1].hole_begin : G.n_holes;
        for (int k = hb; k < he; ++k) {
            const float4 ha = G.h.a[k], hbv = G.h.b[k];
            if (!ray_may_hit(seg, hole_box(ha, hbv))) continue;
            const float len = chord_hole(p.x, p.y, p.z, q.x, q.y, q.z, ha.x, ha.y, ha.z, ha.w, hbv.x);
            if (len == 0.0f) continue;
            int f = cone_filter(cs, p, ha.x, hbv.w, ha.w, hbv.z);
            if (f < 0) f = cone_hole_exact(cs, p, ha.x, hbv.w, ha.w, hbv.z) ? 1 : 0;
            if (!f) continue;
            in_holes += len;
            att += hbv.y * len;
            if (RECORD && len > 0.0f) {
                if (rec_h < kRecHoles) rec[2 + rec_h] = k;
                else atomicOr(status, kStatusRecordOverflow);
                ++rec_h;
            }
        }
        const PlateBox& pb = G.plate[m];
        const float through = pb.thickness * r * seg.inv_dy;
        if ((through - in_holes) >= 0.00001f) att += pb.mu_total * (through - in_holes);
    }
    for (int k = 0; k < G.n_crystals; ++k) {
        if (k == d) continue;
        const float4 lo = G.c.lo[k], hi = G.c.hi[k];
        if (!ray_may_hit(seg, Box3{lo.x - kMargin, lo.y - kMargin, lo.z - kMargin, hi.x + kMargin, hi.y + kMargin,
                                   hi.z + kMargin}))
            continue;
        const float4 kp = G.c.pos[k], ks = G.c.size[k], kr = G.c.rot[k];
        const float xIa = (p.x - kp.x) * kr.x - (p.z - kp.z) * kr.y;
        const float yIa = p.y - kp.y;
        const float zIa = (p.x - kp.x) * kr.y + (p.z - kp.z) * kr.x;
        const float xDa = (q.x - kp.x) * kr.x - (q.z - kp.z) * kr.y;
        const float yDa = q.y - kp.y;
        const float zDa = (q.x - kp.x) * kr.y + (q.z - kp.z) * kr.x;
        const Box3 kb{-0.5f * ks.x, -0.5f * ks.y, -0.5f * ks.z, 0.5f * ks.x, 0.5f * ks.y, 0.5f * ks.z};
        const float len = chord_through(xIa, yIa, zIa, xDa, yDa, zDa, kb);
        if (len == 0.0f) continue;
        int f = cone_filter(cs, p, kp.x, kp.y, kp.z, 0.5f * ks.w);
        if (f < 0) f = cone_crystal_exact(cs, p, kp.x, kp.y, kp.z, ks.w) ? 1 : 0;
        if (!f) continue;
        att += len * kp.w;
        if (RECORD && len > 0.0f) {
            if (rec_c < kRecCrystals) rec[3 + kRecHoles + rec_c] = k;
            else atomicOr(status, kStatusRecordOverflow);
            ++rec_c;
        }
    }
    if (RECORD) {
        rec[0] = (int)plate_miss;
        rec[1] = rec_h < kRecHoles ? rec_h : kRecHoles;
        rec[2 + kRecHoles] = rec_c < kRecCrystals ? rec_c : kRecCrystals;
        if (plate_miss) return 0.0f;
    }
    return ray_value(D, ps, xDs, yDs, zDs, att, r, inv_r, dxw, dy, dzw);
}

// The warp's sum over every ray of voxel (ix, iy, iz) for detecting crystal d
// through trace_ray_global (same value on every lane); taken only for voxels
// whose candidates overflow the lists.
template <bool RECORD>
__device__ __forceinline__ float slow_voxel(const PEParams& P, const DevGeometry& G, const PeSmem& S, const Detecting& D,
                                         int d, int ix, int iy, int iz, int rec_slot, int lane) {
    float acc = 0.0f, comp = 0.0f;
    const int n = P.n_sv * P.n_sc;
    for (int e = lane; e < n; e += 32) {
        const int s = fast_div(e, P.n_sc, P.inv_n_sc);
        const int c = e - s * P.n_sc;                      // (sz * dX + sx) * dY + sy, the oracle's order
        const int t = fast_div(c, P.dY, P.inv_dY);
        const int sy = c - t * P.dY;
        const int sz = fast_div(t, P.dX, P.inv_dX);
        const int sx = t - sz * P.dX;
        const Vec3 p = subpoint_of(P, ix, iy, iz, s);
        const ConeSelf cs = cone_self(D, p);
        Vec3 ps;
        ps.x = (p.x - D.cx) * D.cm - (p.z - D.cz) * D.sm;
        ps.y = p.y - D.cy;
        ps.z = (p.x - D.cx) * D.sm + (p.z - D.cz) * D.cm;
        const SubCell cell = sub_cell(D, S, sx, sy, sz);
        int* rec = nullptr;
        if (RECORD) rec = P.rec_out + ((long long)rec_slot * P.n_sv * P.n_sc + (long long)e) * kRecWords;
        const float v = trace_ray_global<RECORD>(G, D, d, p, ps, cs, cell, rec, P.status);
        const float y = v - comp;
        const float tt = acc + y;
        comp = (tt - acc) - y;
        acc = tt;
    }
    float v = acc - comp;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Ordered compaction of a warp-wide predicate into a list; returns the new count.
// Entries beyond `cap` are counted but not stored.
__device__ __forceinline__ int warp_append(bool pass, int value, unsigned short* list, int count, int cap, int lane) {
    const unsigned bal = __ballot_sync(0xffffffffu, pass);
    const int pos = count + __popc(bal & lanemask_lt());
    if (pass && pos < cap) list[pos] = (unsigned short)value;
    return count + __popc(bal);
}

// One tile (8 crystals x one voxel brick) of geometry G.  Shared by the
// one-launch-per-geometry kernel and the persistent batch kernel.
template <bool RECORD>
__device__ __forceinline__ void pe_tile(const PEParams& P, const DevGeometry& G, PeSmem& S, long long tile) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    const int ct = (int)(tile % P.n_ctiles);
    const long long vt = tile / P.n_ctiles;
    const int bxi = (int)(vt % P.tiles_x);
    const int byi = (int)((vt / P.tiles_x) % P.tiles_y);
    const int bzi = (int)(vt / ((long long)P.tiles_x * P.tiles_y));
    const int ix0 = bxi * P.bx, iy0 = byi * P.by, iz0 = P.z0 + bzi * P.bz;
    const int ix1 = min(ix0 + P.bx, P.nx), iy1 = min(iy0 + P.by, P.ny), iz1 = min(iz0 + P.bz, P.z0 + P.nzs);
    const int d0 = P.row0 + ct * kPeWarps;

    // Sub-cell centre fractions (s + 0.5) / d, rounded as the reference rounds them.
    for (int i = tid; i < 3 * kMaxSubcellsPerAxis; i += kPeThreads) {
        const int a = i / kMaxSubcellsPerAxis, s = i - a * kMaxSubcellsPerAxis;
        const int dv = a == 0 ? P.dX : (a == 1 ? P.dY : P.dZ);
        S.frac[a][s] = ((float)s + 0.5f) / (float)dv;
    }

    // ---- 1. tile cull -------------------------------------------------------
    // Sub-point box of a voxel range: extreme fine voxel centres, rotated.
    auto point_box_of = [&](int ax0, int ay0, int az0, int ax1, int ay1, int az1) {
        Vec3 c0 = subpoint(P, ax0 * P.kx, ay0 * P.ky, az0 * P.kz);
        Vec3 c1 = subpoint(P, ax1 * P.kx - 1, ay0 * P.ky, az0 * P.kz);
        Vec3 c2 = subpoint(P, ax0 * P.kx, ay1 * P.ky - 1, az0 * P.kz);
        Vec3 c3 = subpoint(P, ax1 * P.kx - 1, ay1 * P.ky - 1, az0 * P.kz);
        Vec3 c4 = subpoint(P, ax0 * P.kx, ay0 * P.ky, az1 * P.kz - 1);
        Box3 A;
        A.x1 = fminf(fminf(c0.x, c1.x), fminf(c2.x, c3.x)) - kMargin;
        A.x2 = fmaxf(fmaxf(c0.x, c1.x), fmaxf(c2.x, c3.x)) + kMargin;
        A.y1 = fminf(fminf(c0.y, c1.y), fminf(c2.y, c3.y)) - kMargin;
        A.y2 = fmaxf(fmaxf(c0.y, c1.y), fmaxf(c2.y, c3.y)) + kMargin;
        A.z1 = fminf(c0.z, c4.z) - kMargin;
        A.z2 = fmaxf(c0.z, c4.z) + kMargin;
        return A;
    };
    const Box3 A = point_box_of(ix0, iy0, iz0, ix1, iy1, iz1);
    if (tid < kPeWarps) {
        const int d = d0 + tid;
        if (d < P.row1) {
            const float4 lo = G.c.lo[d], hi = G.c.hi[d];
            S.d_box[tid] = Box3{lo.x - kMargin, lo.y - kMargin, lo.z - kMargin, hi.x + kMargin, hi.y + kMargin, hi.z + kMargin};
        } else {
            S.d_box[tid] = Box3{1e30f, 1e30f, 1e30f, -1e30f, -1e30f, -1e30f};
        }
    }
    __syncthreads();
    const int n_d = min(kPeWarps, P.row1 - d0);
    // The tile's crystals side by side: a candidate the bundle from A to their
    // union box misses is missed by every crystal's own bundle.
    Box3 U = S.d_box[0];
    for (int j = 1; j < n_d; ++j) {
        const Box3 b = S.d_box[j];
        U = Box3{fminf(U.x1, b.x1), fminf(U.y1, b.y1), fminf(U.z1, b.z1), fmaxf(U.x2, b.x2), fmaxf(U.y2, b.y2),
                 fmaxf(U.z2, b.z2)};
    }
    const Bundle bu = make_bundle(A, U);
    auto tile_hit = [&](const Box3& K) {
        if (!bundle_hit(bu, K)) return false;
        if (n_d == 1) return true;
        for (int j = 0; j < n_d; ++j)
            if (bundle_hit(make_bundle(A, S.d_box[j]), K)) return true;
        return false;
    };

    int base = 0;
    for (int k0 = 0; k0 < G.n_crystals; k0 += kPeThreads) {
        const int k = k0 + tid;
        bool pass = false;
        float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), hi = lo;
        if (k < G.n_crystals) {
            lo = G.c.lo[k];
            hi = G.c.hi[k];
            const Box3 K{lo.x - kMargin, lo.y - kMargin, lo.z - kMargin, hi.x + kMargin, hi.y + kMargin, hi.z + kMargin};
            pass = tile_hit(K);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, pass);
        if (lane == 0) S.warp_cnt[warp] = __popc(bal);
        __syncthreads();
        int off = base, total = 0;
        for (int w = 0; w < kPeWarps; ++w) {
            const int cnt = S.warp_cnt[w];
            if (w < warp) off += cnt;
            total += cnt;
        }
        off += __popc(bal & lanemask_lt());
        if (pass) {
            if (off < kSupC) {
                S.c_pos[off] = G.c.pos[k];
                S.c_size[off] = G.c.size[k];
                const float4 rr = G.c.rot[k];
                S.c_lo[off] = make_float4(lo.x - kMargin, lo.y - kMargin, lo.z - kMargin, rr.x);
                S.c_hi[off] = make_float4(hi.x + kMargin, hi.y + kMargin, hi.z + kMargin, rr.y);
                S.c_id[off] = k;
            }
        }
        base += total;
        __syncthreads();
    }
    const int n_c = min(base, kSupC);
    const bool over_c = base > kSupC;
    base = 0;
    for (int k0 = 0; k0 < G.n_holes; k0 += kPeThreads) {
        const int k = k0 + tid;
        bool pass = false;
        float4 ha = make_float4(0.f, 0.f, 0.f, 0.f), hb = ha;
        if (k < G.n_holes) {
            ha = G.h.a[k];
            hb = G.h.b[k];
            const Box3 K = hole_box(ha, hb);
            pass = tile_hit(K);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, pass);
        if (lane == 0) S.warp_cnt[warp] = __popc(bal);
        __syncthreads();
        int off = base, total = 0;
        for (int w = 0; w < kPeWarps; ++w) {
            const int cnt = S.warp_cnt[w];
            if (w < warp) off += cnt;
            total += cnt;
        }
        off += __popc(bal & lanemask_lt());
        if (pass) {
            if (off < kSupH) {
                S.h_a[off] = ha;
                S.h_b[off] = hb;
                S.h_id[off] = k;
            }
        }
        base += total;
        __syncthreads();
    }
    const int n_h = min(base, kSupH);
    if (tid == 0) {
        S.n_c = n_c;
        S.n_h = n_h;
        S.overflow = over_c || base > kSupH;
    }
    __syncthreads();

    // ---- 2. per-warp crystal, voxel walk --------------------------------------
    const int tv = P.bx * P.by * P.bz;
    const int d = d0 + warp;
    WarpLists& L = S.wl[warp];
    if (d < P.row1) {
        Detecting D;
        {
            const float4 pos = G.c.pos[d], sz = G.c.size[d], rt = G.c.rot[d], ph = G.c.phys[d];
            D.cx = pos.x; D.cy = pos.y; D.cz = pos.z; D.mu_t = pos.w; D.mu_pe = ph.x;
            D.w = sz.x; D.t = sz.y; D.h = sz.z; D.crit = sz.w;
            D.cm = rt.x; D.sm = rt.y; D.cp = rt.z; D.sp = rt.w;
            D.world = S.d_box[warp];
            D.area_x = D.t * D.h / (float)P.dZ / (float)P.dY;
            D.area_z = D.w * D.t / (float)P.dX / (float)P.dY;
            D.area_y = D.w * D.h / (float)P.dX / (float)P.dZ;
            D.hx = 0.5f * D.w / (float)P.dX;
            D.hy = 0.5f * D.t / (float)P.dY;
            D.hz = 0.5f * D.h / (float)P.dZ;
        }
        const bool absorbing = D.mu_t > 0.01f;   // PESysMatGen.cu:504, :598
        // Candidates the whole brick can reach for this crystal (bundle from the
        // brick's sub-point box A): the per-voxel lists narrow from these when
        // they fit, instead of from the tile's staged set.
        bool brick = false;
        if (absorbing && !S.overflow) {
            const Bundle bb = make_bundle(A, D.world);
            int nb = 0;
            for (int k0 = 0; k0 < n_c; k0 += 32) {
                const int k = k0 + lane;
                const bool pass = k < n_c && S.c_id[k] != d && bundle_hit(bb, box_of(S.c_lo[k], S.c_hi[k]));
                nb = warp_append(pass, k, L.blist_c, nb, kListC, lane);
            }
            int nbh = 0;
            for (int k0 = 0; k0 < n_h; k0 += 32) {
                const int k = k0 + lane;
                const bool pass = k < n_h && bundle_hit(bb, hole_box(S.h_a[k], S.h_b[k]));
                nbh = warp_append(pass, k, L.blist_h, nbh, kListH, lane);
            }
            brick = nb <= kListC && nbh <= kListH;
            if (lane == 0) {
                L.nb_c = nb;
                L.nb_h = nbh;
            }
            __syncwarp();
        }
        unsigned long long cnt_rays = 0, cnt_cry = 0, cnt_hole = 0, cnt_cone = 0;
        unsigned long long* pc_cry = P.counters ? &cnt_cry : nullptr;
        unsigned long long* pc_hole = P.counters ? &cnt_hole : nullptr;
        unsigned long long* pc_cone = P.counters ? &cnt_cone : nullptr;
        // Entries of few rays go VP neighbouring voxels of the brick to a group
        // (P.pair, up to 8): a pass then traces one sub-cell column from all of
        // them, and the lanes of each voxel are summed apart.
        const int VP = RECORD ? 1 : P.pair;
        for (int vl = 0; vl < tv; vl += VP) {
            // voxel u of the group is brick voxel vl + u
            auto vox_of = [&](int u, int& x, int& y, int& z) {
                const int b = vl + u;
                x = ix0 + b % P.bx;
                y = iy0 + (b / P.bx) % P.by;
                z = iz0 + b / (P.bx * P.by);
            };
            int ix, iy, iz;
            vox_of(0, ix, iy, iz);
            unsigned valid = 0u;
            int lox = 1 << 30, loy = 1 << 30, loz = 1 << 30, hix = -1, hiy = -1, hiz = -1;
            for (int u = 0; u < VP; ++u) {
                int x, y, z;
                vox_of(u, x, y, z);
                if (vl + u < tv && x < ix1 && y < iy1 && z < iz1) {
                    valid |= 1u << u;
                    lox = min(lox, x); loy = min(loy, y); loz = min(loz, z);
                    hix = max(hix, x); hiy = max(hiy, y); hiz = max(hiz, z);
                }
            }
            if (!valid) continue;
            int rec_slot = -1;
            if (RECORD) {
                const long long vox = ((long long)iz * P.ny + iy) * P.nx + ix;
                for (int i = 0; i < P.rec_n; ++i)
                    if (P.rec_rows[i] == d && P.rec_vox[i] == vox) rec_slot = i;
                if (rec_slot < 0) continue;
            }
            float acc = 0.0f, comp = 0.0f;
            int lane_vox = 0;
            if (absorbing) {
                // Voxel-level candidate lists: staged crystals/holes the bundle from
                // the sub-points of the group's voxels (the box of their voxel
                // range) to the crystal can reach.
                const Box3 Avox = point_box_of(lox, loy, loz, hix + 1, hiy + 1, hiz + 1);
                bool slow = S.overflow != 0;
                if (!slow) {
                    const Bundle bv = make_bundle(Avox, D.world);
                    int cnt = 0;
                    const int src_c = brick ? L.nb_c : n_c;
                    for (int i0 = 0; i0 < src_c; i0 += 32) {
                        const int i = i0 + lane;
                        int k = i;
                        bool pass = false;
                        if (i < src_c) {
                            k = brick ? (int)L.blist_c[i] : i;
                            pass = (brick || S.c_id[k] != d) && bundle_hit(bv, box_of(S.c_lo[k], S.c_hi[k]));
                        }
                        cnt = warp_append(pass, k, L.list_c, cnt, kListC, lane);
                    }
                    int cnth = 0;
                    const int src_h = brick ? L.nb_h : n_h;
                    for (int i0 = 0; i0 < src_h; i0 += 32) {
                        const int i = i0 + lane;
                        int k = i;
                        bool pass = false;
                        if (i < src_h) {
                            k = brick ? (int)L.blist_h[i] : i;
                            pass = bundle_hit(bv, hole_box(S.h_a[k], S.h_b[k]));
                        }
                        cnth = warp_append(pass, k, L.list_h, cnth, kListH, lane);
                    }
                    slow = cnt > kListC || cnth > kListH;
                    cnt = min(cnt, kListC);
                    cnth = min(cnth, kListH);
                    __syncwarp();
                    // First list index of each plate's holes (hole ids ascend with the plate).
                    for (int m = 0; m <= G.n_plates; ++m) {
                        const int first = (m < G.n_plates) ? G.plate[m].hole_begin : G.n_holes;
                        int below = 0;
                        for (int i0 = 0; i0 < cnth; i0 += 32) {
                            const int i = i0 + lane;
                            below += __popc(__ballot_sync(0xffffffffu, i < cnth && S.h_id[L.list_h[i]] < first));
                        }
                        if (lane == 0) L.plate_begin[m] = below;
                    }
                    if (lane == 0) {
                        L.n_c = cnt;
                        L.n_h = cnth;
                    }
                    __syncwarp();
                }
                if (slow) {
                    // The candidates do not fit the shared-memory lists: the group's
                    // voxels through the geometry tables, same decisions and values.
                    for (int u = 0; u < VP; ++u) {
                        if (!((valid >> u) & 1u)) continue;
                        int x, y, z;
                        vox_of(u, x, y, z);
                        const float w = slow_voxel<RECORD>(P, G, S, D, d, x, y, z, rec_slot, lane);
                        if (lane == 0) S.out[warp][vl + u] = w * P.inv_sv;
                    }
                    __syncwarp();
                    continue;
                }
                const int lc = L.n_c, lh = L.n_h;
                const int nwc = (lc + 31) >> 5, nwh = (lh + 31) >> 5;
                // points of the group: the sub-points of voxel 0, then of voxel 1, ...
                const int n_pts = VP * P.n_sv;
                for (int s0 = 0; s0 < n_pts; s0 += P.group) {
                    const int gn = min(P.group, n_pts - s0);
                    // The cone (ConeSelf) of each sub-point of the group, for the
                    // cone tests trace_ray takes on the candidates a ray crosses.
                    if (lane < gn) {
                        const int u = (VP == 1) ? 0 : (s0 + lane) / P.n_sv;
                        int x = ix, y = iy, z = iz;
                        if (u > 0) vox_of(u, x, y, z);
                        const Vec3 p = subpoint_of(P, x, y, z, s0 + lane - u * P.n_sv);
                        const ConeSelf cs = cone_self(D, p);
                        L.cs[lane] = make_float4(cs.ux, cs.uy, cs.uz, cs.crit_self);
                        L.pt[lane] = make_float4(p.x, p.y, p.z, 0.0f);
                        L.pself[lane] = make_float4((p.x - D.cx) * D.cm - (p.z - D.cz) * D.sm, p.y - D.cy,
                                                    (p.x - D.cx) * D.sm + (p.z - D.cz) * D.cm, 0.0f);
                    }
                    __syncwarp();
                    // Rays of the group, ordered (sub-cell column, sub-point, depth
                    // sub-cell) and dealt 32 to a warp pass: a pass traces the depth
                    // cells of one column (or a few) from neighbouring sub-points,
                    // rays that run almost together through the plates and the
                    // crystals in front, so the lanes meet the same candidates.
                    const int cb = gn * P.dY;                  // rays per sub-cell column
                    const float inv_cb = 1.0f / (float)cb;
                    const int nr = gn * P.n_sc;
                    // Full groups of one voxel deal the same sub-cells to the same
                    // passes, so the first group's pass masks serve the others.
                    const bool keep = VP == 1 && gn == P.group && nr <= 32 * kPassSlots;
                    for (int q0 = 0; q0 < nr; q0 += 32) {
                        const int slot = keep ? (q0 >> 5) : 0;
                        const int e = q0 + lane;
                        bool active = e < nr;
                        int j = 0, sx = 0, sy = 0, sz = 0, u = 0;
                        if (active) {
                            const int col = fast_div(e, cb, inv_cb);
                            const int r = e - col * cb;
                            j = fast_div(r, P.dY, P.inv_dY);
                            sy = r - j * P.dY;
                            sz = fast_div(col, P.dX, P.inv_dX);
                            sx = col - sz * P.dX;
                            if (VP > 1) {
                                u = (s0 + j) / P.n_sv;
                                active = (valid >> u) & 1u;
                                lane_vox = u;
                            }
                        }
                        const SubCell cell = sub_cell(D, S, sx, sy, sz);
                        if (nr <= 32) {
                            // One pass holds every ray of the group: its bundle is the
                            // voxel's own, which the list was built from.
                            if (lane < nwc) {
                                const int n_in = lc - (lane << 5);
                                L.pass_c[slot][lane] = n_in >= 32 ? 0xffffffffu : ((1u << n_in) - 1u);
                            }
                            if (lane < nwh) {
                                const int n_in = lh - (lane << 5);
                                L.pass_h[slot][lane] = n_in >= 32 ? 0xffffffffu : ((1u << n_in) - 1u);
                            }
                        } else if (!(keep && s0 > 0)) {
                            // The pass's bundle: from the voxel's sub-point box to the
                            // box of its rays' sub-cell centres.
                            float bx1 = active ? cell.q.x : 3.0e38f, bx2 = active ? cell.q.x : -3.0e38f;
                            float by1 = active ? cell.q.y : 3.0e38f, by2 = active ? cell.q.y : -3.0e38f;
                            float bz1 = active ? cell.q.z : 3.0e38f, bz2 = active ? cell.q.z : -3.0e38f;
                            for (int o = 16; o > 0; o >>= 1) {
                                bx1 = fminf(bx1, __shfl_xor_sync(0xffffffffu, bx1, o));
                                bx2 = fmaxf(bx2, __shfl_xor_sync(0xffffffffu, bx2, o));
                                by1 = fminf(by1, __shfl_xor_sync(0xffffffffu, by1, o));
                                by2 = fmaxf(by2, __shfl_xor_sync(0xffffffffu, by2, o));
                                bz1 = fminf(bz1, __shfl_xor_sync(0xffffffffu, bz1, o));
                                bz2 = fmaxf(bz2, __shfl_xor_sync(0xffffffffu, bz2, o));
                            }
                            const Bundle bq = make_bundle(Avox, Box3{bx1, by1, bz1, bx2, by2, bz2});
                            // Narrow the voxel's candidates to those the pass can reach; a
                            // candidate dropped here is one that no ray of the pass can
                            // reach, i.e. one trace_ray would skip by its own window test.
                            for (int w = 0; w < nwc; ++w) {
                                bool pass = false;
                                if ((w << 5) + lane < lc) {
                                    const int k = L.list_c[(w << 5) + lane];
                                    pass = bundle_hit(bq, box_of(S.c_lo[k], S.c_hi[k]));
                                }
                                const unsigned bal = __ballot_sync(0xffffffffu, pass);
                                if (lane == 0) L.pass_c[slot][w] = bal;
                            }
                            for (int w = 0; w < nwh; ++w) {
                                bool pass = false;
                                if ((w << 5) + lane < lh) {
                                    const int k = L.list_h[(w << 5) + lane];
                                    pass = bundle_hit(bq, hole_box(S.h_a[k], S.h_b[k]));
                                }
                                const unsigned bal = __ballot_sync(0xffffffffu, pass);
                                if (lane == 0) L.pass_h[slot][w] = bal;
                            }
                        }
                        __syncwarp();
                        if (active) {
                            const float4 p4 = L.pt[j], ps4 = L.pself[j];
                            const Vec3 p{p4.x, p4.y, p4.z};
                            const Vec3 ps{ps4.x, ps4.y, ps4.z};
                            int* rec = nullptr;
                            if (RECORD) {
                                const int c = (sz * P.dX + sx) * P.dY + sy;   // the oracle's sub-cell order
                                rec = P.rec_out + ((long long)rec_slot * P.n_sv * P.n_sc + (long long)(s0 + j) * P.n_sc + c) *
                                                      kRecWords;
                            }
                            const float v = trace_ray<RECORD>(P, G, S, L, L.pass_c[slot], L.pass_h[slot], &L.cs[j], D,
                                                              p, ps, cell, rec, P.status,
                                                              pc_cry, pc_hole, pc_cone);
                            if (P.counters) ++cnt_rays;
                            // Kahan summation of the lane's rays.
                            const float y = v - comp;
                            const float t = acc + y;
                            comp = (t - acc) - y;
                            acc = t;
                        }
                        __syncwarp();
                    }
                    __syncwarp();
                }
            }
            const float v = acc - comp;
            for (int u = 0; u < VP; ++u) {
                // a lane's rays all belong to one voxel of the group (pe_plan
                // picks VP so that the lane-to-point map is the same every pass)
                float w = lane_vox == u ? v : 0.0f;
                for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
                if (lane == 0 && ((valid >> u) & 1u)) S.out[warp][vl + u] = w * P.inv_sv;
            }
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

template <bool RECORD>
__global__ void __launch_bounds__(kPeThreads, 2) pe_trace_kernel(PEParams P, DevGeometry G) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PeSmem& S = *reinterpret_cast<PeSmem*>(smem_raw);
    const long long tile = P.tile_list ? P.tile_list[blockIdx.x] : (long long)blockIdx.x;
    pe_tile<RECORD>(P, G, S, tile);
}

// The batch's geometries, in constant memory: the tile code reads launch
// parameters in its inner loops, and constant-bank loads of a warp-uniform
// index cost what kernel-parameter loads cost.  Written by the batch's own
// graph (a device-to-device copy before each chunk's launch).
__constant__ PeBatchGeom c_batch[kBatchConst];

// Persistent kernel over the (geometry, tile) items of up to kBatchConst
// geometries: each CTA takes the next item from a global counter until all
// are done.  Geometries are laid out largest first, so the dynamic hand-out
// balances the tail.  No CTA waits on another: the counter only hands out work.
__global__ void __launch_bounds__(kPeThreads, 2) pe_batch_kernel(int n_geoms, long long total,
                                                                 unsigned long long* counter) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PeSmem& S = *reinterpret_cast<PeSmem*>(smem_raw);
    __shared__ long long s_item;
    __shared__ int s_geom;
    for (;;) {
        if (threadIdx.x == 0) {
            const long long item = (long long)atomicAdd(counter, 1ULL);
            int lo = 0, hi = n_geoms - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (c_batch[mid].tile_begin <= item) lo = mid;
                else hi = mid - 1;
            }
            s_item = item;
            s_geom = lo;
        }
        __syncthreads();
        const long long item = s_item;
        const int g = s_geom;
        if (item >= total) break;
        pe_tile<false>(c_batch[g].P, c_batch[g].G, S, item - c_batch[g].tile_begin);
        __syncthreads();
    }
}

}  // namespace

size_t pe_smem_bytes() { return sizeof(PeSmem); }

// The dynamic shared memory limit is a per-device function attribute: set it
// once per (device, kernel).
static cudaError_t allow_smem(const void* fn, int which) {
    static unsigned long long done[3] = {0, 0, 0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 64 && (done[which] >> dev) & 1ULL) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(PeSmem));
    if (e == cudaSuccess && dev < 64) done[which] |= 1ULL << dev;
    return e;
}

cudaError_t pe_launch(const PEParams& p, const DevGeometry& geo, bool record, long long n_tiles, cudaStream_t stream) {
    const size_t smem = sizeof(PeSmem);
    if (n_tiles <= 0) return cudaSuccess;
    if (n_tiles > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    if (record) {
        cudaError_t e = allow_smem((const void*)pe_trace_kernel<true>, 0);
        if (e != cudaSuccess) return e;
        pe_trace_kernel<true><<<(unsigned)n_tiles, kPeThreads, smem, stream>>>(p, geo);
    } else {
        cudaError_t e = allow_smem((const void*)pe_trace_kernel<false>, 1);
        if (e != cudaSuccess) return e;
        pe_trace_kernel<false><<<(unsigned)n_tiles, kPeThreads, smem, stream>>>(p, geo);
    }
    return cudaGetLastError();
}

cudaError_t pe_batch_launch(const PeBatchGeom* geoms, int n_geoms, long long total, unsigned long long* counter,
                            int grid, cudaStream_t stream) {
    if (total <= 0) return cudaSuccess;
    if (n_geoms < 1 || n_geoms > kBatchConst) return cudaErrorInvalidValue;
    cudaError_t e = allow_smem((const void*)pe_batch_kernel, 2);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbolAsync(c_batch, geoms, sizeof(PeBatchGeom) * (size_t)n_geoms, 0, cudaMemcpyDeviceToDevice,
                                stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    pe_batch_kernel<<<grid, kPeThreads, sizeof(PeSmem), stream>>>(n_geoms, total, counter);
    return cudaGetLastError();
}

int pe_batch_blocks_per_sm() {
    int n = 0;
    if (allow_smem((const void*)pe_batch_kernel, 2) != cudaSuccess) return 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pe_batch_kernel, kPeThreads, sizeof(PeSmem)) != cudaSuccess)
        return 1;
    return n > 0 ? n : 1;
}

}  // namespace smb
