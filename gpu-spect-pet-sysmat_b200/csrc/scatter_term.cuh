// One term of the primary-Compton scatter sysmat, host- and device-callable:
// the kernels in scatter_kernel.cu evaluate it on the GPU, and host-side
// checks run the same arithmetic on the CPU.  See scatter_kernel.cu for the
// physics and the reference lines each step follows.
#pragma once

#include <cmath>

#include "scatter.h"
#include "tracer.cuh"

namespace smb {

constexpr float kDelta = 0.01f;   // the reference's DeltaTheta, as a float
constexpr float kNodesPerRad = (float)kKnNodes / 3.14159265358979323846f;

SM_HD float sm_rsqrt(float x) {
#ifdef __CUDA_ARCH__
    return rsqrtf(x);
#else
    return 1.0f / std::sqrt(x);
#endif
}

SM_HD int sm_rint(float x) {
#ifdef __CUDA_ARCH__
    return __float2int_rn(x);
#else
    return (int)std::nearbyint(x);
#endif
}

// ---- Klein-Nishina rectangle sum in closed form ---------------------------------------
// sum_{i=0}^{n} g(a + i delta) delta = [F(b) - F(a)] + delta/2 (g(a) + g(b))
//   + delta^2/12 (g'(b) - g'(a)) + O(delta^4 g'''),  b = a + n delta.
struct KnEval {
    float f_hi, f_lo, part, g, dg;
};

SM_HD KnEval kn_at(const KnNode* kn, float theta) {
    int j = sm_rint(theta * kNodesPerRad);
    j = j < 0 ? 0 : (j > kKnNodes ? kKnNodes : j);
    const KnNode n = kn[j];
    const float t = theta - n.theta;
    KnEval e;
    e.f_hi = n.f_hi;
    e.f_lo = n.f_lo;
    e.part = t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, n.c4 * 0.2f, n.c3 * 0.25f), n.c2 * (1.0f / 3.0f)), n.c1 * 0.5f), n.c0);
    e.g = fmaf(t, fmaf(t, fmaf(t, fmaf(t, n.c4, n.c3), n.c2), n.c1), n.c0);
    e.dg = fmaf(t, fmaf(t, fmaf(t, 4.0f * n.c4, 3.0f * n.c3), 2.0f * n.c2), n.c1);
    return e;
}

SM_HD float kn_rect_sum(const KnNode* kn, float a, int n) {
    const float b = a + (float)n * kDelta;     // the reference's last sample, theta_low + n * DeltaTheta
    const KnEval A = kn_at(kn, a), B = kn_at(kn, b);
    const float integral = ((B.f_hi - A.f_hi) + (B.f_lo - A.f_lo)) + (B.part - A.part);
    return integral + 0.5f * kDelta * (A.g + B.g) + (kDelta * kDelta / 12.0f) * (B.dg - A.dg);
}

// angle between u and e (atan2 of |u x e| and u . e: accurate at every angle)
SM_HD float angle_between(float ux, float uy, float uz, float ex, float ey, float ez) {
    const float cx = uy * ez - uz * ey, cy = uz * ex - ux * ez, cz = ux * ey - uy * ex;
    return atan2f(sqrtf(fmaf(cx, cx, fmaf(cy, cy, cz * cz))), fmaf(ux, ex, fmaf(uy, ey, uz * ez)));
}

// Per-lane constants of the detecting crystal.
struct Det {
    float x, y, z, cm, sm;       // centre (world, y with Image[11]); cos(-rot), sin(-rot)
    float hw, ht, hh;            // half sizes
    float r_unit;                // bounding radius of the unit (scatter.cu:1243)
    float mu_pe, mu_c, res, lo, hi;
    bool on;
};

// Per-(lane, scatter point) constants.
struct Src {
    float sx, sy, sz;            // scatter point, world
    float ssx, ssy, ssz;         // ... in the detecting crystal's frame
    float bx, by, bz, bb, L;     // D - S, |D - S|^2, |D - S|
    float e[8][3];               // unit vectors from S to the unit's corners (detector frame)
    float4 pr;                   // pair data
};

SM_HD void make_src(const Det& D, float4 S, float4 pr, Src& C) {
    C.sx = S.x;
    C.sy = S.y;
    C.sz = S.z;
    C.ssx = (S.x - D.x) * D.cm - (S.z - D.z) * D.sm;
    C.ssy = S.y - D.y;
    C.ssz = (S.x - D.x) * D.sm + (S.z - D.z) * D.cm;
    C.bx = D.x - S.x;
    C.by = D.y - S.y;
    C.bz = D.z - S.z;
    C.bb = fmaf(C.bx, C.bx, fmaf(C.by, C.by, C.bz * C.bz));
    C.L = sqrtf(C.bb);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float ex = ((i & 1) ? D.hw : -D.hw) - C.ssx;
        const float ey = ((i & 2) ? D.ht : -D.ht) - C.ssy;
        const float ez = ((i & 4) ? D.hh : -D.hh) - C.ssz;
        const float inv = sm_rsqrt(fmaf(ex, ex, fmaf(ey, ey, ez * ez)));
        C.e[i][0] = ex * inv;
        C.e[i][1] = ey * inv;
        C.e[i][2] = ez * inv;
    }
    C.pr = pr;
}

// One term without its weight W.  I: voxel (world); Is: voxel in the detector frame.
SM_HD float scatter_term(const ScatterParams& P, const Det& D, const Src& C, const KnNode* kn,
                                              float inv_norm, float ix, float iy, float iz, float isx, float isy,
                                              float isz) {
    // scatter angle at S between I -> S and S -> D (scatter.cu:1225)
    const float ax = C.sx - ix, ay = C.sy - iy, az = C.sz - iz;
    const float aa = fmaf(ax, ax, fmaf(ay, ay, az * az));
    const float inv_ab = sm_rsqrt(aa * C.bb);
    float c = fmaf(ax, C.bx, fmaf(ay, C.by, az * C.bz)) * inv_ab;
    c = fminf(1.0f, fmaxf(-1.0f, c));
    const float r = fmaf(P.alpha, 1.0f - c, 1.0f);       // E0 / E'
    const float E = P.e0 / r;
    const float res_e = D.res * sqrtf(E / P.e0);
    const float k2 = 2.0f * res_e / 2.35482f;
    if ((E * (1.0f + k2) <= D.lo) || (E * (1.0f - k2) >= D.hi)) return 0.0f;   // 2-sigma window cut (:1231)
    const float s2 = res_e / 2.35482f * E * 1.41421356237309515f;
    // 0.5 (erf(z2) - erf(z1)), through erfc when both limits lie on one side of E'
    const float z1 = (D.lo - E) / s2, z2 = (D.hi - E) / s2;
    float p_win;
    if (z1 > 0.0f) p_win = 0.5f * (erfcf(z1) - erfcf(z2));
    else if (z2 < 0.0f) p_win = 0.5f * (erfcf(-z2) - erfcf(-z1));
    else p_win = 0.5f * (erff(z2) - erff(z1));
    // azimuth range (:1244-1252)
    const float cx = ay * C.bz - az * C.by, cy = az * C.bx - ax * C.bz, cz = ax * C.by - ay * C.bx;
    const float sn = sqrtf(fmaf(cx, cx, fmaf(cy, cy, cz * cz))) * inv_ab;
    float phi_frac = 1.0f;
    if (!(C.L * sn * 2.0f <= D.r_unit)) phi_frac = 4.0f * asinf(fminf(D.r_unit / 2.0f / C.L / sn, 1.0f)) * 0.159154943091895336f;
    // polar range over the unit's corners (:1272-1298)
    const float ux = C.ssx - isx, uy = C.ssy - isy, uz = C.ssz - isz;
    // u . e_i orders the corners by angle (u is not normalised: the scale is common)
    float cmax = fmaf(ux, C.e[0][0], fmaf(uy, C.e[0][1], uz * C.e[0][2])), cmin = cmax;
    float nx0 = C.e[0][0], ny0 = C.e[0][1], nz0 = C.e[0][2], fx0 = nx0, fy0 = ny0, fz0 = nz0;   // nearest / farthest
#pragma unroll
    for (int i = 1; i < 8; ++i) {
        const float ci = fmaf(ux, C.e[i][0], fmaf(uy, C.e[i][1], uz * C.e[i][2]));
        if (ci > cmax) { cmax = ci; nx0 = C.e[i][0]; ny0 = C.e[i][1]; nz0 = C.e[i][2]; }
        if (ci < cmin) { cmin = ci; fx0 = C.e[i][0]; fy0 = C.e[i][1]; fz0 = C.e[i][2]; }
    }
    float th_lo = angle_between(ux, uy, uz, nx0, ny0, nz0);
    const float th_hi = angle_between(ux, uy, uz, fx0, fy0, fz0);
    // the line from the voxel through S continues into the unit: theta_min = 0 (:1264-1266, :1293-1296)
    const float dis = sqrtf(fmaf(ux, ux, fmaf(uy, uy, uz * uz)));
    const float xt = C.ssx + 1000.0f * (C.ssx - isx) / dis;
    const float yt = C.ssy + 1000.0f * (C.ssy - isy) / dis;
    const float zt = C.ssz + 1000.0f * (C.ssz - isz) / dis;
    const Box3 ub{-D.hw, -D.ht, -D.hh, D.hw, D.ht, D.hh};
    if (chord_through(isx, isy, isz, xt, yt, zt, ub) > 0.001f) th_lo = 0.0f;
    const int n = (int)((th_hi - th_lo) / kDelta);
    const float ratio = kn_rect_sum(kn, th_lo, n) * inv_norm;
    // attenuation and absorption at E' (:1309-1392)
    const float r3 = r * r * r;
    const float mu_pe = D.mu_pe * r3, mu_c = D.mu_c * r, mu = mu_pe + mu_c;
    const float att = fmaf(C.pr.x, r3, fmaf(C.pr.y, r, C.pr.z * mu));
    const float absorb = -expm1f(-C.pr.w * mu) * mu_pe / mu;
    return phi_frac * ratio * p_win * expf(-att) * absorb;
}

}  // namespace smb
