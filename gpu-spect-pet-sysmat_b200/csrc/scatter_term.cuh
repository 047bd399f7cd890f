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

// Fast quotient and square root for values (never for a decision the
// reference takes): about 2 ulp, against ~10 instructions for the IEEE forms
// this translation unit is compiled with.
SM_HD float sm_fdiv(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdividef(a, b);
#else
    return a / b;
#endif
}

SM_HD float sm_fsqrt(float x) { return x > 0.0f ? x * sm_rsqrt(x) : 0.0f; }

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
    return atan2f(sm_fsqrt(fmaf(cx, cx, fmaf(cy, cy, cz * cz))), fmaf(ux, ex, fmaf(uy, ey, uz * ez)));
}

// Per-lane constants of the detecting crystal.
struct Det {
    float x, y, z, cm, sm;       // centre (world, y with Image[11]); cos(-rot), sin(-rot)
    float hw, ht, hh;            // half sizes
    float r_unit;                // bounding radius of the unit (scatter.cu:1243)
    float mu_pe, mu_c, res, lo, hi;
    float c_cut;                 // cos(theta) at or below which the 2-sigma window cut rejects, less a margin
    bool on;
};

// The lower window cut as a bound on cos(theta): E' (1 + k sqrt(E'/E0)) <= lo
// (scatter.cu:1231) rejects every E' up to the root E*, i.e. every cos(theta)
// up to 1 - (E0/E* - 1)/alpha.  Returns that cosine less a margin of 2e-3
// (far above the rounding of the per-term test), -2 when nothing is cut and
// 2 when everything is.  The upper cut is left to the per-term test.
SM_HD float window_cos_cut(float e0, float alpha, float res, float lo) {
    const float k = 2.0f * res / 2.35482f;
    auto lhs = [&](float E) { return E * (1.0f + k * sqrtf(E / e0)) - lo; };
    float a = e0 / (1.0f + 2.0f * alpha), b = e0;   // E' over theta in [pi, 0]
    if (lhs(b) <= 0.0f) return 2.0f;
    if (lhs(a) > 0.0f) return -2.0f;
    for (int it = 0; it < 40; ++it) {
        const float m = 0.5f * (a + b);
        if (lhs(m) <= 0.0f) a = m;
        else b = m;
    }
    return 1.0f - (e0 / a - 1.0f) / alpha - 2e-3f;
}

// Per-(lane, scatter point) constants.
struct Src {
    float sx, sy, sz;            // scatter point, world
    float ssx, ssy, ssz;         // ... in the detecting crystal's frame
    float bx, by, bz, bb, L;     // D - S, |D - S|^2, |D - S|
    float phi_k;                 // R_unit / (2 L)
    float c_len;                 // below this cos(theta) the line I -> S misses the unit's bounding sphere
    float e[8][3];               // unit vectors from S to the unit's corners (detector frame)
    float4 pr;                   // pair data
};

// S, its detector-frame image and D - S: what the column cull needs.
SM_HD void make_src_basic(const Det& D, float4 S, Src& C) {
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
}

// The rest of the per-(lane, scatter point) constants.
SM_HD void make_src_rest(const Det& D, float4 pr, Src& C) {
    C.phi_k = D.r_unit / 2.0f / C.L;
    const float q = D.r_unit / C.L;
    C.c_len = q < 1.0f ? sqrtf(1.0f - q * q) - 1e-3f : -2.0f;
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

// Largest cos(theta) over the voxel column I0 + t e, t in [0, T] (|e| = 1):
// with w = S - I = w_perp + u e, u = (w0 . e) - t, cos = (B + u beta) / sqrt(A + u^2)
// (A = |w_perp|^2, B = w_perp . b^, beta = e . b^) is stationary only at u = beta A / B.
SM_HD float column_max_cos(const Src& C, float i0x, float i0y, float i0z, float ex, float ey, float ez, float T) {
    const float wx = C.sx - i0x, wy = C.sy - i0y, wz = C.sz - i0z;
    const float inv_l = sm_rsqrt(C.bb);
    const float bx = C.bx * inv_l, by = C.by * inv_l, bz = C.bz * inv_l;
    const float p = fmaf(wx, ex, fmaf(wy, ey, wz * ez));
    const float px = wx - p * ex, py = wy - p * ey, pz = wz - p * ez;
    const float A = fmaf(px, px, fmaf(py, py, pz * pz));
    const float B = fmaf(px, bx, fmaf(py, by, pz * bz));
    const float beta = fmaf(ex, bx, fmaf(ey, by, ez * bz));
    auto f = [&](float u) { return (B + u * beta) * sm_rsqrt(A + u * u); };
    float m = fmaxf(f(p), f(p - T));
    if (B != 0.0f) {
        const float us = beta * A / B;
        if (us > p - T && us < p) m = fmaxf(m, f(us));
    }
    return m;
}

SM_HD void make_src(const Det& D, float4 S, float4 pr, Src& C) {
    make_src_basic(D, S, C);
    make_src_rest(D, pr, C);
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
    const float E = sm_fdiv(P.e0, r);
    const float res_e = D.res * sm_rsqrt(r);                // res sqrt(E'/E0)
    const float k2 = res_e * (2.0f / 2.35482f);
    if ((E * (1.0f + k2) <= D.lo) || (E * (1.0f - k2) >= D.hi)) return 0.0f;   // 2-sigma window cut (:1231)
    const float inv_s2 = sm_fdiv(2.35482f / 1.41421356237309515f, res_e * E);   // 1 / (sigma sqrt 2)
    // 0.5 (erf(z2) - erf(z1)), through erfc when both limits lie on one side of E'
    const float z1 = (D.lo - E) * inv_s2, z2 = (D.hi - E) * inv_s2;
    float p_win;
    if (z1 > 0.0f) p_win = 0.5f * (erfcf(z1) - erfcf(z2));
    else if (z2 < 0.0f) p_win = 0.5f * (erfcf(-z2) - erfcf(-z1));
    else p_win = 0.5f * (erff(z2) - erff(z1));
    // azimuth range (:1244-1252)
    const float cx = ay * C.bz - az * C.by, cy = az * C.bx - ax * C.bz, cz = ax * C.by - ay * C.bx;
    const float sn = sm_fsqrt(fmaf(cx, cx, fmaf(cy, cy, cz * cz))) * inv_ab;
    float phi_frac = 1.0f;
    if (!(C.L * sn * 2.0f <= D.r_unit)) phi_frac = 4.0f * asinf(fminf(sm_fdiv(C.phi_k, sn), 1.0f)) * 0.159154943091895336f;
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
    // the line from the voxel through S continues into the unit: theta_min = 0 (:1264-1266, :1293-1296);
    // it cannot unless it passes the unit's bounding sphere (cos(theta) >= c_len)
    if (c >= C.c_len) {
        const float dis = sqrtf(fmaf(ux, ux, fmaf(uy, uy, uz * uz)));
        const float xt = C.ssx + 1000.0f * (C.ssx - isx) / dis;
        const float yt = C.ssy + 1000.0f * (C.ssy - isy) / dis;
        const float zt = C.ssz + 1000.0f * (C.ssz - isz) / dis;
        const Box3 ub{-D.hw, -D.ht, -D.hh, D.hw, D.ht, D.hh};
        if (chord_through(isx, isy, isz, xt, yt, zt, ub) > 0.001f) th_lo = 0.0f;
    }
    const int n = (int)((th_hi - th_lo) / kDelta);
    const float ratio = kn_rect_sum(kn, th_lo, n) * inv_norm;
    // attenuation and absorption at E' (:1309-1392)
    const float r3 = r * r * r;
    const float mu_pe = D.mu_pe * r3, mu_c = D.mu_c * r, mu = mu_pe + mu_c;
    const float att = fmaf(C.pr.x, r3, fmaf(C.pr.y, r, C.pr.z * mu));
    const float absorb = -expm1f(-C.pr.w * mu) * sm_fdiv(mu_pe, mu);
    return phi_frac * ratio * p_win * expf(-att) * absorb;
}

}  // namespace smb
