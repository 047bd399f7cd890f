// Device ray primitives of the photoelectric tracer.
//
// Every hit/miss decision here is taken in IEEE single precision with the same
// operations, in the same order, as the reference primitives
// (PEGen_RayTracing_CircularHole/PESysMatGen.cu:19-373).  The translation unit
// is compiled with -fmad=false -prec-div=true -prec-sqrt=true, so no multiply
// and add are fused behind our back: the lists of holes and crystals a ray
// hits are the reference's, bit for bit.  Where a value (not a decision) has
// a better-conditioned form, the better form is used and says so.
#pragma once

#include <cmath>

#include <cuda_runtime.h>

// Host and device: the kernels use these, and host-side checks of the
// kernels' arithmetic call the same code.
#ifndef SM_HD
#define SM_HD __host__ __device__ __forceinline__
#endif

namespace smb {

struct Vec3 {
    float x, y, z;
};

struct Box3 {
    float x1, y1, z1, x2, y2, z2;
};

// Entry/exit parameters of one slab for a segment parameterised by length
// t_total (PESysMatGen.cu:57-64 and every slab of :19-151).
SM_HD void slab_pair(float a_in, float a_out, float lo, float hi, float t_total, float& t_lo,
                                          float& t_hi) {
    float inv = t_total / (a_out - a_in);
    if (inv < 0.0f) {
        t_lo = (hi - a_in) * inv;
        t_hi = (lo - a_in) * inv;
    } else {
        t_hi = (hi - a_in) * inv;
        t_lo = (lo - a_in) * inv;
    }
}

// Intersection of two slabs; false when they are disjoint.
SM_HD bool slab_2d(float a_in, float a_out, float a_lo, float a_hi, float b_in, float b_out,
                                        float b_lo, float b_hi, float t_total, float& tmin, float& tmax) {
    float ta0, ta1, tb0, tb1;
    slab_pair(a_in, a_out, a_lo, a_hi, t_total, ta0, ta1);
    slab_pair(b_in, b_out, b_lo, b_hi, t_total, tb0, tb1);
    if ((ta0 > tb1) || (tb0 > ta1)) return false;
    tmin = (tb0 > ta0) ? tb0 : ta0;
    tmax = (tb1 < ta1) ? tb1 : ta1;
    return true;
}

// Slab entry/exit of the segment a -> b (after its degenerate cases).
// Returns 0 for "no overlap", 1 for an overlap [tmin, tmax] of a segment of
// length t_total; the axis-degenerate answers (a full box side) come back as
// code 2 with the length in tmax.
SM_HD int slab_segment(float xi, float yi, float zi, float xo, float yo, float zo, const Box3& b,
                                            bool inside_variant, float& tmin, float& tmax, float& t_total) {
    const float eps = 0.001f;
    bool cx = fabsf(xo - xi) < eps, cy = fabsf(yo - yi) < eps, cz = fabsf(zo - zi) < eps;
    if (cx & cy & cz) return 0;
    if (cx & cy) {  // along z
        if ((xi >= b.x1 & xi <= b.x2) & (yi >= b.y1 & yi <= b.y2)) {
            if (!inside_variant) {
                if ((zi <= b.z1 & zo >= b.z2) || (zo <= b.z1 & zi >= b.z2)) { tmax = fabsf(b.z2 - b.z1); return 2; }
            } else {
                if (zi < zo) { tmax = zo - b.z1; return 2; }
                if (zi > zo) { tmax = b.z2 - zo; return 2; }
            }
        }
        return 0;
    }
    if (cz & cy) {  // along x
        if ((zi >= b.z1 & zi <= b.z2) & (yi >= b.y1 & yi <= b.y2)) {
            if (!inside_variant) {
                if ((xi <= b.x1 & xo >= b.x2) || (xo <= b.x1 & xi >= b.x2)) { tmax = fabsf(b.x2 - b.x1); return 2; }
            } else {
                if (xi < xo) { tmax = xo - b.x1; return 2; }
                if (xi > xo) { tmax = b.x2 - xo; return 2; }
            }
        }
        return 0;
    }
    if (cx & cz) {  // along y
        if ((xi >= b.x1 & xi <= b.x2) & (zi >= b.z1 & zi <= b.z2)) {
            if (!inside_variant) {
                if ((yi <= b.y1 & yo >= b.y2) || (yo <= b.y1 & yi >= b.y2)) { tmax = fabsf(b.y2 - b.y1); return 2; }
            } else {
                if (yi < yo) { tmax = yo - b.y1; return 2; }
                if (yi > yo) { tmax = b.y2 - yo; return 2; }
            }
        }
        return 0;
    }
    if (cx) {  // plane x = const: slabs y, z
        if (xi >= b.x2 || xi <= b.x1) return 0;
        t_total = sqrtf((yo - yi) * (yo - yi) + (zo - zi) * (zo - zi));
        return slab_2d(yi, yo, b.y1, b.y2, zi, zo, b.z1, b.z2, t_total, tmin, tmax) ? 1 : 0;
    }
    if (cy) {  // plane y = const: slabs x, z
        if (yi >= b.y2 || yi <= b.y1) return 0;
        t_total = sqrtf((xo - xi) * (xo - xi) + (zo - zi) * (zo - zi));
        return slab_2d(xi, xo, b.x1, b.x2, zi, zo, b.z1, b.z2, t_total, tmin, tmax) ? 1 : 0;
    }
    if (cz) {  // plane z = const: slabs x, y
        if (zi >= b.z2 || zi <= b.z1) return 0;
        t_total = sqrtf((xo - xi) * (xo - xi) + (yo - yi) * (yo - yi));
        return slab_2d(xi, xo, b.x1, b.x2, yi, yo, b.y1, b.y2, t_total, tmin, tmax) ? 1 : 0;
    }
    t_total = sqrtf((xo - xi) * (xo - xi) + (yo - yi) * (yo - yi) + (zo - zi) * (zo - zi));
    if (!slab_2d(xi, xo, b.x1, b.x2, yi, yo, b.y1, b.y2, t_total, tmin, tmax)) return 0;
    float tz0, tz1;
    slab_pair(zi, zo, b.z1, b.z2, t_total, tz0, tz1);
    if ((tmin > tz1) || (tz0 > tmax)) return 0;
    if (tz0 > tmin) tmin = tz0;
    if (tz1 < tmax) tmax = tz1;
    return 1;
}

// Chord of segment a -> b through box, counted only if the segment enters and
// leaves strictly inside (PESysMatGen.cu:19-151).
SM_HD float chord_through(float xi, float yi, float zi, float xo, float yo, float zo,
                                               const Box3& b) {
    const float eps = 0.001f;
    float tmin = 0.0f, tmax = 0.0f, t_total = 0.0f;
    int code = slab_segment(xi, yi, zi, xo, yo, zo, b, false, tmin, tmax, t_total);
    if (code == 0) return 0.0f;
    if (code == 2) return tmax;
    if ((tmax - tmin) < eps) return 0.0f;
    if (tmin >= t_total || tmax >= t_total) return 0.0f;
    if (tmin <= eps || tmax <= eps) return 0.0f;
    return tmax - tmin;
}

// Chord from the box entry to the end of the segment inside the box
// (PESysMatGen.cu:153-307).
SM_HD float chord_to_end(float xi, float yi, float zi, float xo, float yo, float zo,
                                              const Box3& b) {
    const float eps = 0.001f;
    if (fabsf(yo - yi) < 0.001f) return 0.0f;
    float tmin = 0.0f, tmax = 0.0f, t_total = 0.0f;
    int code = slab_segment(xi, yi, zi, xo, yo, zo, b, true, tmin, tmax, t_total);
    if (code == 0) return 0.0f;
    if (code == 2) return tmax;
    if ((tmax - tmin) < eps) return 0.0f;
    if (tmin >= t_total) return 0.0f;
    if (tmax <= eps) return 0.0f;
    if ((tmax >= t_total) && (tmin > eps)) return t_total - tmin;
    if ((tmin <= eps) && (tmax <= t_total)) return tmax;
    if ((tmin <= eps) && (tmax >= t_total)) return t_total;
    return tmax - tmin;
}

// Chord through a hole: cylinder of radius R, axis parallel to y at (xc, zc),
// between the planes y1 < y2 (PESysMatGen.cu:309-373).  Decisions in single
// precision as the reference; for rays that enter or leave through the wall
// the value t2 - t1 comes from a double-precision discriminant when it is
// small relative to its terms (near-tangent rays), where the single-precision
// difference (kx^2+kz^2)R^2 - (kx z - kz x)^2 cancels.
SM_HD float chord_hole(float xi, float yi, float zi, float xo, float yo, float zo, float xc,
                                            float y1, float y2, float zc, float R) {
    if (fabsf(y1 - y2) < 0.001f) return 0.0f;
    float t_total = sqrtf((xo - xi) * (xo - xi) + (yo - yi) * (yo - yi) + (zo - zi) * (zo - zi));
    float kx = (xo - xi) / t_total, ky = (yo - yi) / t_total, kz = (zo - zi) / t_total;
    float x_a = xi + kx / ky * (y1 - yi), x_b = xi + kx / ky * (y2 - yi);
    float z_a = zi + kz / ky * (y1 - yi), z_b = zi + kz / ky * (y2 - yi);
    float t_a = (y1 - yi) / ky, t_b = (y2 - yi) / ky;
    bool in_a = (x_a - xc) * (x_a - xc) + (z_a - zc) * (z_a - zc) <= R * R;
    bool in_b = (x_b - xc) * (x_b - xc) + (z_b - zc) * (z_b - zc) <= R * R;
    const float tiny = 0.0001f;
    if (in_a && in_b) {
        if (t_a <= tiny || t_b <= tiny) return 0.0f;
        if (t_a >= t_total || t_b >= t_total) return 0.0f;
        return fabsf(t_b - t_a);
    }
    float px = xi - xc, pz = zi - zc;
    float kk = kx * kx + kz * kz;
    float cross = kx * pz - kz * px;
    float disc = kk * R * R - cross * cross;
    if (disc <= 0.00001f) return 0.0f;
    float sq = sqrtf(disc);
    float t1 = (-(kx * px + kz * pz) - sq) / kk;
    float t2 = (-(kx * px + kz * pz) + sq) / kk;
    if (!in_a && !in_b) {
        if (!((t1 >= t_a) && (t2 <= t_b))) return 0.0f;
        if (t2 <= tiny || t1 <= tiny) return 0.0f;
        if (t2 >= t_total || t1 >= t_total) return 0.0f;
    } else if (in_a) {  // enters through the y1 cap, leaves through the wall
        if (t2 <= tiny || t_a <= tiny) return 0.0f;
        if (t2 >= t_total || t_a >= t_total) return 0.0f;
    } else {            // enters through the wall, leaves through the y2 cap
        if (t_b <= tiny || t1 <= tiny) return 0.0f;
        if (t_b >= t_total || t1 >= t_total) return 0.0f;
    }
    // Value (the decision above is unchanged): near-tangent rays get the wall
    // roots from a double-precision discriminant.
    double r1 = t1, r2 = t2;
    if (disc < 0.01f * (kk * R * R)) {
        double kxd = kx, kzd = kz, pxd = px, pzd = pz, Rd = R;
        double kkd = kxd * kxd + kzd * kzd;
        double cr = kxd * pzd - kzd * pxd;
        double dd = kkd * Rd * Rd - cr * cr;
        double s = sqrt(dd > 0.0 ? dd : 0.0);
        double bd = kxd * pxd + kzd * pzd;
        r1 = (-bd - s) / kkd;
        r2 = (-bd + s) / kkd;
    }
    if (!in_a && !in_b) return (float)(r2 - r1);
    if (in_a) return (float)(r2 - (double)t_a);
    return (float)((double)t_b - r1);
}

// Conservative culling: can any segment from a point of box A to a point of
// box B meet box K?  K must already be inflated by the safety margin.  Uses
// the depth (y) ordering of the scanner: at depth y a segment a -> b sits at
// lateral position a + (b - a) * lambda, lambda = (y - a_y) / (b_y - a_y);
// lambda is monotone in y, a_y and b_y, so its range over K's depth band comes
// from box corners.  Returns true whenever the ordering assumption fails.
__device__ __forceinline__ bool window_hit(const Box3& A, const Box3& B, const Box3& K) {
    if (K.y1 > fmaxf(A.y2, B.y2) || K.y2 < fminf(A.y1, B.y1)) return false;   // K outside every segment's depth range
    if (!(A.y2 < K.y1) || !(A.y2 < B.y1)) return true;
    float yhi = fminf(K.y2, B.y2);
    float lmin = (K.y1 - A.y2) / (B.y2 - A.y2);
    float lmax = fminf(1.0f, (yhi - A.y1) / (B.y1 - A.y1));
    lmin = fmaxf(lmin, 0.0f);
    float xa = A.x1 + (B.x1 - A.x1) * lmin, xb = A.x1 + (B.x1 - A.x1) * lmax;
    float xc = A.x2 + (B.x2 - A.x2) * lmin, xd = A.x2 + (B.x2 - A.x2) * lmax;
    if (fminf(xa, xb) > K.x2 || fmaxf(xc, xd) < K.x1) return false;
    float za = A.z1 + (B.z1 - A.z1) * lmin, zb = A.z1 + (B.z1 - A.z1) * lmax;
    float zc = A.z2 + (B.z2 - A.z2) * lmin, zd = A.z2 + (B.z2 - A.z2) * lmax;
    if (fminf(za, zb) > K.z2 || fmaxf(zc, zd) < K.z1) return false;
    return true;
}

}  // namespace smb
