/* TEST INFRASTRUCTURE ONLY -- part of the CPU oracle, never linked into the product.
 *
 * The reference's three ray primitives restated, templated on the number type
 * (oracle_common.h): chord_through (PESysMatGen.cu:19-151, duplicated in
 * scatter.cu as length_box_ray), chord_to_end (PESysMatGen.cu:153-307,
 * length_box_ray_inside) and chord_hole (PESysMatGen.cu:309-373,
 * length_cylinder_ray).  Shared by the photoelectric and scatter oracles.
 */
#ifndef SYSMAT_ORACLE_PRIMS_H
#define SYSMAT_ORACLE_PRIMS_H

#include "oracle_common.h"

namespace oracle {

/* ---------------------------------------------------------------------------
 * Chord of the segment in -> out through an axis-aligned box, counted only when
 * the segment enters and leaves the box strictly inside (eps = 1e-3 mm)
 * (PESysMatGen.cu:19-151).  Degenerate directions (a coordinate changing by
 * less than eps) use the 1-D or 2-D slab test of the remaining axes.
 * ------------------------------------------------------------------------- */
template <class N>
inline N slab_pair(N a_in, N a_out, N lo, N hi, N t_total, N* t_lo, N* t_hi) {
    N inv = t_total / (a_out - a_in);
    if (inv < N(0.0f)) { *t_lo = (hi - a_in) * inv; *t_hi = (lo - a_in) * inv; }
    else               { *t_hi = (hi - a_in) * inv; *t_lo = (lo - a_in) * inv; }
    return inv;
}

/* 2-D slab intersection on axes (a, b); returns false when the slabs miss. */
template <class N>
inline bool slab_2d(N a_in, N a_out, N a_lo, N a_hi, N b_in, N b_out, N b_lo, N b_hi, N t_total,
                    N* tmin, N* tmax) {
    N ta0, ta1, tb0, tb1;
    slab_pair(a_in, a_out, a_lo, a_hi, t_total, &ta0, &ta1);
    slab_pair(b_in, b_out, b_lo, b_hi, t_total, &tb0, &tb1);
    if ((ta0 > tb1) || (tb0 > ta1)) return false;
    if (tb0 > ta0) ta0 = tb0;
    if (tb1 < ta1) ta1 = tb1;
    *tmin = ta0; *tmax = ta1;
    return true;
}

template <class N>
inline N chord_through(N xi, N yi, N zi, N xo, N yo, N zo,
                       N x1, N y1, N z1, N x2, N y2, N z2) {
    const N eps = N(0.001f);
    const N zero = N(0.0f);
    bool cx = m_fabs(xo - xi) < eps, cy = m_fabs(yo - yi) < eps, cz = m_fabs(zo - zi) < eps;
    if (cx & cy & cz) return zero;
    if (cx & cy) {                                       /* along z */
        if ((xi >= x1 & xi <= x2) & (yi >= y1 & yi <= y2))
            if ((zi <= z1 & zo >= z2) || (zo <= z1 & zi >= z2)) return m_fabs(z2 - z1);
        return zero;
    }
    if (cz & cy) {                                       /* along x */
        if ((zi >= z1 & zi <= z2) & (yi >= y1 & yi <= y2))
            if ((xi <= x1 & xo >= x2) || (xo <= x1 & xi >= x2)) return m_fabs(x2 - x1);
        return zero;
    }
    if (cx & cz) {                                       /* along y */
        if ((xi >= x1 & xi <= x2) & (zi >= z1 & zi <= z2))
            if ((yi <= y1 & yo >= y2) || (yo <= y1 & yi >= y2)) return m_fabs(y2 - y1);
        return zero;
    }
    N tmin, tmax, t_total;
    if (cx) {                                            /* in a plane x = const: (y, z) */
        if (xi >= x2 || xi <= x1) return zero;
        t_total = m_sqrt((yo - yi) * (yo - yi) + (zo - zi) * (zo - zi));
        if (!slab_2d(yi, yo, y1, y2, zi, zo, z1, z2, t_total, &tmin, &tmax)) return zero;
    } else if (cy) {                                     /* plane y = const: (x, z) */
        if (yi >= y2 || yi <= y1) return zero;
        t_total = m_sqrt((xo - xi) * (xo - xi) + (zo - zi) * (zo - zi));
        if (!slab_2d(xi, xo, x1, x2, zi, zo, z1, z2, t_total, &tmin, &tmax)) return zero;
    } else if (cz) {                                     /* plane z = const: (x, y) */
        if (zi >= z2 || zi <= z1) return zero;
        t_total = m_sqrt((xo - xi) * (xo - xi) + (yo - yi) * (yo - yi));
        if (!slab_2d(xi, xo, x1, x2, yi, yo, y1, y2, t_total, &tmin, &tmax)) return zero;
    } else {                                             /* general: x, then y, then z */
        t_total = m_sqrt((xo - xi) * (xo - xi) + (yo - yi) * (yo - yi) + (zo - zi) * (zo - zi));
        if (!slab_2d(xi, xo, x1, x2, yi, yo, y1, y2, t_total, &tmin, &tmax)) return zero;
        N tz0, tz1;
        slab_pair(zi, zo, z1, z2, t_total, &tz0, &tz1);
        if ((tmin > tz1) || (tz0 > tmax)) return zero;
        if (tz0 > tmin) tmin = tz0;
        if (tz1 < tmax) tmax = tz1;
    }
    if ((tmax - tmin) < eps) return zero;
    if (tmin >= t_total || tmax >= t_total) return zero;
    if (tmin <= eps || tmax <= eps) return zero;
    return tmax - tmin;
}

/* ---------------------------------------------------------------------------
 * Chord from where the segment in -> out enters a box to where it ends inside
 * it (PESysMatGen.cu:153-307).  Zero when the segment barely changes depth
 * (|dy| < 1e-3).  Used for the path inside the detecting crystal.
 * ------------------------------------------------------------------------- */
template <class N>
inline N chord_to_end(N xi, N yi, N zi, N xo, N yo, N zo,
                      N x1, N y1, N z1, N x2, N y2, N z2) {
    const N eps = N(0.001f);
    const N zero = N(0.0f);
    if (m_fabs(yo - yi) < N(0.001f)) return zero;
    bool cx = m_fabs(xo - xi) < eps, cy = m_fabs(yo - yi) < eps, cz = m_fabs(zo - zi) < eps;
    if (cx & cy & cz) return zero;
    if (cx & cy) {
        if ((xi >= x1 & xi <= x2) & (yi >= y1 & yi <= y2)) {
            if (zi < zo) return zo - z1;
            else if (zi > zo) return z2 - zo;
        }
        return zero;
    }
    if (cz & cy) {
        if ((zi >= z1 & zi <= z2) & (yi >= y1 & yi <= y2)) {
            if (xi < xo) return xo - x1;
            else if (xi > xo) return x2 - xo;
        }
        return zero;
    }
    if (cx & cz) {
        if ((xi >= x1 & xi <= x2) & (zi >= z1 & zi <= z2)) {
            if (yi < yo) return yo - y1;
            else if (yi > yo) return y2 - yo;
        }
        return zero;
    }
    N tmin, tmax, t_total;
    if (cx) {
        if (xi >= x2 || xi <= x1) return zero;
        t_total = m_sqrt((yo - yi) * (yo - yi) + (zo - zi) * (zo - zi));
        if (!slab_2d(yi, yo, y1, y2, zi, zo, z1, z2, t_total, &tmin, &tmax)) return zero;
    } else if (cy) {
        if (yi >= y2 || yi <= y1) return zero;
        t_total = m_sqrt((xo - xi) * (xo - xi) + (zo - zi) * (zo - zi));
        if (!slab_2d(xi, xo, x1, x2, zi, zo, z1, z2, t_total, &tmin, &tmax)) return zero;
    } else if (cz) {
        if (zi >= z2 || zi <= z1) return zero;
        t_total = m_sqrt((xo - xi) * (xo - xi) + (yo - yi) * (yo - yi));
        if (!slab_2d(xi, xo, x1, x2, yi, yo, y1, y2, t_total, &tmin, &tmax)) return zero;
    } else {
        t_total = m_sqrt((xo - xi) * (xo - xi) + (yo - yi) * (yo - yi) + (zo - zi) * (zo - zi));
        if (!slab_2d(xi, xo, x1, x2, yi, yo, y1, y2, t_total, &tmin, &tmax)) return zero;
        N tz0, tz1;
        slab_pair(zi, zo, z1, z2, t_total, &tz0, &tz1);
        if ((tmin > tz1) || (tz0 > tmax)) return zero;
        if (tz0 > tmin) tmin = tz0;
        if (tz1 < tmax) tmax = tz1;
    }
    if ((tmax - tmin) < eps) return zero;
    if (tmin >= t_total) return zero;
    if (tmax <= eps) return zero;
    if ((tmax >= t_total) && (tmin > eps)) return t_total - tmin;
    if ((tmin <= eps) && (tmax <= t_total)) return tmax;
    if ((tmin <= eps) && (tmax >= t_total)) return t_total;
    return tmax - tmin;
}

/* ---------------------------------------------------------------------------
 * Chord through a hole: a cylinder of radius R with its axis parallel to y at
 * (xc, zc), between the planes y1 and y2 (PESysMatGen.cu:309-373).  The end
 * caps are tested first; otherwise the wall quadratic, with near-tangent rays
 * (discriminant <= 1e-5) counted as a miss.
 * ------------------------------------------------------------------------- */
template <class N>
inline N chord_hole(N xi, N yi, N zi, N xo, N yo, N zo, N xc, N y1, N y2, N zc, N R) {
    const N zero = N(0.0f);
    if (m_fabs(y1 - y2) < N(0.001f)) return zero;
    N t_total = m_sqrt((xo - xi) * (xo - xi) + (yo - yi) * (yo - yi) + (zo - zi) * (zo - zi));
    N kx = (xo - xi) / t_total, ky = (yo - yi) / t_total, kz = (zo - zi) / t_total;
    N x_a = xi + kx / ky * (y1 - yi), x_b = xi + kx / ky * (y2 - yi);
    N z_a = zi + kz / ky * (y1 - yi), z_b = zi + kz / ky * (y2 - yi);
    N t_a = (y1 - yi) / ky, t_b = (y2 - yi) / ky;
    bool in_a = (x_a - xc) * (x_a - xc) + (z_a - zc) * (z_a - zc) <= R * R;
    bool in_b = (x_b - xc) * (x_b - xc) + (z_b - zc) * (z_b - zc) <= R * R;
    const N tiny = N(0.0001f);
    if (in_a && in_b) {
        if (t_a <= tiny || t_b <= tiny) return zero;
        if (t_a >= t_total || t_b >= t_total) return zero;
        return m_fabs(t_b - t_a);
    }
    N px = xi - xc, pz = zi - zc;
    N disc = (kx * kx + kz * kz) * R * R - (kx * pz - kz * px) * (kx * pz - kz * px);
    if (disc <= N(0.00001f)) return zero;
    N t1 = (-(kx * px + kz * pz) - m_sqrt(disc)) / (kx * kx + kz * kz);
    N t2 = (-(kx * px + kz * pz) + m_sqrt(disc)) / (kx * kx + kz * kz);
    if (!in_a && !in_b) {
        if ((t1 >= t_a) && (t2 <= t_b)) {
            if (t2 <= tiny || t1 <= tiny) return zero;
            if (t2 >= t_total || t1 >= t_total) return zero;
            return t2 - t1;
        }
        return zero;
    }
    if (in_a) {                                          /* enters through cap a, leaves by the wall */
        if (t2 <= tiny || t_a <= tiny) return zero;
        if (t2 >= t_total || t_a >= t_total) return zero;
        return t2 - t_a;
    }
    if (t_b <= tiny || t1 <= tiny) return zero;          /* enters by the wall, leaves through cap b */
    if (t_b >= t_total || t1 >= t_total) return zero;
    return t_b - t1;
}

}  /* namespace oracle */

#endif
