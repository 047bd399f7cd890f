/* TEST INFRASTRUCTURE ONLY -- CPU oracle for the primary-Compton scatter sysmat.
 * Never linked into the product; used by tests/ and bench.py's CPU baseline as
 * the checker.
 *
 * A restatement of the reference's scatter path
 * (ScatterGen_RayTracing_CircularHole/scatter.cu), templated on the number
 * type (oracle_common.h): float repeats the reference's single-precision
 * arithmetic, including the places where C++ promotes an expression to double
 * (M_PI, sqrt(2.0)); double is the FP64 judge.
 *
 *   bitmap_crystal_word      geometryRelationShip_Crystal2Crystal  (scatter.cu:1440-1540)
 *   bitmap_collimator_word   geometryRelationShip_Collimator2Crystal (:1939-2009)
 *   compton_integral         computeComptonIntegral + diffComptonSection (:961-995)
 *   scatter_term             the body of crystalScatterSysMatCuda (:1077-1437) and
 *                            collimatorScatterSysMatCuda (:1544-1936) for one
 *                            (detector, voxel, scatter point)
 *
 * The one generalisation: a scatter crystal may be split into kx x ky x kz
 * scatter points (sub-cell centres of the crystal, in its own frame, with the
 * formula the reference uses for detector sub-units, scatter.cu:1199-1201),
 * each carrying 1/(kx ky kz) of the crystal's Compton probability and using
 * the bitmap of the crystal pair.  With 1 x 1 x 1 the point is the crystal
 * centre and the result is the reference's.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

#include "oracle_common.h"
#include "oracle_prims.h"

namespace oracle {
namespace {

/* float: the reference's float arithmetic promoted to double for one
 * operation and rounded back (x * sqrt(2.0), 2.0f * M_PI). */
inline float dpromote_mul(float a, double c) { return (float)((double)a * c); }
inline double dpromote_mul(double a, double c) { return a * c; }

inline int trunc_int(float v) { return (int)v; }
inline int trunc_int(double v) { return (int)v; }

template <class N> inline N from_int(int i) { return N((float)i); }
template <> inline double from_int<double>(int i) { return (double)i; }

template <class N> inline N lit_delta();   /* the 0.01 the kernels pass as DeltaTheta */
template <> inline float lit_delta<float>() { return 0.01f; }
template <> inline double lit_delta<double>() { return 0.01; }

template <class N>
N dist3(N x1, N y1, N z1, N x2, N y2, N z2) {   /* calculateDist, scatter.cu:1032-1035 */
    return m_sqrt((x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2) + (z1 - z2) * (z1 - z2));
}

/* diffComptonSection (scatter.cu:961-978): Klein-Nishina, unnormalised. */
template <class N>
N klein_nishina(N theta, N E0) {
    N c = m_cos(theta);
    N alpha = E0 / N(511.0f);
    N f1 = alpha * (N(1.0f) - c);
    N f2 = N(1.0f) + c * c;
    return f2 / (N(1.0f) + f1) / (N(1.0f) + f1) * (N(1.0f) + f1 * f1 / f2 / (N(1.0f) + f1));
}

/* computeComptonIntegral (scatter.cu:981-995): rectangle rule from theta_low
 * with numSteps + 1 samples, numSteps = (int)((hi - lo) / delta). */
template <class N>
N compton_integral(N E0, N lo, N hi, N delta) {
    N total = N(0.0f);
    int steps = trunc_int((hi - lo) / delta);
    for (int i = 0; i <= steps; ++i) {
        N theta = lo + from_int<N>(i) * delta;
        total += klein_nishina(theta, E0) * m_sin(theta) * delta;
    }
    return total;
}

/* calculateConeAngle (scatter.cu:998-1017): angle at A between S->A and A->D. */
template <class N>
N cone_angle(N xs, N ys, N zs, N xa, N ya, N za, N xd, N yd, N zd) {
    N v0 = xa - xs, v1 = ya - ys, v2 = za - zs;
    N w0 = xd - xa, w1 = yd - ya, w2 = zd - za;
    N dot = w0 * v0 + w1 * v1 + w2 * v2;
    N m1 = m_sqrt(v0 * v0 + v1 * v1 + v2 * v2);
    N m2 = m_sqrt(w0 * w0 + w1 * w1 + w2 * w2);
    N c = dot / (m1 * m2);
    if (c > N(1.0f)) c = N(1.0f);
    if (c < N(-1.0f)) c = N(-1.0f);
    return m_acos(c);
}

/* calculateScatterEnergy (scatter.cu:1020-1027). */
template <class N>
N scatter_energy(N theta, N E0) {
    N c = m_cos(theta);
    return E0 / (N(1.0f) + (E0 / N(511.0f)) * (N(1.0f) - c));
}

/* calculategaussianIntegral (scatter.cu:1029-1031). */
template <class N>
N window_probability(N E, N res, N lower, N upper) {
    N sigma = res / N(2.35482f) * E;
    N s2 = dpromote_mul(sigma, std::sqrt(2.0));
    N z1 = (lower - E) / s2;
    N z2 = (upper - E) / s2;
    return N(0.5f) * (m_erf(z2) - m_erf(z1));
}

struct Tables {
    const float* col;
    const float* det;
    const float* img;
    const float* phys;
    int n_crystals, nx, ny, nz;
};

/* Bits (i, j, k) of the crystal bitmap (scatter.cu:1440-1540): does crystal k's
 * bounding sphere lie in the cone from i towards j (seen from i or from j)?
 * Always in single precision, as the reference computes the files. */
bool bitmap_crystal_bit(const float* det, int i, int j, int k) {
    auto R = [&](int c) {
        float w = det[12 * c + 4], h = det[12 * c + 6], t = det[12 * c + 5];
        return std::sqrt(w * w + h * h + t * t) / 2.0f;
    };
    float xi = det[12 * i + 1], yi = det[12 * i + 2], zi = det[12 * i + 3];
    float xj = det[12 * j + 1], yj = det[12 * j + 2], zj = det[12 * j + 3];
    float xk = det[12 * k + 1], yk = det[12 * k + 2], zk = det[12 * k + 3];
    float Ri = R(i), Rj = R(j), Rk = R(k);
    float Lij = dist3(xi, yi, zi, xj, yj, zj);
    float crit_ij = Ri / Lij, crit_ji = Rj / Lij;
    float ex_ij = (xi - xj) / Lij, ey_ij = (yi - yj) / Lij, ez_ij = (zi - zj) / Lij;
    float ex_ji = (xj - xi) / Lij, ey_ji = (yj - yi) / Lij, ez_ji = (zj - zi) / Lij;
    float Lik = dist3(xk, yk, zk, xi, yi, zi);
    float crit_ki = Rk / Lik;
    float Ljk = dist3(xk, yk, zk, xj, yj, zj);
    float crit_kj = Rk / Ljk;
    float ex_ki = (xk - xi) / Lik, ey_ki = (yk - yi) / Lik, ez_ki = (zk - zi) / Lik;
    float ex_kj = (xk - xj) / Ljk, ey_kj = (yk - yj) / Ljk, ez_kj = (zk - zj) / Ljk;
    float di = dist3(ex_ki, ey_ki, ez_ki, ex_ji, ey_ji, ez_ji);
    if (di <= crit_ki + crit_ji) return true;
    float dj = dist3(ex_kj, ey_kj, ez_kj, ex_ij, ey_ij, ez_ij);
    return dj <= crit_kj + crit_ij;
}

/* Bit (hole i, crystal j, crystal k) of the collimator bitmap (scatter.cu:1939-2009). */
bool bitmap_collimator_bit(const float* det, const float* col, int i, int j, int k) {
    float xc = col[9 * i + 100];
    float yc = (col[9 * i + 101] + col[9 * i + 102]) / 2.0f;
    float zc = col[9 * i + 103];
    float wj = det[12 * j + 4], hj = det[12 * j + 6], tj = det[12 * j + 5];
    float Rj = std::sqrt(wj * wj + hj * hj + tj * tj) / 2.0f;
    float xj = det[12 * j + 1], yj = det[12 * j + 2], zj = det[12 * j + 3];
    float Lij = dist3(xc, yc, zc, xj, yj, zj);
    float crit_ji = Rj / Lij;
    float ex_ji = (xj - xc) / Lij, ey_ji = (yj - yc) / Lij, ez_ji = (zj - zc) / Lij;
    float wk = det[12 * k + 4], hk = det[12 * k + 6], tk = det[12 * k + 5];
    float Rk = std::sqrt(wk * wk + hk * hk + tk * tk) / 2.0f;
    float xk = det[12 * k + 1], yk = det[12 * k + 2], zk = det[12 * k + 3];
    float Lik = dist3(xk, yk, zk, xc, yc, zc);
    float crit_ki = Rk / Lik;
    float ex_ki = (xk - xc) / Lik, ey_ki = (yk - yc) / Lik, ez_ki = (zk - zc) / Lik;
    float di = dist3(ex_ki, ey_ki, ez_ki, ex_ji, ey_ji, ez_ji);
    return di <= crit_ki + crit_ji;
}

inline bool bit_of(const uint32_t* words, long long bit) { return (words[bit >> 5] >> (bit & 31)) & 1u; }

/* One (detector d, voxel, scatter point) term of the reference's scatter
 * kernels, added to *acc exactly as the kernel's atomicAdd does (the product
 * is formed in double, scatter.cu:1427 / :1924, then rounded to N).
 * kind 0: crystal scatter, scatter crystal s (its sub-point (px, py, pz) of
 * (kx, ky, kz)); kind 1: collimator scatter, layer-0 hole s. */
template <class N>
void scatter_term(const Tables& T, const uint32_t* bitmap, int kind, int d, int vox, int s, int px, int py, int pz,
                  int kx, int ky, int kz, float pe_value, N norm, N* acc) {
    const float* det = T.det;
    const float* img = T.img;
    const float* phys = T.phys;
    const int N_c = T.n_crystals;
    const N FOV = tab<N>(img, 11);
    const N angle = tab<N>(img, 20) * tab<N>(img, 7);
    const int nx = T.nx, ny = T.ny, nz = T.nz;
    int iz = vox / (ny * nx);
    int rem = vox % (ny * nx);
    int iy = rem / nx, ix = rem % nx;

    int use_compton = (int)std::floor(phys[0] + 0.5f);
    int same_window = (int)std::floor(phys[4] + 0.5f);
    N E0 = tab<N>(phys, 7);
    N res = tab<N>(det, d * 12 + 10);
    N lower, upper;
    if (same_window > 0) { lower = tab<N>(phys, 5); upper = tab<N>(phys, 6); }
    else {
        lower = (N(1.0f) - res / N(2.0f)) * E0;
        upper = (N(1.0f) + res / N(2.0f)) * E0;
    }
    N mu_t = tab<N>(det, d * 12 + 7), mu_pe = tab<N>(det, d * 12 + 8), mu_c = tab<N>(det, d * 12 + 9);

    N xI = (from_int<N>(ix) - from_int<N>(nx) / N(2.0f) + N(0.5f)) * tab<N>(img, 3);
    N yI = (from_int<N>(iy) - from_int<N>(ny) / N(2.0f) + N(0.5f)) * tab<N>(img, 4);
    N zI = (from_int<N>(iz) - from_int<N>(nz) / N(2.0f) + N(0.5f)) * tab<N>(img, 5);
    xI = xI + tab<N>(img, 8);
    yI = yI + tab<N>(img, 9);
    zI = zI + tab<N>(img, 10);
    N xr = xI * m_cos(angle) - yI * m_sin(angle);
    N yr = xI * m_sin(angle) + yI * m_cos(angle);
    xI = xr;
    yI = yr;

    N xD0 = tab<N>(det, 12 * d + 1), yD0 = tab<N>(det, 12 * d + 2) + FOV, zD0 = tab<N>(det, 12 * d + 3);
    N w = tab<N>(det, 12 * d + 4), h = tab<N>(det, 12 * d + 6), t = tab<N>(det, 12 * d + 5);
    N rotD = tab<N>(det, 12 * d + 11);
    N xI_s = (xI - xD0) * m_cos(-rotD) - (zI - zD0) * m_sin(-rotD);
    N yI_s = yI - yD0;
    N zI_s = (xI - xD0) * m_sin(-rotD) + (zI - zD0) * m_cos(-rotD);

    /* scatter point and its probability */
    N xS, yS, zS, prob;
    if (kind == 0) {
        N pe = N(pe_value);
        prob = pe * mu_c / mu_pe;
        N xs0 = tab<N>(det, s * 12 + 1), ys0 = tab<N>(det, s * 12 + 2) + FOV, zs0 = tab<N>(det, s * 12 + 3);
        if (kx * ky * kz == 1) {
            xS = xs0; yS = ys0; zS = zs0;
        } else {
            N ws = tab<N>(det, 12 * s + 4), hs = tab<N>(det, 12 * s + 6), ts = tab<N>(det, 12 * s + 5);
            N rs = tab<N>(det, 12 * s + 11);
            N xl = -ws / N(2.0f) + from_float<N>((float)px + 0.5f) / from_float<N>((float)kx) * ws;
            N zl = -hs / N(2.0f) + from_float<N>((float)pz + 0.5f) / from_float<N>((float)kz) * hs;
            N yl = -ts / N(2.0f) + from_float<N>((float)py + 0.5f) / from_float<N>((float)ky) * ts;
            xS = xs0 + (xl * m_cos(rs) - zl * m_sin(rs));
            zS = zs0 + (xl * m_sin(rs) + zl * m_cos(rs));
            yS = ys0 + yl;
            prob = prob / from_float<N>((float)(kx * ky * kz));
        }
    } else {
        const float* col = T.col;
        xS = tab<N>(col, s * 9 + 100);
        yS = (tab<N>(col, s * 9 + 101) + tab<N>(col, s * 9 + 102)) / N(2.0f) + FOV;
        zS = tab<N>(col, s * 9 + 103);
        N vr = N(0.1f);
        N L_ih = dist3(xI, yI, zI, xS, yS, zS);
        /* (r r M_PI + (y2 - y1) r) / (4 M_PI L L) * |yS - yI| / L: double from M_PI on,
         * rounded once into `solid_angle` (scatter.cu:1711-1712) */
        N thick = tab<N>(col, s * 9 + 102) - tab<N>(col, s * 9 + 101);
        N sa = N(((double)(vr * vr) * M_PI + (double)(thick * vr)) / (4.0 * M_PI * (double)L_ih * (double)L_ih) *
                 (double)m_fabs(yS - yI) / (double)L_ih);
        prob = sa / tab<N>(col, 15) * tab<N>(col, 17);
    }

    if (use_compton != 1 || !(mu_t > N(0.01f))) return;

    /* detector unit = the whole crystal (the reference's divide = 1) */
    N xDs = -w / N(2.0f) + from_float<N>(0.0f + 0.5f) / from_float<N>(1.0f) * w;
    N zDs = -h / N(2.0f) + from_float<N>(0.0f + 0.5f) / from_float<N>(1.0f) * h;
    N yDs = -t / N(2.0f) + from_float<N>(0.0f + 0.5f) / from_float<N>(1.0f) * t;
    N xDr = xDs * m_cos(rotD) - zDs * m_sin(rotD);
    N zDr = xDs * m_sin(rotD) + zDs * m_cos(rotD);
    N xD = xD0 + xDr, zD = zD0 + zDr, yD = yD0 + yDs;

    N theta = cone_angle(xI, yI, zI, xS, yS, zS, xD, yD, zD);
    N E = scatter_energy(theta, E0);
    N res_E = res * m_sqrt(E / E0);
    if (((E * (N(1.0f) + N(2.0f) * res_E / N(2.35482f))) <= lower) ||
        (E * (N(1.0f) - N(2.0f) * res_E / N(2.35482f)) >= upper))
        return;
    N p_win = window_probability(E, res_E, lower, upper);
    N L = dist3(xS, yS, zS, xD, yD, zD);
    N R_unit = m_sqrt(w * w / N(1.0f) / N(1.0f) + h * h / N(1.0f) / N(1.0f) + t * t / N(1.0f) / N(1.0f)) / N(2.0f);
    N range_phi;
    if (L * m_sin(theta) * N(2.0f) <= R_unit) range_phi = N(2.0 * M_PI);   /* 2.0f * M_PI, rounded to N */
    else {
        N q = R_unit / N(2.0f) / L / m_sin(theta);
        range_phi = N(4.0f) * m_asin(q <= N(1.0f) ? q : N(1.0f));
    }
    N xS_s = (xS - xD0) * m_cos(-rotD) - (zS - zD0) * m_sin(-rotD);
    N yS_s = yS - yD0;
    N zS_s = (xS - xD0) * m_sin(-rotD) + (zS - zD0) * m_cos(-rotD);
    N x1 = (from_float<N>(0.0f) / from_float<N>(1.0f) - N(0.5f)) * w;
    N x2 = ((from_float<N>(0.0f) + N(1.0f)) / from_float<N>(1.0f) - N(0.5f)) * w;
    N y1 = (from_float<N>(0.0f) / from_float<N>(1.0f) - N(0.5f)) * t;
    N y2 = ((from_float<N>(0.0f) + N(1.0f)) / from_float<N>(1.0f) - N(0.5f)) * t;
    N z1 = (from_float<N>(0.0f) / from_float<N>(1.0f) - N(0.5f)) * h;
    N z2 = ((from_float<N>(0.0f) + N(1.0f)) / from_float<N>(1.0f) - N(0.5f)) * h;
    N ext = N(1000.0f);
    N dIS = dist3(xS_s, yS_s, zS_s, xI_s, yI_s, zI_s);
    N xt = xS_s + ext * (xS_s - xI_s) / dIS;
    N yt = yS_s + ext * (yS_s - yI_s) / dIS;
    N zt = zS_s + ext * (zS_s - zI_s) / dIS;
    N length = chord_through(xI_s, yI_s, zI_s, xt, yt, zt, x1, y1, z1, x2, y2, z2);
    N th[8];
    th[0] = cone_angle(xI_s, yI_s, zI_s, xS_s, yS_s, zS_s, x1, y1, z1);
    th[1] = cone_angle(xI_s, yI_s, zI_s, xS_s, yS_s, zS_s, x2, y1, z1);
    th[2] = cone_angle(xI_s, yI_s, zI_s, xS_s, yS_s, zS_s, x1, y2, z1);
    th[3] = cone_angle(xI_s, yI_s, zI_s, xS_s, yS_s, zS_s, x1, y1, z2);
    th[4] = cone_angle(xI_s, yI_s, zI_s, xS_s, yS_s, zS_s, x2, y2, z1);
    th[5] = cone_angle(xI_s, yI_s, zI_s, xS_s, yS_s, zS_s, x2, y1, z2);
    th[6] = cone_angle(xI_s, yI_s, zI_s, xS_s, yS_s, zS_s, x1, y2, z2);
    th[7] = cone_angle(xI_s, yI_s, zI_s, xS_s, yS_s, zS_s, x2, y2, z2);
    N tmin = th[0], tmax = th[0];
    for (int i = 1; i < 8; ++i) {
        if (th[i] > tmax) tmax = th[i];
        if (th[i] < tmin) tmin = th[i];
    }
    if (length > N(0.001f)) tmin = N(0.0f);
    N ratio = compton_integral(E0, tmin, tmax, lit_delta<N>()) / norm;

    /* attenuation by the other crystals flagged in the bitmap, at energy E */
    N att = N(0.0f);
    for (int k = 0; k < N_c; ++k) {
        if (k == d || (kind == 0 && k == s)) continue;
        long long bit;
        if (kind == 0) {
            int a = s, b = d;
            if (a > b) { int tmp = a; a = b; b = tmp; }
            long long pair = (long long)a * N_c - ((long long)a * (a + 1)) / 2 + b;
            bit = pair * N_c + k;
        } else {
            bit = (long long)s * N_c * N_c + (long long)d * N_c + k;
        }
        if (!bit_of(bitmap, bit)) continue;
        N xk = tab<N>(det, 12 * k + 1), yk = tab<N>(det, 12 * k + 2) + FOV, zk = tab<N>(det, 12 * k + 3);
        N wk = tab<N>(det, 12 * k + 4), hk = tab<N>(det, 12 * k + 6), tk = tab<N>(det, 12 * k + 5);
        N rk = tab<N>(det, 12 * k + 11);
        N cpe = tab<N>(det, 12 * k + 8), cc = tab<N>(det, 12 * k + 9);
        cpe = cpe * E0 * E0 * E0 / E / E / E;
        cc = cc * E0 / E;
        N ct = cpe + cc;
        N xa = (xS - xk) * m_cos(-rk) - (zS - zk) * m_sin(-rk);
        N ya = yS - yk;
        N za = (xS - xk) * m_sin(-rk) + (zS - zk) * m_cos(-rk);
        N xb = (xD - xk) * m_cos(-rk) - (zD - zk) * m_sin(-rk);
        N yb = yD - yk;
        N zb = (xD - xk) * m_sin(-rk) + (zD - zk) * m_cos(-rk);
        N len = chord_through(xa, ya, za, xb, yb, zb, N(-0.5f) * wk, N(-0.5f) * tk, N(-0.5f) * hk, N(0.5f) * wk,
                              N(0.5f) * tk, N(0.5f) * hk);
        att = att + len * ct;
    }
    /* inside the detecting crystal, up to the unit */
    N xDs_s = xDs, yDs_s = yDs, zDs_s = zDs;
    N l1 = chord_to_end(xS_s, yS_s, zS_s, xDs_s, yDs_s, zDs_s, -w / N(2.0f), -t / N(2.0f), -h / N(2.0f), w / N(2.0f),
                        t / N(2.0f), h / N(2.0f));
    N l2 = chord_to_end(xS_s, yS_s, zS_s, xDs_s, yDs_s, zDs_s, x1, y1, z1, x2, y2, z2);
    N a_pe = mu_pe * E0 * E0 * E0 / E / E / E;
    N a_c = mu_c * E0 / E;
    N a_t = a_pe + a_c;
    att = att + (l1 - l2) * a_t;
    xt = xDs_s + ext * (xDs_s - xS_s) / L;
    yt = yDs_s + ext * (yDs_s - yS_s) / L;
    zt = zDs_s + ext * (zDs_s - zS_s) / L;
    N labs = chord_through(xS_s, yS_s, zS_s, xt, yt, zt, x1, y1, z1, x2, y2, z2);

    /* prob * Range_Phi / 2.0f / M_PI * ... : double from the division by M_PI on */
    N head = prob * range_phi / N(2.0f);
    double v = (double)head / M_PI * (double)ratio * (double)p_win * (double)m_exp(-att) *
               (double)(N(1.0f) - m_exp(-labs * a_t)) * (double)a_pe / (double)a_t;
    *acc = *acc + N(v);
}

}  // namespace

/* bits of the crystal bitmap that fall in word w */
static uint32_t crystal_word(const float* det, int N_c, long long w) {
    uint32_t word = 0;
    const long long total = ((long long)N_c * (N_c + 1) / 2) * N_c;
    for (int b = 0; b < 32; ++b) {
        long long bit = w * 32 + b;
        if (bit >= total) break;
        long long pair = bit / N_c;
        int k = (int)(bit % N_c);
        /* invert pair = i*N - i(i+1)/2 + j, i <= j */
        int i = 0;
        while ((long long)(i + 1) * N_c - ((long long)(i + 1) * (i + 2)) / 2 + (i + 1) <= pair) ++i;
        int j = (int)(pair - ((long long)i * N_c - ((long long)i * (i + 1)) / 2));
        if (i >= j || k == i || k == j) continue;
        if (bitmap_crystal_bit(det, i, j, k)) word |= 1u << b;
    }
    return word;
}

}  /* namespace oracle */

using namespace oracle;

extern "C" {

int oracle_bitmap_crystal(const float* det, long long ndet, uint32_t* words, long long n_words) {
    (void)ndet;
    const int N_c = (int)std::floor(det[0] + 0.0001f);
#pragma omp parallel for schedule(dynamic, 256)
    for (long long w = 0; w < n_words; ++w) words[w] = crystal_word(det, N_c, w);
    return 0;
}

int oracle_bitmap_collimator(const float* det, long long ndet, const float* col, long long ncol, uint32_t* words,
                             long long n_words) {
    (void)ndet;
    (void)ncol;
    const int N_c = (int)std::floor(det[0] + 0.0001f);
    const int H = (int)std::floor(col[10] + 0.01f);
    const long long total = (long long)H * N_c * N_c;
#pragma omp parallel for schedule(dynamic, 256)
    for (long long w = 0; w < n_words; ++w) {
        uint32_t word = 0;
        for (int b = 0; b < 32; ++b) {
            long long bit = w * 32 + b;
            if (bit >= total) break;
            int i = (int)(bit / ((long long)N_c * N_c));
            int j = (int)((bit / N_c) % N_c);
            int k = (int)(bit % N_c);
            if (bitmap_collimator_bit(det, col, i, j, k)) word |= 1u << b;
        }
        words[w] = word;
    }
    return 0;
}

/* kind 0: crystal scatter (pe = [N][V] float32, sp = scatter points per
 * crystal), kind 1: collimator scatter.  img[20] is the rotation index.
 * mode 0: float (the reference's arithmetic), 1: double. */
int oracle_scatter_entries(int kind, const float* col, const float* det, const float* img, const float* phys,
                           const float* pe, const uint32_t* bitmap, const int* sp, const long long* rows,
                           const long long* vox, long long n, int mode, double* out, int nthreads) {
    Tables T;
    T.col = col;
    T.det = det;
    T.img = img;
    T.phys = phys;
    T.n_crystals = (int)std::floor(det[0] + 0.0001f);
    T.nx = (int)std::floor(img[0] + 0.001f);
    T.ny = (int)std::floor(img[1] + 0.001f);
    T.nz = (int)std::floor(img[2] + 0.001f);
    const long long V = (long long)T.nx * T.ny * T.nz;
    const int H = kind == 1 ? (int)std::floor(col[10] + 0.000001f) : 0;
    const int kx = sp[0], ky = sp[1], kz = sp[2];
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (long long e = 0; e < n; ++e) {
        const int d = (int)rows[e], v = (int)vox[e];
        if (mode == 0) {
            /* integration_Compton (scatter.cu:1166), once per cell */
            const float norm = compton_integral<float>(phys[7], 0.0f, (float)M_PI, 0.01f);
            float acc = 0.0f;
            if (kind == 0) {
                for (int s = 0; s < T.n_crystals; ++s) {
                    if (s == d) continue;
                    for (int pz = 0; pz < kz; ++pz)
                        for (int px = 0; px < kx; ++px)
                            for (int py = 0; py < ky; ++py)
                                scatter_term<float>(T, bitmap, 0, d, v, s, px, py, pz, kx, ky, kz, pe[s * V + v], norm, &acc);
                }
            } else {
                for (int h = 0; h < H; ++h) scatter_term<float>(T, bitmap, 1, d, v, h, 0, 0, 0, 1, 1, 1, 0.0f, norm, &acc);
            }
            out[e] = (double)acc;
        } else {
            const double norm = compton_integral<double>((double)phys[7], 0.0, M_PI, 0.01);
            double acc = 0.0;
            if (kind == 0) {
                for (int s = 0; s < T.n_crystals; ++s) {
                    if (s == d) continue;
                    for (int pz = 0; pz < kz; ++pz)
                        for (int px = 0; px < kx; ++px)
                            for (int py = 0; py < ky; ++py)
                                scatter_term<double>(T, bitmap, 0, d, v, s, px, py, pz, kx, ky, kz, pe[s * V + v], norm, &acc);
                }
            } else {
                for (int h = 0; h < H; ++h) scatter_term<double>(T, bitmap, 1, d, v, h, 0, 0, 0, 1, 1, 1, 0.0f, norm, &acc);
            }
            out[e] = acc;
        }
    }
    return 0;
}

/* args: n x 3 floats (E0, lo, hi) */
int oracle_compton_integral_batch(const float* args, long long n, int mode, double* out) {
    for (long long i = 0; i < n; ++i) {
        const float* a = args + 3 * i;
        if (mode == 0) out[i] = (double)compton_integral<float>(a[0], a[1], a[2], 0.01f);
        else out[i] = compton_integral<double>(a[0], a[1], a[2], 0.01);
    }
    return 0;
}

}  /* extern "C" */
