// Host tables for the scatter kernels (scatter.h): raw crystal and hole
// positions for the bitmaps, scatter points, and the Klein-Nishina table.
//
// Compiled with -ffp-contract=off: positions and radii must round as the
// reference's single-precision expressions do (scatter.cu:1466-1511, :1961-1994,
// :1211-1219, :1700-1702).
#include <algorithm>
#include <cmath>

#include "common.h"
#include "scatter.h"

namespace smb {

namespace {

// Truncated Taylor series in t (coefficients of t^0 .. t^4), double precision.
struct Series {
    double c[5];
};

Series s_const(double v) { return Series{{v, 0, 0, 0, 0}}; }

Series s_add(const Series& a, const Series& b) {
    Series r;
    for (int i = 0; i < 5; ++i) r.c[i] = a.c[i] + b.c[i];
    return r;
}

Series s_scale(const Series& a, double k) {
    Series r;
    for (int i = 0; i < 5; ++i) r.c[i] = a.c[i] * k;
    return r;
}

Series s_mul(const Series& a, const Series& b) {
    Series r{{0, 0, 0, 0, 0}};
    for (int i = 0; i < 5; ++i)
        for (int j = 0; i + j < 5; ++j) r.c[i + j] += a.c[i] * b.c[j];
    return r;
}

Series s_inv(const Series& a) {   // 1 / a, a.c[0] != 0
    Series r{{0, 0, 0, 0, 0}};
    r.c[0] = 1.0 / a.c[0];
    for (int n = 1; n < 5; ++n) {
        double acc = 0.0;
        for (int k = 1; k <= n; ++k) acc += a.c[k] * r.c[n - k];
        r.c[n] = -acc / a.c[0];
    }
    return r;
}

// g(theta0 + t) = KN(theta0 + t) sin(theta0 + t) as a series in t.
// KN = f2 / (1 + f1)^2 (1 + f1^2 / (f2 (1 + f1))), f1 = alpha (1 - cos), f2 = 1 + cos^2
// (diffComptonSection, scatter.cu:961-978).
Series g_series(double theta0, double alpha) {
    const double c0 = std::cos(theta0), s0 = std::sin(theta0);
    // cos(theta0 + t) = c0 cos t - s0 sin t, sin(theta0 + t) = s0 cos t + c0 sin t
    const Series cos_t{{1.0, 0.0, -0.5, 0.0, 1.0 / 24.0}};
    const Series sin_t{{0.0, 1.0, 0.0, -1.0 / 6.0, 0.0}};
    const Series cs = s_add(s_scale(cos_t, c0), s_scale(sin_t, -s0));
    const Series sn = s_add(s_scale(cos_t, s0), s_scale(sin_t, c0));
    const Series f1 = s_scale(s_add(s_const(1.0), s_scale(cs, -1.0)), alpha);
    const Series f2 = s_add(s_const(1.0), s_mul(cs, cs));
    const Series u = s_add(s_const(1.0), f1);
    const Series iu = s_inv(u);
    const Series kn = s_mul(s_mul(s_mul(f2, iu), iu), s_add(s_const(1.0), s_mul(s_mul(s_mul(f1, f1), s_inv(f2)), iu)));
    return s_mul(kn, sn);
}

double g_value(double theta, double alpha) {
    const double c = std::cos(theta);
    const double f1 = alpha * (1.0 - c), f2 = 1.0 + c * c;
    return f2 / (1.0 + f1) / (1.0 + f1) * (1.0 + f1 * f1 / f2 / (1.0 + f1)) * std::sin(theta);
}

// integral of g over [a, b], 8-point Gauss-Legendre (exact to rounding for
// the table's sub-degree intervals)
double g_integral(double a, double b, double alpha) {
    static const double x[4] = {0.1834346424956498, 0.5255324099163290, 0.7966664774136267, 0.9602898564975363};
    static const double w[4] = {0.3626837833783620, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763};
    const double m = 0.5 * (a + b), h = 0.5 * (b - a);
    double s = 0.0;
    for (int i = 0; i < 4; ++i) s += w[i] * (g_value(m - h * x[i], alpha) + g_value(m + h * x[i], alpha));
    return s * h;
}

void build_kn_table(float e0, std::vector<KnNode>* out, float* inv_norm) {
    const double alpha = (double)e0 / 511.0;
    out->assign(kKnNodes + 1, KnNode{});
    double F = 0.0, prev = 0.0;
    for (int j = 0; j <= kKnNodes; ++j) {
        const float th = (float)(M_PI * (double)j / (double)kKnNodes);
        const double thd = (double)th;
        if (j > 0) F += g_integral(prev, thd, alpha);
        prev = thd;
        const Series g = g_series(thd, alpha);
        KnNode& n = (*out)[j];
        n.theta = th;
        n.f_hi = (float)F;
        n.f_lo = (float)(F - (double)n.f_hi);
        n.c0 = (float)g.c[0];
        n.c1 = (float)g.c[1];
        n.c2 = (float)g.c[2];
        n.c3 = (float)g.c[3];
        n.c4 = (float)g.c[4];
    }
    // The reference normalises by its own rectangle sum over [0, pi]:
    // computeComptonIntegral(E0, 0, M_PI, 0.01), samples i * 0.01f for
    // i = 0 .. (int)(3.1415927f / 0.01f) (scatter.cu:1166).
    const float hi = (float)M_PI;
    const int steps = (int)((hi - 0.0f) / 0.01f);
    double norm = 0.0;
    for (int i = 0; i <= steps; ++i) {
        const float th = 0.0f + (float)i * 0.01f;
        norm += g_value((double)th, alpha) * (double)0.01f;
    }
    *inv_norm = (float)(1.0 / norm);
}

}  // namespace

int build_scatter_tables(const HostGeometry& g, const int sp[3], HostScatterTables* out) {
    HostScatterTables& T = *out;
    T = HostScatterTables();
    for (int a = 0; a < 3; ++a) {
        if (sp[a] < 1 || sp[a] > 16) return fail(SM_ERR_INVALID, "scatter points sp[%d] = %d must be in 1..16", a, sp[a]);
        T.sp[a] = sp[a];
    }
    T.n_points = sp[0] * sp[1] * sp[2];
    const int N = g.n_crystals;
    const float* det = g.detector.data();
    const float* col = g.collimator.data();
    const float fov = g.fov;
    T.crystal_raw.resize(4 * (size_t)N);
    T.crystal_src.resize(4 * (size_t)N * T.n_points);
    for (int d = 0; d < N; ++d) {
        const float* D = det + 12 * (size_t)d;
        const float w = D[4], t = D[5], h = D[6];
        float* r = &T.crystal_raw[4 * (size_t)d];
        r[0] = D[1];
        r[1] = D[2];
        r[2] = D[3];
        r[3] = std::sqrt(w * w + h * h + t * t) / 2.0f;      // R_detector (scatter.cu:1472)
        const float x0 = D[1], y0 = D[2] + fov, z0 = D[3], rot = D[11];
        int p = 0;
        // scatter points in the reference's sub-unit loop order: z, x, then depth y (scatter.cu:1191-1195)
        for (int pz = 0; pz < sp[2]; ++pz)
            for (int px = 0; px < sp[0]; ++px)
                for (int py = 0; py < sp[1]; ++py, ++p) {
                    float* q = &T.crystal_src[4 * ((size_t)d * T.n_points + p)];
                    if (T.n_points == 1) {
                        q[0] = x0;
                        q[1] = y0;
                        q[2] = z0;
                    } else {
                        const float xl = -w / 2.0f + ((float)px + 0.5f) / (float)sp[0] * w;
                        const float zl = -h / 2.0f + ((float)pz + 0.5f) / (float)sp[2] * h;
                        const float yl = -t / 2.0f + ((float)py + 0.5f) / (float)sp[1] * t;
                        q[0] = x0 + (xl * std::cos(rot) - zl * std::sin(rot));
                        q[2] = z0 + (xl * std::sin(rot) + zl * std::cos(rot));
                        q[1] = y0 + yl;
                    }
                    q[3] = 0.0f;
                }
    }
    // layer-0 holes: Collimator[10] of them (scatter.cu:2223)
    int h0 = g.n_plates > 0 ? (int)std::floor(col[10] + 0.01f) : 0;
    if (h0 > g.n_holes) h0 = g.n_holes;
    if (h0 < 0) h0 = 0;
    T.hole_raw.resize(4 * (size_t)(h0 > 0 ? h0 : 1), 0.0f);
    T.hole_src.resize(4 * (size_t)(h0 > 0 ? h0 : 1), 0.0f);
    for (int i = 0; i < h0; ++i) {
        const float* H = col + 100 + 9 * (size_t)i;
        float* r = &T.hole_raw[4 * (size_t)i];
        r[0] = H[0];
        r[1] = (H[1] + H[2]) / 2.0f;
        r[2] = H[3];
        r[3] = 0.0f;
        float* s = &T.hole_src[4 * (size_t)i];
        s[0] = H[0];
        s[1] = (H[1] + H[2]) / 2.0f + fov;
        s[2] = H[3];
        s[3] = H[2] - H[1];
    }
    build_kn_table(g.physics[7], &T.kn, &T.kn_inv_norm);
    return SM_OK;
}

// Depth layers (crystal centres within a quarter of the thinnest crystal of
// each other in y) first, then a Morton curve over x and z quantised by the
// narrowest crystal, so that 32 consecutive ranks form a compact 2-D patch of
// one layer.  Lanes of a warp are detectors; a patch makes the energy-window
// cull and the scattered photon's path coherent across the warp.
std::vector<int> spatial_order(const HostGeometry& g, int row0, int row1) {
    std::vector<int> ids(row1 - row0);
    for (int i = 0; i < row1 - row0; ++i) ids[i] = row0 + i;
    return spatial_order_of(g, ids);
}

std::vector<int> spatial_order_of(const HostGeometry& g, const std::vector<int>& ids_in) {
    std::vector<int> ids = ids_in;
    const int n = (int)ids.size();
    if (n <= 1) return ids;
    float tmin = 1e30f, wmin = 1e30f, xmin = 1e30f, zmin = 1e30f;
    for (int d : ids) {
        const float* sz = &g.c_size[4 * (size_t)d];
        const float* ps = &g.c_pos[4 * (size_t)d];
        tmin = std::min(tmin, sz[1]);
        wmin = std::min(wmin, std::min(sz[0], sz[2]));
        xmin = std::min(xmin, ps[0]);
        zmin = std::min(zmin, ps[2]);
    }
    std::vector<int> by_y = ids;
    std::stable_sort(by_y.begin(), by_y.end(), [&](int a, int b) { return g.c_pos[4 * (size_t)a + 1] < g.c_pos[4 * (size_t)b + 1]; });
    std::vector<long long> layer(g.n_crystals, 0);
    long long lay = 0;
    float prev = g.c_pos[4 * (size_t)by_y[0] + 1];
    for (int d : by_y) {
        const float y = g.c_pos[4 * (size_t)d + 1];
        if (y - prev > 0.25f * tmin) ++lay;
        prev = y;
        layer[d] = lay;
    }
    auto spread = [](uint32_t v) {   // 16 bits -> even bit positions
        uint64_t x = v & 0xffffu;
        x = (x | (x << 8)) & 0x00ff00ffu;
        x = (x | (x << 4)) & 0x0f0f0f0fu;
        x = (x | (x << 2)) & 0x33333333u;
        x = (x | (x << 1)) & 0x55555555u;
        return x;
    };
    std::vector<uint64_t> key(g.n_crystals, 0);
    for (int d : ids) {
        const float* ps = &g.c_pos[4 * (size_t)d];
        const uint32_t ix = (uint32_t)std::min(65535.0f, std::max(0.0f, std::floor((ps[0] - xmin) / wmin + 0.5f)));
        const uint32_t iz = (uint32_t)std::min(65535.0f, std::max(0.0f, std::floor((ps[2] - zmin) / wmin + 0.5f)));
        key[d] = ((uint64_t)layer[d] << 32) | spread(ix) | (spread(iz) << 1);
    }
    std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) { return key[a] < key[b]; });
    return ids;
}

}  // namespace smb
