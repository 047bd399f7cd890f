/* TEST INFRASTRUCTURE ONLY -- CPU oracle for the photoelectric (PE) sysmat.
 * Never linked into the product; used by tests/, the smoke check and
 * bench.py's CPU baseline as the checker.
 *
 * A restatement of the reference PE kernel photodetectorCudaMe
 * (PEGen_RayTracing_CircularHole/PESysMatGen.cu:375-764) and its three ray
 * primitives (:19-373), templated on the number type (see oracle_common.h):
 * float reproduces the reference's results bit for bit (pinned in tests
 * against the reference's own code built on the host), double is the FP64
 * oracle, Dual takes the reference's single-precision decisions with FP64
 * magnitudes.  Voxel sub-sampling (kx, ky, kz) is the reference evaluated on
 * the k-times finer voxel grid and averaged over each coarse voxel; crystal
 * sub-cells are a runtime grid (the reference hard-codes 8 x 16 x 8).
 *
 * Besides values, the oracle can record, for every ray, the plates whose box
 * the ray fails to traverse (the 1e5 penalty), and the holes and crystals that
 * the ray hits with a non-zero chord among the reference's candidates.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

#include "oracle_common.h"
#include "oracle_prims.h"

namespace oracle {


/* ---------------------------------------------------------------------------
 * Per-ray hit record.
 * ------------------------------------------------------------------------- */
struct HitLog {
    std::vector<int32_t> words;   /* per ray: ray, plate-miss mask, nh, holes..., nc, crystals... */
};

static inline int ifloor(float v) { return (int)std::floor(v); }

/* One cell (crystal `row`, voxel `col0` of the slab described by img[2],
 * img[30], img[31]) of the reference PE kernel, on the grid in `img`. */
template <class N>
static N pe_cell(const float* col, const float* det, const float* img, int row, int col0,
                 int dvx, int dvy, int dvz, HitLog* log, int ray_base) {
    const int n_plates = (int)std::floor(col[0] + 0.000001f);
    const int n_det = (int)std::floor(det[0] + 0.000001f);
    const N fov = tab<N>(img, 11);
    const int nx = ifloor(img[0]), ny = ifloor(img[1]), nz_full = ifloor(img[30]);
    const int z0 = (int)std::floor(img[31] + 0.001f);
    const N vx = tab<N>(img, 3), vy = tab<N>(img, 4), vz = tab<N>(img, 5);
    const N angle = tab<N>(img, 20) * tab<N>(img, 7);

    const int iz = z0 + col0 / (ny * nx);
    const int rem = col0 % (ny * nx);
    const int iy = rem / nx, ix = rem % nx;

    /* Voxel centre, FOV shift, rotation about z (PESysMatGen.cu:437-449). */
    N xI = N(((float)ix - nx / 2.0f + 0.5f)) * vx;
    N yI = N(((float)iy - ny / 2.0f + 0.5f)) * vy;
    N zI = N(((float)iz - nz_full / 2.0f + 0.5f)) * vz;
    xI = xI + tab<N>(img, 8); yI = yI + tab<N>(img, 9); zI = zI + tab<N>(img, 10);
    {
        N xr = xI * m_cos(angle) - yI * m_sin(angle);
        N yr = xI * m_sin(angle) + yI * m_cos(angle);
        xI = xr; yI = yr;
    }

    /* The detecting crystal and the voxel in its own frame (:451-471). */
    const long long b = 12LL * row;
    const N xc = tab<N>(det, b + 1), yc = tab<N>(det, b + 2) + fov, zc = tab<N>(det, b + 3);
    const N rot = tab<N>(det, b + 11);
    const N w = tab<N>(det, b + 4), h = tab<N>(det, b + 6), t = tab<N>(det, b + 5);
    const N xIs = (xI - xc) * m_cos(-rot) - (zI - zc) * m_sin(-rot);
    const N yIs = yI - yc;
    const N zIs = (xI - xc) * m_sin(-rot) + (zI - zc) * m_cos(-rot);
    const N half = N(2.0f);
    const N bx1 = -w / half, bx2 = w / half, by1 = -t / half, by2 = t / half, bz1 = -h / half, bz2 = h / half;
    const N mu_t = tab<N>(det, b + 7), mu_pe = tab<N>(det, b + 8);

    /* Candidate crystals and holes: bounding-sphere cone tests from the voxel (:480-590). */
    std::vector<int> cand_det;
    std::vector<std::vector<int>> cand_hole(n_plates > 0 ? n_plates : 0);
    std::vector<int> holes_in(n_plates > 0 ? n_plates : 0);
    for (int l = 0; l < n_plates; ++l) holes_in[l] = ifloor(col[(l + 1) * 10 + 0]);

    N result = N(0.0f);
    if (!(mu_t > N(0.01f))) return result;

    {
        N dist = m_sqrt((yc - yI) * (yc - yI) + (xc - xI) * (xc - xI) + (zc - zI) * (zc - zI));
        N crit_self = m_sqrt(w * w + h * h + t * t) / dist / half;
        N ux = (xc - xI) / dist, uy = (yc - yI) / dist, uz = (zc - zI) / dist;
        for (int k = 0; k < n_det; ++k) {
            if (k == row) continue;
            const long long c = 12LL * k;
            N wk = tab<N>(det, c + 4), hk = tab<N>(det, c + 6), tk = tab<N>(det, c + 5);
            N crit = m_sqrt(wk * wk + hk * hk + tk * tk);
            N xk = tab<N>(det, c + 1), yk = tab<N>(det, c + 2) + fov, zk = tab<N>(det, c + 3);
            N dk = m_sqrt((xI - xk) * (xI - xk) + (yI - yk) * (yI - yk) + (zI - zk) * (zI - zk));
            crit = crit / dk / half;
            xk = (xk - xI) / dk; yk = (yk - yI) / dk; zk = (zk - zI) / dk;
            if (m_sqrt((zk - uz) * (zk - uz) + (yk - uy) * (yk - uy) + (xk - ux) * (xk - ux)) <= crit + crit_self)
                cand_det.push_back(k);
        }
        int id = 0;
        for (int l = 0; l < n_plates; ++l) {
            for (int j = 0; j < holes_in[l]; ++j, ++id) {
                const long long o = 100LL + 9LL * id;
                N hx = tab<N>(col, o), hy1 = tab<N>(col, o + 1) + fov, hy2 = tab<N>(col, o + 2) + fov;
                N hz = tab<N>(col, o + 3), R = tab<N>(col, o + 4);
                N hy = (hy1 + hy2) / half;
                N crit = m_sqrt(R * R * N(4.0f) + (hy1 - hy2) * (hy1 - hy2)) / half;
                N dh = m_sqrt((xI - hx) * (xI - hx) + (yI - hy) * (yI - hy) + (zI - hz) * (zI - hz));
                crit = crit / dh;
                hx = (hx - xI) / dh; hy = (hy - yI) / dh; hz = (hz - zI) / dh;
                if (m_sqrt((hz - uz) * (hz - uz) + (hy - uy) * (hy - uy) + (hx - ux) * (hx - ux)) <= crit + crit_self)
                    cand_hole[l].push_back(id);
            }
        }
    }

    const N cos_r = m_cos(rot), sin_r = m_sin(rot);
    const N fdx = from_float<N>((float)dvx), fdy = from_float<N>((float)dvy), fdz = from_float<N>((float)dvz);
    std::vector<int32_t> hole_hits, det_hits;
    int ray = ray_base;
    for (int sz = 0; sz < dvz; ++sz)
    for (int sx = 0; sx < dvx; ++sx)
    for (int sy = 0; sy < dvy; ++sy, ++ray) {
        /* Sub-cell centre in the crystal frame, then in the world (:606-616). */
        N xDs = -w / half + from_float<N>((float)sx + 0.5f) / fdx * w;
        N zDs = -h / half + from_float<N>((float)sz + 0.5f) / fdz * h;
        N yDs = -t / half + from_float<N>((float)sy + 0.5f) / fdy * t;
        N xD = xc + (xDs * cos_r - zDs * sin_r);
        N zD = zc + (xDs * sin_r + zDs * cos_r);
        N yD = yc + yDs;

        /* Solid angle of the sub-cell: the largest projected face (:618-639). */
        N dsq = (yD - yI) * (yD - yI) + (xD - xI) * (xD - xI) + (zD - zI) * (zD - zI);
        N cosang = (yD - yI) / m_sqrt(dsq);
        N sa_x = solid_face(t * h / fdz / fdy, dsq, m_fabs((xD - xI) * cos_r - (zD - zI) * sin_r), m_sqrt(dsq));
        N sa_z = solid_face(w * t / fdx / fdy, dsq, m_fabs((xD - xI) * sin_r + (zD - zI) * cos_r), m_sqrt(dsq));
        N sa_y = solid_face(w * h / fdx / fdz, dsq, m_fabs(yD - yI), m_sqrt(dsq));
        N sa = ref_max(ref_max(sa_x, sa_y), sa_z);

        N att = N(0.0f);
        uint32_t plate_miss = 0;
        /* A ray that does not traverse a plate's box counts as blocked (:643-659). */
        for (int l = 0; l < n_plates; ++l) {
            const int o = (l + 1) * 10;
            N px1 = -tab<N>(col, o + 1) / half, px2 = tab<N>(col, o + 1) / half;
            N py1 = -tab<N>(col, o + 2) / half + fov + tab<N>(col, o + 4);
            N py2 = tab<N>(col, o + 2) / half + fov + tab<N>(col, o + 4);
            N pz1 = -tab<N>(col, o + 3) / half, pz2 = tab<N>(col, o + 3) / half;
            N len = chord_through(xI, yI, zI, xD, yD, zD, px1, py1, pz1, px2, py2, pz2);
            if (len < N(0.1f)) { att += N(100000.0f); plate_miss |= (1u << l); }
        }
        /* Plates: holes among the candidates, tungsten for the rest of T/cos (:661-685). */
        hole_hits.clear();
        for (int l = 0; l < n_plates; ++l) {
            const int o = (l + 1) * 10;
            N in_holes = N(0.0f);
            N through = tab<N>(col, o + 2) / cosang;
            N mu_plate = tab<N>(col, o + 5);
            for (int id : cand_hole[l]) {
                const long long q = 100LL + 9LL * id;
                N len = chord_hole(xI, yI, zI, xD, yD, zD, tab<N>(col, q), tab<N>(col, q + 1) + fov,
                                   tab<N>(col, q + 2) + fov, tab<N>(col, q + 3), tab<N>(col, q + 4));
                in_holes += len;
                att += tab<N>(col, q + 5) * len;
                if (len > N(0.0f)) hole_hits.push_back(id);
            }
            if ((through - in_holes) >= N(0.00001f)) att += mu_plate * (through - in_holes);
        }
        /* Other crystals among the candidates, each in its own frame (:687-725). */
        det_hits.clear();
        for (int k : cand_det) {
            const long long c = 12LL * k;
            N xa = tab<N>(det, c + 1), ya = tab<N>(det, c + 2) + fov, za = tab<N>(det, c + 3);
            N wa = tab<N>(det, c + 4), ha = tab<N>(det, c + 6), ta = tab<N>(det, c + 5);
            N mua = tab<N>(det, c + 7), ra = tab<N>(det, c + 11);
            N ca = m_cos(-ra), sa_ = m_sin(-ra);
            N xIa = (xI - xa) * ca - (zI - za) * sa_, yIa = yI - ya, zIa = (xI - xa) * sa_ + (zI - za) * ca;
            N xDa = (xD - xa) * ca - (zD - za) * sa_, yDa = yD - ya, zDa = (xD - xa) * sa_ + (zD - za) * ca;
            N hf = N(0.5f);
            N len = chord_through(xIa, yIa, zIa, xDa, yDa, zDa, -hf * wa, -hf * ta, -hf * ha, hf * wa, hf * ta, hf * ha);
            att += len * mua;
            if (len > N(0.0f)) det_hits.push_back(k);
        }
        /* Path inside the detecting crystal before the sub-cell (:727-746). */
        N ux1 = (from_float<N>((float)sx) / fdx - N(0.5f)) * w, ux2 = ((from_float<N>((float)sx) + N(1.0f)) / fdx - N(0.5f)) * w;
        N uy1 = (from_float<N>((float)sy) / fdy - N(0.5f)) * t, uy2 = ((from_float<N>((float)sy) + N(1.0f)) / fdy - N(0.5f)) * t;
        N uz1 = (from_float<N>((float)sz) / fdz - N(0.5f)) * h, uz2 = ((from_float<N>((float)sz) + N(1.0f)) / fdz - N(0.5f)) * h;
        N l1 = chord_to_end(xIs, yIs, zIs, xDs, yDs, zDs, bx1, by1, bz1, bx2, by2, bz2);
        N l2 = chord_to_end(xIs, yIs, zIs, xDs, yDs, zDs, ux1, uy1, uz1, ux2, uy2, uz2);
        att += (l1 - l2) * mu_t;
        N eff = N(1.0f);
        eff *= m_exp(-att);
        /* Absorption in the sub-cell along the extended ray (:749-759). */
        N ext = N(1000.0f);
        N xt = xDs + ext * (xDs - xIs) / m_sqrt(dsq);
        N yt = yDs + ext * (yDs - yIs) / m_sqrt(dsq);
        N zt = zDs + ext * (zDs - zIs) / m_sqrt(dsq);
        N labs = chord_through(xIs, yIs, zIs, xt, yt, zt, ux1, uy1, uz1, ux2, uy2, uz2);
        N absorb = (N(1.0f) - m_exp(-labs * mu_t)) * mu_pe / mu_t;
        result = result + eff * sa * absorb;

        if (log) {
            log->words.push_back(ray);
            log->words.push_back((int32_t)plate_miss);
            log->words.push_back((int32_t)hole_hits.size());
            log->words.insert(log->words.end(), hole_hits.begin(), hole_hits.end());
            log->words.push_back((int32_t)det_hits.size());
            log->words.insert(log->words.end(), det_hits.begin(), det_hits.end());
        }
    }
    return result;
}

/* The image table of the k-times finer voxel grid covering the whole volume. */
static void fine_image(const float* img, const int sv[3], float* out) {
    std::memcpy(out, img, 100 * sizeof(float));
    for (int a = 0; a < 3; ++a) {
        int n = ifloor(img[a] + 0.001f);
        out[a] = (float)(n * sv[a]);
        out[3 + a] = img[3 + a] / (float)sv[a];
    }
    out[30] = out[2];
    out[31] = 0.0f;
}

/* Mean over the sub-points of coarse voxel `vox` of fine-grid cells. */
template <class N>
static double pe_entry(const float* col, const float* det, const float* fimg, const int sv[3], const int grid[3],
                       int row, long long vox, const int sc[3], HitLog* log) {
    const int nx = grid[0], ny = grid[1];
    const int ix = (int)(vox % nx), iy = (int)((vox / nx) % ny), iz = (int)(vox / ((long long)nx * ny));
    const int fnx = nx * sv[0], fny = ny * sv[1];
    const int rays_per_point = sc[0] * sc[1] * sc[2];
    double sum = 0.0;
    int s = 0;
    for (int sz = 0; sz < sv[2]; ++sz)
    for (int sy = 0; sy < sv[1]; ++sy)
    for (int sx = 0; sx < sv[0]; ++sx, ++s) {
        long long fvox = ((long long)(iz * sv[2] + sz) * fny + (iy * sv[1] + sy)) * fnx + (ix * sv[0] + sx);
        N v = pe_cell<N>(col, det, fimg, row, (int)fvox, sc[0], sc[1], sc[2], log, s * rays_per_point);
        sum += mag(v);
    }
    return sum / (double)(sv[0] * sv[1] * sv[2]);
}

}  /* namespace oracle */

using namespace oracle;

extern "C" {

/* mode: 0 = float (reference arithmetic), 1 = double, 2 = Dual (float decisions, double magnitudes). */
int oracle_pe_entries(const float* col, long long ncol, const float* det, long long ndet, const float* img,
                      const int* sv, const int* sc, int rotation, const long long* rows, const long long* voxels,
                      long long n, int mode, double* out, int nthreads) {
    (void)ncol; (void)ndet;
    float fimg[100];
    fine_image(img, sv, fimg);
    fimg[20] = (float)rotation;
    int grid[3] = {ifloor(img[0] + 0.001f), ifloor(img[1] + 0.001f), ifloor(img[2] + 0.001f)};
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
    for (long long i = 0; i < n; ++i) {
        int row = (int)rows[i];
        if (mode == 0) out[i] = pe_entry<float>(col, det, fimg, sv, grid, row, voxels[i], sc, nullptr);
        else if (mode == 1) out[i] = pe_entry<double>(col, det, fimg, sv, grid, row, voxels[i], sc, nullptr);
        else out[i] = pe_entry<Dual>(col, det, fimg, sv, grid, row, voxels[i], sc, nullptr);
    }
    return 0;
}

/* Hit lists of every ray of entry (row, voxel), single-precision decisions.
 * Writes the word stream described in HitLog; returns its length, or -needed
 * when `cap` is too small. */
long long oracle_pe_hits(const float* col, const float* det, const float* img, const int* sv, const int* sc,
                         int rotation, long long row, long long voxel, int32_t* out, long long cap) {
    float fimg[100];
    fine_image(img, sv, fimg);
    fimg[20] = (float)rotation;
    int grid[3] = {ifloor(img[0] + 0.001f), ifloor(img[1] + 0.001f), ifloor(img[2] + 0.001f)};
    HitLog log;
    pe_entry<float>(col, det, fimg, sv, grid, (int)row, voxel, sc, &log);
    long long n = (long long)log.words.size();
    if (n > cap) return -n;
    std::memcpy(out, log.words.data(), (size_t)n * sizeof(int32_t));
    return n;
}

/* Primitive batches for the primitive-level pins: float arithmetic (the
 * reference's), and dual (single-precision decisions, double magnitudes). */
int oracle_box_ray_batch_dual(const float* a, long long n, double* out) {
    for (long long i = 0; i < n; ++i, a += 12)
        out[i] = chord_through<Dual>(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11]).d;
    return 0;
}
int oracle_box_inside_batch_dual(const float* a, long long n, double* out) {
    for (long long i = 0; i < n; ++i, a += 12)
        out[i] = chord_to_end<Dual>(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11]).d;
    return 0;
}
int oracle_cylinder_batch_dual(const float* a, long long n, double* out) {
    for (long long i = 0; i < n; ++i, a += 11)
        out[i] = chord_hole<Dual>(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10]).d;
    return 0;
}
int oracle_box_ray_batch(const float* a, long long n, double* out) {
    for (long long i = 0; i < n; ++i, a += 12)
        out[i] = chord_through<float>(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11]);
    return 0;
}
int oracle_box_inside_batch(const float* a, long long n, double* out) {
    for (long long i = 0; i < n; ++i, a += 12)
        out[i] = chord_to_end<float>(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11]);
    return 0;
}
int oracle_cylinder_batch(const float* a, long long n, double* out) {
    for (long long i = 0; i < n; ++i, a += 11)
        out[i] = chord_hole<float>(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10]);
    return 0;
}

}  /* extern "C" */
