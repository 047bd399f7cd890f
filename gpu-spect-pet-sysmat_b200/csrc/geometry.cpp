// Params table parsing, validation and device layout (see geometry.h).
//
// Compiled with -ffp-contract=off: the derived values must round exactly like
// the reference's per-thread single-precision expressions.
#include "geometry.h"

#include <cmath>
#include <cstring>

#include <cuda_runtime.h>

#include "common.h"

namespace smb {

static int count_of(float v) { return (int)std::floor(v + 0.000001f); }

int parse_geometry(const float* col, size_t n_col, const float* det, size_t n_det, const float* img,
                   size_t n_img, const float* phy, size_t n_phy, HostGeometry* out) {
    if (!col || !det || !img) return fail(SM_ERR_INVALID, "collimator, detector and image tables are required");
    if (n_col < 100) return fail(SM_ERR_INVALID, "collimator table has %zu floats, need at least 100", n_col);
    if (n_det < 1) return fail(SM_ERR_INVALID, "detector table is empty");
    if (n_img < 12) return fail(SM_ERR_INVALID, "image table has %zu floats, need at least 12", n_img);
    HostGeometry& g = *out;
    g = HostGeometry();

    g.image.assign(100, 0.0f);
    std::memcpy(g.image.data(), img, sizeof(float) * (n_img < 100 ? n_img : 100));
    g.physics.assign(100, 0.0f);
    if (phy) std::memcpy(g.physics.data(), phy, sizeof(float) * (n_phy < 100 ? n_phy : 100));
    g.collimator.assign(col, col + n_col);
    g.detector.assign(det, det + n_det);

    // ---- image (ReadMe.txt: Param_Image) ----
    g.nx = (int)std::floor(img[0] + 0.001f);
    g.ny = (int)std::floor(img[1] + 0.001f);
    g.nz = (int)std::floor(img[2] + 0.001f);
    if (g.nx < 1 || g.ny < 1 || g.nz < 1)
        return fail(SM_ERR_INVALID, "image grid %d x %d x %d: every dimension must be >= 1 (Image[0..2])", g.nx, g.ny, g.nz);
    if ((int64_t)g.nx * g.ny * g.nz > (int64_t)1 << 31)
        return fail(SM_ERR_CAPACITY, "image grid has more than 2^31 voxels");
    for (int a = 0; a < 3; ++a) {
        g.voxel[a] = img[3 + a];
        g.shift[a] = img[8 + a];
        if (!(g.voxel[a] > 0.0f)) return fail(SM_ERR_INVALID, "voxel size Image[%d] = %g must be > 0", 3 + a, g.voxel[a]);
    }
    g.n_rotations = (int)std::floor(img[6] + 0.001f);
    if (g.n_rotations < 1) g.n_rotations = 1;
    g.angle_per_rotation = img[7];
    g.fov = img[11];

    // ---- collimator (ReadMe.txt: Param_Collimator) ----
    g.n_plates = count_of(col[0]);
    if (g.n_plates < 0 || g.n_plates > kMaxPlates)
        return fail(SM_ERR_CAPACITY, "collimator has %d plates; supported 0..%d (Collimator[0])", g.n_plates, kMaxPlates);
    int hole = 0;
    for (int l = 0; l < g.n_plates; ++l) {
        const float* L = col + (l + 1) * 10;
        int nh = (int)std::floor(L[0]);
        if (nh < 0) return fail(SM_ERR_INVALID, "plate %d: negative hole count", l);
        PlateBox& p = g.plate[l];
        p.x1 = -L[1] / 2.0f;
        p.x2 = L[1] / 2.0f;
        p.y1 = -L[2] / 2.0f + g.fov + L[4];
        p.y2 = L[2] / 2.0f + g.fov + L[4];
        p.z1 = -L[3] / 2.0f;
        p.z2 = L[3] / 2.0f;
        p.thickness = L[2];
        p.mu_total = L[5];
        p.mu_pe = L[6];
        p.mu_compton = L[7];
        p.hole_begin = hole;
        hole += nh;
        p.hole_end = hole;
        if (!(L[2] > 0.0f)) return fail(SM_ERR_INVALID, "plate %d: thickness Collimator[%d] must be > 0", l, (l + 1) * 10 + 2);
    }
    g.n_holes = hole;
    if ((size_t)100 + (size_t)9 * g.n_holes > n_col)
        return fail(SM_ERR_CAPACITY, "%d holes need %zu collimator floats, table has %zu", g.n_holes,
                    (size_t)100 + (size_t)9 * g.n_holes, n_col);
    g.h_a.resize(4 * (size_t)g.n_holes);
    g.h_b.resize(4 * (size_t)g.n_holes);
    g.h_plate.resize(g.n_holes);
    for (int l = 0; l < g.n_plates; ++l) {
        for (int id = g.plate[l].hole_begin; id < g.plate[l].hole_end; ++id) {
            const float* H = col + 100 + 9 * (size_t)id;
            float x = H[0], y1 = H[1] + g.fov, y2 = H[2] + g.fov, z = H[3], R = H[4];
            if (!(R >= 0.0f)) return fail(SM_ERR_INVALID, "hole %d: radius must be >= 0", id);
            float crit = std::sqrt(R * R * 4.0f + (y1 - y2) * (y1 - y2)) / 2.0f;   // PESysMatGen.cu:566-567
            float yc = (y1 + y2) / 2.0f;                                           // :564
            float* a = &g.h_a[4 * (size_t)id];
            float* b = &g.h_b[4 * (size_t)id];
            a[0] = x; a[1] = y1; a[2] = y2; a[3] = z;
            b[0] = R; b[1] = H[5]; b[2] = crit; b[3] = yc;
            g.h_plate[id] = l;
        }
    }

    // ---- detector (ReadMe.txt: Param_Detector) ----
    g.n_crystals = count_of(det[0]);
    if (g.n_crystals < 1) return fail(SM_ERR_INVALID, "detector has %d crystals (Detector[0])", g.n_crystals);
    if ((size_t)1 + (size_t)12 * g.n_crystals > n_det)
        return fail(SM_ERR_CAPACITY, "%d crystals need %zu detector floats, table has %zu", g.n_crystals,
                    (size_t)1 + (size_t)12 * g.n_crystals, n_det);
    if (g.n_crystals > (1 << 24)) return fail(SM_ERR_CAPACITY, "more than 2^24 crystals");
    size_t n4 = 4 * (size_t)g.n_crystals;
    g.c_pos.resize(n4); g.c_size.resize(n4); g.c_rot.resize(n4); g.c_phys.resize(n4);
    g.c_lo.resize(n4); g.c_hi.resize(n4);
    for (int d = 0; d < g.n_crystals; ++d) {
        const float* D = det + 12 * (size_t)d;
        float w = D[4], t = D[5], h = D[6], rot = D[11];
        if (!(w > 0.0f && t > 0.0f && h > 0.0f))
            return fail(SM_ERR_INVALID, "crystal %d: sizes must be > 0 (Detector[%zu..%zu])", d, 12 * (size_t)d + 4, 12 * (size_t)d + 6);
        float cy = D[2] + g.fov;
        float crit = std::sqrt(w * w + h * h + t * t);                          // PESysMatGen.cu:510-512, :526-528
        float cm = std::cos(-rot), sm = std::sin(-rot), cp = std::cos(rot), sp = std::sin(rot);
        float ex = std::fabs(cp) * (w / 2.0f) + std::fabs(sp) * (h / 2.0f);
        float ez = std::fabs(sp) * (w / 2.0f) + std::fabs(cp) * (h / 2.0f);
        float* P = &g.c_pos[4 * (size_t)d];
        P[0] = D[1]; P[1] = cy; P[2] = D[3]; P[3] = D[7];
        float* S = &g.c_size[4 * (size_t)d];
        S[0] = w; S[1] = t; S[2] = h; S[3] = crit;
        float* R = &g.c_rot[4 * (size_t)d];
        R[0] = cm; R[1] = sm; R[2] = cp; R[3] = sp;
        float* Q = &g.c_phys[4 * (size_t)d];
        Q[0] = D[8]; Q[1] = D[9]; Q[2] = D[10]; Q[3] = rot;
        float* lo = &g.c_lo[4 * (size_t)d];
        float* hi = &g.c_hi[4 * (size_t)d];
        lo[0] = D[1] - ex; lo[1] = cy - t / 2.0f; lo[2] = D[3] - ez; lo[3] = 0.0f;
        hi[0] = D[1] + ex; hi[1] = cy + t / 2.0f; hi[2] = D[3] + ez; hi[3] = 0.0f;
    }
    return SM_OK;
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

int upload_geometry(const HostGeometry& g, DeviceGeometryBuffer* out) {
    struct Part { const void* src; size_t bytes; size_t off; };
    Part parts[] = {
        {g.c_pos.data(), g.c_pos.size() * 4, 0}, {g.c_size.data(), g.c_size.size() * 4, 0},
        {g.c_rot.data(), g.c_rot.size() * 4, 0}, {g.c_phys.data(), g.c_phys.size() * 4, 0},
        {g.c_lo.data(), g.c_lo.size() * 4, 0},   {g.c_hi.data(), g.c_hi.size() * 4, 0},
        {g.h_a.data(), g.h_a.size() * 4, 0},     {g.h_b.data(), g.h_b.size() * 4, 0},
        {g.h_plate.data(), g.h_plate.size() * 4, 0},
    };
    size_t total = 0;
    for (Part& p : parts) {
        p.off = total;
        total = align_up(total + (p.bytes ? p.bytes : 16), 256);
    }
    std::vector<unsigned char> host(total, 0);
    for (Part& p : parts)
        if (p.bytes) std::memcpy(host.data() + p.off, p.src, p.bytes);
    void* blob = nullptr;
    SM_CUDA(cudaMalloc(&blob, total));
    int rc = check_cuda(cudaMemcpy(blob, host.data(), total, cudaMemcpyHostToDevice), "upload geometry");
    if (rc != SM_OK) {
        cudaFree(blob);
        return rc;
    }
    unsigned char* base = (unsigned char*)blob;
    DevGeometry& v = out->view;
    v.n_crystals = g.n_crystals;
    v.n_holes = g.n_holes;
    v.n_plates = g.n_plates;
    v.fov = g.fov;
    v.c.pos = (const float4*)(base + parts[0].off);
    v.c.size = (const float4*)(base + parts[1].off);
    v.c.rot = (const float4*)(base + parts[2].off);
    v.c.phys = (const float4*)(base + parts[3].off);
    v.c.lo = (const float4*)(base + parts[4].off);
    v.c.hi = (const float4*)(base + parts[5].off);
    v.h.a = (const float4*)(base + parts[6].off);
    v.h.b = (const float4*)(base + parts[7].off);
    v.h.plate = (const int*)(base + parts[8].off);
    for (int l = 0; l < kMaxPlates; ++l) v.plate[l] = g.plate[l];
    out->blob = blob;
    out->bytes = total;
    return SM_OK;
}

void free_geometry(DeviceGeometryBuffer* buf) {
    if (buf->blob) cudaFree(buf->blob);
    buf->blob = nullptr;
    buf->bytes = 0;
}

}  // namespace smb
