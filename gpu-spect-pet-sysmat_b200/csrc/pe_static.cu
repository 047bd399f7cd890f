// Photoelectric sysmat without any device allocation: sm_pe_compute_static.
//
// Some callers cannot call cudaMalloc: a host application that hands every
// byte of device memory to its own arena or pool and forbids other
// allocators, a plugin loaded into such a process, or code that must not
// take the implicit device-wide synchronisation cudaMalloc/cudaFree can
// cause.  For them this entry point keeps all of its device working memory
// (the derived geometry tables and the kernel's status word) in one
// file-scope __device__ array of fixed size, kStaticBytes below.  Every GPU
// that loads the library holds that array until the process exits.
//
// The same trace kernel as sm_pe_compute runs on the same derived geometry
// (every value derived with the same single-precision expressions as
// geometry.cpp), so the two entry points give the same sysmat.
#include <cmath>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "common.h"
#include "geometry.h"
#include "pe.h"

namespace smb {
namespace {

// Device working memory of sm_pe_compute_static: bytes [0, 256) hold the
// status word, the derived geometry follows.  4 MiB covers, for example,
// 40000 crystals with 2000 holes, or 30000 crystals with 20000 holes.
constexpr size_t kStaticBytes = size_t(4) << 20;
constexpr size_t kStatusBytes = 256;

__device__ __align__(256) unsigned char g_pe_static_scratch[kStaticBytes];

// Host image of the array: the geometry is derived here and copied over.
alignas(256) unsigned char g_stage[kStaticBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;                                    // one call at a time per process
unsigned char* g_scratch_addr[kMaxDevices] = {};   // device address of the array, per device

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

int count_of(float v) { return (int)std::floor(v + 0.000001f); }

// Byte offsets of the geometry arrays inside the scratch array, in the order
// crystal pos, size, rot, phys, lo, hi, hole a, hole b, hole plate.
struct StaticLayout {
    size_t off[9];
    size_t total;
};

StaticLayout layout_for(int n_crystals, int n_holes) {
    const size_t bytes[9] = {16 * (size_t)n_crystals, 16 * (size_t)n_crystals, 16 * (size_t)n_crystals,
                             16 * (size_t)n_crystals, 16 * (size_t)n_crystals, 16 * (size_t)n_crystals,
                             16 * (size_t)n_holes,    16 * (size_t)n_holes,    4 * (size_t)n_holes};
    StaticLayout L;
    size_t at = kStatusBytes;
    for (int i = 0; i < 9; ++i) {
        L.off[i] = at;
        at = align256(at + (bytes[i] ? bytes[i] : 16));
    }
    L.total = at;
    return L;
}

// Validates the tables and derives the geometry straight into g_stage (no
// heap use).  Fills the scalar fields and plates of *g; its arrays stay empty.
// Same checks and same single-precision expressions as parse_geometry
// (PESysMatGen.cu:452-471, :510-512, :526-538, :559-573, :647-654).
int derive_into_stage(const float* col, size_t n_col, const float* det, size_t n_det, const float* img, size_t n_img,
                      HostGeometry* out, StaticLayout* lay) {
    if (!col || !det || !img) return fail(SM_ERR_INVALID, "collimator, detector and image tables are required");
    if (n_col < 100) return fail(SM_ERR_INVALID, "collimator table has %zu floats, need at least 100", n_col);
    if (n_det < 1) return fail(SM_ERR_INVALID, "detector table is empty");
    if (n_img < 12) return fail(SM_ERR_INVALID, "image table has %zu floats, need at least 12", n_img);
    HostGeometry& g = *out;
    g.nx = (int)std::floor(img[0] + 0.001f);
    g.ny = (int)std::floor(img[1] + 0.001f);
    g.nz = (int)std::floor(img[2] + 0.001f);
    if (g.nx < 1 || g.ny < 1 || g.nz < 1)
        return fail(SM_ERR_INVALID, "image grid %d x %d x %d: every dimension must be >= 1 (Image[0..2])", g.nx, g.ny, g.nz);
    if ((int64_t)g.nx * g.ny * g.nz > (int64_t)1 << 31) return fail(SM_ERR_CAPACITY, "image grid has more than 2^31 voxels");
    for (int a = 0; a < 3; ++a) {
        g.voxel[a] = img[3 + a];
        g.shift[a] = img[8 + a];
        if (!(g.voxel[a] > 0.0f)) return fail(SM_ERR_INVALID, "voxel size Image[%d] = %g must be > 0", 3 + a, g.voxel[a]);
    }
    g.n_rotations = (int)std::floor(img[6] + 0.001f);
    if (g.n_rotations < 1) g.n_rotations = 1;
    g.angle_per_rotation = img[7];
    g.fov = img[11];

    g.n_plates = count_of(col[0]);
    if (g.n_plates < 0 || g.n_plates > kMaxPlates)
        return fail(SM_ERR_CAPACITY, "collimator has %d plates; supported 0..%d (Collimator[0])", g.n_plates, kMaxPlates);
    int hole = 0;
    for (int l = 0; l < g.n_plates; ++l) {
        const float* L = col + (l + 1) * 10;
        const int nh = (int)std::floor(L[0]);
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
    g.n_crystals = count_of(det[0]);
    if (g.n_crystals < 1) return fail(SM_ERR_INVALID, "detector has %d crystals (Detector[0])", g.n_crystals);
    if ((size_t)1 + (size_t)12 * g.n_crystals > n_det)
        return fail(SM_ERR_CAPACITY, "%d crystals need %zu detector floats, table has %zu", g.n_crystals,
                    (size_t)1 + (size_t)12 * g.n_crystals, n_det);
    if (g.n_crystals > (1 << 24)) return fail(SM_ERR_CAPACITY, "more than 2^24 crystals");

    *lay = layout_for(g.n_crystals, g.n_holes);
    if (lay->total > kStaticBytes)
        return fail(SM_ERR_CAPACITY,
                    "%d crystals and %d holes need %zu bytes of device working memory; sm_pe_compute_static holds at "
                    "most %zu (use sm_pe_compute, which allocates)",
                    g.n_crystals, g.n_holes, lay->total, kStaticBytes);
    std::memset(g_stage, 0, lay->total);

    float* h_a = reinterpret_cast<float*>(g_stage + lay->off[6]);
    float* h_b = reinterpret_cast<float*>(g_stage + lay->off[7]);
    int* h_plate = reinterpret_cast<int*>(g_stage + lay->off[8]);
    for (int l = 0; l < g.n_plates; ++l) {
        for (int id = g.plate[l].hole_begin; id < g.plate[l].hole_end; ++id) {
            const float* H = col + 100 + 9 * (size_t)id;
            const float x = H[0], y1 = H[1] + g.fov, y2 = H[2] + g.fov, z = H[3], R = H[4];
            if (!(R >= 0.0f)) return fail(SM_ERR_INVALID, "hole %d: radius must be >= 0", id);
            const float crit = std::sqrt(R * R * 4.0f + (y1 - y2) * (y1 - y2)) / 2.0f;
            const float yc = (y1 + y2) / 2.0f;
            float* a = h_a + 4 * (size_t)id;
            float* b = h_b + 4 * (size_t)id;
            a[0] = x; a[1] = y1; a[2] = y2; a[3] = z;
            b[0] = R; b[1] = H[5]; b[2] = crit; b[3] = yc;
            h_plate[id] = l;
        }
    }
    float* c_pos = reinterpret_cast<float*>(g_stage + lay->off[0]);
    float* c_size = reinterpret_cast<float*>(g_stage + lay->off[1]);
    float* c_rot = reinterpret_cast<float*>(g_stage + lay->off[2]);
    float* c_phys = reinterpret_cast<float*>(g_stage + lay->off[3]);
    float* c_lo = reinterpret_cast<float*>(g_stage + lay->off[4]);
    float* c_hi = reinterpret_cast<float*>(g_stage + lay->off[5]);
    for (int d = 0; d < g.n_crystals; ++d) {
        const float* D = det + 12 * (size_t)d;
        const float w = D[4], t = D[5], h = D[6], rot = D[11];
        if (!(w > 0.0f && t > 0.0f && h > 0.0f))
            return fail(SM_ERR_INVALID, "crystal %d: sizes must be > 0 (Detector[%zu..%zu])", d, 12 * (size_t)d + 4,
                        12 * (size_t)d + 6);
        const float cy = D[2] + g.fov;
        const float crit = std::sqrt(w * w + h * h + t * t);
        const float cm = std::cos(-rot), sm = std::sin(-rot), cp = std::cos(rot), sp = std::sin(rot);
        const float ex = std::fabs(cp) * (w / 2.0f) + std::fabs(sp) * (h / 2.0f);
        const float ez = std::fabs(sp) * (w / 2.0f) + std::fabs(cp) * (h / 2.0f);
        float* P = c_pos + 4 * (size_t)d;
        P[0] = D[1]; P[1] = cy; P[2] = D[3]; P[3] = D[7];
        float* S = c_size + 4 * (size_t)d;
        S[0] = w; S[1] = t; S[2] = h; S[3] = crit;
        float* Rr = c_rot + 4 * (size_t)d;
        Rr[0] = cm; Rr[1] = sm; Rr[2] = cp; Rr[3] = sp;
        float* Q = c_phys + 4 * (size_t)d;
        Q[0] = D[8]; Q[1] = D[9]; Q[2] = D[10]; Q[3] = rot;
        float* lo = c_lo + 4 * (size_t)d;
        float* hi = c_hi + 4 * (size_t)d;
        lo[0] = D[1] - ex; lo[1] = cy - t / 2.0f; lo[2] = D[3] - ez; lo[3] = 0.0f;
        hi[0] = D[1] + ex; hi[1] = cy + t / 2.0f; hi[2] = D[3] + ez; hi[3] = 0.0f;
    }
    return SM_OK;
}

int validate_static(const HostGeometry& g, const sm_pe_options* opt, int row0, int row1, int z0, int nz, int64_t ld) {
    for (int a = 0; a < 3; ++a) {
        if (opt->sv[a] < 1 || opt->sv[a] > 64) return fail(SM_ERR_INVALID, "sv[%d] = %d must be in 1..64", a, opt->sv[a]);
        if (opt->sc[a] < 1 || opt->sc[a] > kMaxSubcellsPerAxis)
            return fail(SM_ERR_INVALID, "sc[%d] = %d must be in 1..%d", a, opt->sc[a], kMaxSubcellsPerAxis);
        if (opt->tile_voxels[a] < 0) return fail(SM_ERR_INVALID, "tile_voxels[%d] must be >= 0", a);
    }
    if ((int64_t)opt->sv[0] * opt->sv[1] * opt->sv[2] * opt->sc[0] * opt->sc[1] * opt->sc[2] > (1 << 22))
        return fail(SM_ERR_CAPACITY, "more than 2^22 rays per entry");
    if (opt->group < 0 || opt->group > kMaxGroup)
        return fail(SM_ERR_INVALID, "group = %d must be 0 (auto) or 1..%d", opt->group, kMaxGroup);
    if ((int64_t)g.nx * opt->sv[0] > (1 << 24) || (int64_t)g.ny * opt->sv[1] > (1 << 24) ||
        (int64_t)g.nz * opt->sv[2] > (1 << 24))
        return fail(SM_ERR_CAPACITY, "fine voxel grid exceeds 2^24 per axis");
    if (row0 < 0 || row1 > g.n_crystals || row0 >= row1)
        return fail(SM_ERR_INVALID, "row range [%d, %d) outside [0, %d)", row0, row1, g.n_crystals);
    if (z0 < 0 || nz < 1 || z0 + nz > g.nz) return fail(SM_ERR_INVALID, "slab z [%d, %d) outside [0, %d)", z0, z0 + nz, g.nz);
    const int64_t slab = (int64_t)g.nx * g.ny * nz;
    if (ld < slab) return fail(SM_ERR_INVALID, "ld = %lld is smaller than the slab's %lld voxels", (long long)ld, (long long)slab);
    return SM_OK;
}

// Once per device, with that device current: the device address of the array.
// In host code g_pe_static_scratch names a host-side stand-in, never the
// device memory, so only this address may be handed to a kernel.  The address
// is kept for the life of the process: after cudaDeviceReset the module is
// loaded again and the array may move, so the entry point must not be used
// after a reset of a device it has already run on.
int scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return fail(SM_ERR_DEVICE, "device %d beyond %d devices", device, kMaxDevices);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        SM_CUDA(cudaGetSymbolAddress(&p, g_pe_static_scratch));
        g_scratch_addr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[device];
    return SM_OK;
}

}  // namespace
}  // namespace smb

using namespace smb;

extern "C" int sm_pe_compute_static(const float* collimator, size_t n_collimator, const float* detector,
                                    size_t n_detector, const float* image, size_t n_image, const sm_pe_options* opt,
                                    int rotation, int row0, int row1, int z0, int nz, float* dst, int64_t ld,
                                    void* stream_ptr) {
    if (!opt || !dst) return fail(SM_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lock(g_mu);
    int device = -1;
    SM_CUDA(cudaGetDevice(&device));
    int major = 0;
    SM_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    if (major < 10) return fail(SM_ERR_DEVICE, "device %d is not sm_100 class; this build targets sm_100a", device);
    if (opt->flags & SM_PE_AUTOTUNE)
        return fail(SM_ERR_INVALID, "sm_pe_compute_static does not autotune (timing candidates would allocate); "
                                    "pass tile_voxels, e.g. from an earlier sm_pe_autotune");
    if (opt->flags != 0) return fail(SM_ERR_INVALID, "unknown option flags 0x%x", opt->flags);
    cudaPointerAttributes attr;
    SM_CUDA(cudaPointerGetAttributes(&attr, dst));
    if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)
        return fail(SM_ERR_INVALID, "dst must be device memory of the current device");
    if (attr.type == cudaMemoryTypeDevice && attr.device != device)
        return fail(SM_ERR_INVALID, "dst is memory of device %d, the current device is %d", attr.device, device);

    unsigned char* base = nullptr;
    SM_TRY(scratch_address(device, &base));
    HostGeometry g = HostGeometry();   // value-initialised: unused plates are zero
    StaticLayout lay;
    SM_TRY(derive_into_stage(collimator, n_collimator, detector, n_detector, image, n_image, &g, &lay));
    SM_TRY(validate_static(g, opt, row0, row1, z0, nz, ld));

    cudaStream_t stream = (cudaStream_t)stream_ptr;
    PEParams P;
    pe_plan(g, opt->sv, opt->sc, opt->tile_voxels, opt->group, rotation, row0, row1, g.nz, z0, nz, &P);
    // The array keeps the previous call's contents: the status word must
    // start at zero, and the geometry region is overwritten in full.
    SM_CUDA(cudaMemsetAsync(base, 0, kStatusBytes, stream));
    SM_CUDA(cudaMemcpyAsync(base + kStatusBytes, g_stage + kStatusBytes, lay.total - kStatusBytes,
                            cudaMemcpyHostToDevice, stream));
    DevGeometry view{};
    view.n_crystals = g.n_crystals;
    view.n_holes = g.n_holes;
    view.n_plates = g.n_plates;
    view.fov = g.fov;
    view.c.pos = reinterpret_cast<const float4*>(base + lay.off[0]);
    view.c.size = reinterpret_cast<const float4*>(base + lay.off[1]);
    view.c.rot = reinterpret_cast<const float4*>(base + lay.off[2]);
    view.c.phys = reinterpret_cast<const float4*>(base + lay.off[3]);
    view.c.lo = reinterpret_cast<const float4*>(base + lay.off[4]);
    view.c.hi = reinterpret_cast<const float4*>(base + lay.off[5]);
    view.h.a = reinterpret_cast<const float4*>(base + lay.off[6]);
    view.h.b = reinterpret_cast<const float4*>(base + lay.off[7]);
    view.h.plate = reinterpret_cast<const int*>(base + lay.off[8]);
    for (int l = 0; l < kMaxPlates; ++l) view.plate[l] = g.plate[l];
    P.status = reinterpret_cast<int*>(base);
    P.counters = nullptr;
    P.dst = dst;
    P.ld = ld;
    SM_CUDA(pe_launch(P, view, false, P.n_tiles, stream));
    // The status word is read before returning, so a later call cannot
    // overwrite the array while this one's kernel still runs.
    int st = 0;
    SM_CUDA(cudaMemcpyAsync(&st, base, sizeof(int), cudaMemcpyDeviceToHost, stream));
    SM_CUDA(cudaStreamSynchronize(stream));
    if (st != 0) return fail(SM_ERR_CUDA, "device status 0x%x", st);
    return SM_OK;
}
