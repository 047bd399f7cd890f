// Geometry: the Params tables parsed, validated and laid out for the device.
//
// Host and device share these plain structs.  Every derived float below is
// computed on the host with the same IEEE single-precision operations, in the
// same order, as the reference kernels compute it per thread, so the device
// sees bit-identical values (PESysMatGen.cu:452-471, :510-512, :526-538,
// :559-573, :647-654).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <vector_types.h>

namespace smb {

constexpr int kMaxPlates = 9;          // plate records (l+1)*10 must stay below the hole table at 100

// Crystal record, structure of arrays on the device (index = crystal id).
struct DevCrystals {
    const float4* pos;     // cx, cy + FOV, cz, mu_total
    const float4* size;    // width X, thickness Y, height Z, sqrt(w*w + h*h + t*t)
    const float4* rot;     // cos(-rot), sin(-rot), cos(rot), sin(rot)
    const float4* phys;    // mu_pe, mu_compton, energy resolution, rotation
    const float4* lo;      // world AABB min (x, y, z), 0
    const float4* hi;      // world AABB max (x, y, z), 0
};

// Hole record (index = global hole id, plates in order).
struct DevHoles {
    const float4* a;       // x, y1 + FOV, y2 + FOV, z
    const float4* b;       // R, mu_total, bounding half-extent crit, (y1 + y2) / 2
    const int* plate;      // plate index of the hole
};

struct PlateBox {
    float x1, y1, z1, x2, y2, z2;
    float thickness;       // Y extent, for T / cos(theta)
    float mu_total;
    float mu_pe, mu_compton;
    int hole_begin, hole_end;   // global hole id range of this plate
};

struct DevGeometry {
    int n_crystals;
    int n_holes;
    int n_plates;
    float fov;                     // Image[11]
    DevCrystals c;
    DevHoles h;
    PlateBox plate[kMaxPlates];
};

// Host copy of the parsed tables.
struct HostGeometry {
    int n_crystals = 0, n_holes = 0, n_plates = 0;
    int nx = 0, ny = 0, nz = 0, n_rotations = 1;
    float voxel[3] = {0, 0, 0};
    float shift[3] = {0, 0, 0};
    float angle_per_rotation = 0.0f;
    float fov = 0.0f;
    std::vector<float> image;      // 100 floats as given
    std::vector<float> physics;    // 100 floats as given (zeros when absent)
    std::vector<float> collimator; // as given (length n_collimator)
    std::vector<float> detector;   // as given
    std::vector<float> c_pos, c_size, c_rot, c_phys, c_lo, c_hi;   // 4 floats per crystal
    std::vector<float> h_a, h_b;                                  // 4 floats per hole
    std::vector<int> h_plate;
    PlateBox plate[kMaxPlates];
};

// Parses and validates; returns SM_OK or an SM_ERR_* code with sm_last_error set.
int parse_geometry(const float* col, size_t n_col, const float* det, size_t n_det, const float* img,
                   size_t n_img, const float* phy, size_t n_phy, HostGeometry* out);

// Device copy: one allocation holding every array.
struct DeviceGeometryBuffer {
    void* blob = nullptr;
    size_t bytes = 0;
    DevGeometry view{};
};

int upload_geometry(const HostGeometry& g, DeviceGeometryBuffer* out);
void free_geometry(DeviceGeometryBuffer* buf);

}  // namespace smb
