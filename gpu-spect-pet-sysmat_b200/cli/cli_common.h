// Shared pieces of the command-line generators: the Params tables read from
// the working directory as the reference's CLIs read them
// (PEGen_CircularHole.cpp:39-62, ScatterGen_CircularHole.cpp:40-62), the
// geometry banner, and sysmat file names.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "sysmat_b200.h"

namespace cli {

// The four tables in buffers of at least the reference's sizes (80000 /
// 80000 / 100 / 100 floats, zero beyond the file), and the floats each file
// held.  Collimator and detector files longer than 80000 floats (more than
// 8877 holes or 6666 crystals) are read whole.
struct Tables {
    std::vector<float> collimator = std::vector<float>(80000, 0.0f);
    std::vector<float> detector = std::vector<float>(80000, 0.0f);
    std::vector<float> image = std::vector<float>(100, 0.0f);
    std::vector<float> physics = std::vector<float>(100, 0.0f);
    size_t n_collimator = 0, n_detector = 0, n_image = 0, n_physics = 0;
};

// Reads the table; a missing file is fatal (exit 1).  A file shorter than the
// buffer leaves zeros, as the reference's fread into a zeroed buffer does;
// whether the floats it held cover what its counts declare is checked by
// check_params.
inline size_t read_table(const char* name, std::vector<float>& out, bool whole) {
    FILE* f = std::fopen(name, "rb");
    if (!f) {
        std::fprintf(stderr, "ERROR: open %s\n", name);
        std::exit(1);
    }
    if (whole && std::fseek(f, 0, SEEK_END) == 0) {
        const long bytes = std::ftell(f);
        if (bytes > 0 && (size_t)bytes / sizeof(float) > out.size()) out.resize((size_t)bytes / sizeof(float), 0.0f);
        std::fseek(f, 0, SEEK_SET);
    }
    const size_t got = std::fread(out.data(), sizeof(float), out.size(), f);
    std::fclose(f);
    return got;
}

inline Tables read_params() {
    Tables t;
    t.n_collimator = read_table("Params_Collimator.dat", t.collimator, true);
    t.n_detector = read_table("Params_Detector.dat", t.detector, true);
    t.n_image = read_table("Params_Image.dat", t.image, false);
    t.n_physics = read_table("Params_Physics.dat", t.physics, false);
    return t;
}

// The library's table validation on what the files held (a truncated file
// whose counts need more floats than it has is an error here, where the
// reference silently computes with zeros).  Prints the reason and returns
// false on failure.
inline bool check_params(const Tables& t) {
    int64_t info[7];
    if (sm_tables_check(t.collimator.data(), t.n_collimator, t.detector.data(), t.n_detector, t.image.data(),
                        t.n_image, t.physics.data(), t.n_physics, info) != SM_OK) {
        std::fprintf(stderr, "ERROR: Params_*.dat (collimator %zu, detector %zu, image %zu floats read): %s\n",
                     t.n_collimator, t.n_detector, t.n_image, sm_last_error());
        return false;
    }
    return true;
}

inline void print_collimator(const Tables& t) {
    const int layers = (int)std::floor(t.collimator[0] + 0.001f);
    for (int l = 0; l < layers && l < 9; ++l) {
        const float* L = &t.collimator[(l + 1) * 10];
        std::printf("############ Collimator %d ############\n", l);
        std::printf("Number of collimator holes = %g\n", L[0]);
        std::printf("Width of collimator layer(X direction) = %gmm\n", L[1]);
        std::printf("Thickness of collimator layer(Y direction) = %gmm\n", L[2]);
        std::printf("Height of collimator layer(Z direction) = %gmm\n", L[3]);
        std::printf("Collimator Layer to 1st Collimator Layer = %gmm\n", L[4]);
        std::printf("Total Coeff of collimator layer = %g\n", L[5]);
        std::printf("Photon-electric Coeff of collimator layer = %g\n", L[6]);
        std::printf("Compton Coeff of collimator layer = %g\n", L[7]);
    }
    std::printf("FOV center to 1st Collimator = %g\n", t.image[11]);
}

// "<prefix>_shift_%f_%f_%f.sysmat" (PEGen_CircularHole.cpp:146, ScatterGen_CircularHole.cpp:200, :220)
inline std::string sysmat_name(const char* prefix, const Tables& t) {
    char buf[2048];
    std::snprintf(buf, sizeof(buf), "%s_shift_%f_%f_%f.sysmat", prefix, t.image[8], t.image[9], t.image[10]);
    return buf;
}

struct Grid {
    int n_crystals, nx, ny, nz, n_rotations;
    int64_t voxels;
};

inline Grid grid_of(const Tables& t) {
    Grid g;
    g.n_crystals = (int)std::floor(t.detector[0] + 0.001f);
    g.nx = (int)std::floor(t.image[0] + 0.001f);
    g.ny = (int)std::floor(t.image[1] + 0.001f);
    g.nz = (int)std::floor(t.image[2] + 0.001f);
    g.n_rotations = (int)std::floor(t.image[6] + 0.001f);
    if (g.n_rotations < 1) g.n_rotations = 1;
    g.voxels = (int64_t)g.nx * g.ny * g.nz;
    return g;
}

inline bool write_all(FILE* f, const float* p, size_t n) { return std::fwrite(p, sizeof(float), n, f) == n; }

}  // namespace cli
