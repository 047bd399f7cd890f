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

namespace cli {

struct Tables {
    std::vector<float> collimator = std::vector<float>(80000, 0.0f);
    std::vector<float> detector = std::vector<float>(80000, 0.0f);
    std::vector<float> image = std::vector<float>(100, 0.0f);
    std::vector<float> physics = std::vector<float>(100, 0.0f);
};

// Reads the table; a missing file is fatal (exit 1), a short one leaves zeros
// as the reference's unchecked fread does, with a warning.
inline void read_table(const char* name, std::vector<float>& out) {
    FILE* f = std::fopen(name, "rb");
    if (!f) {
        std::fprintf(stderr, "ERROR: open %s\n", name);
        std::exit(1);
    }
    const size_t got = std::fread(out.data(), sizeof(float), out.size(), f);
    std::fclose(f);
    if (got < out.size())
        std::fprintf(stderr, "warning: %s holds %zu of %zu floats; the rest are zero\n", name, got, out.size());
}

inline Tables read_params() {
    Tables t;
    read_table("Params_Collimator.dat", t.collimator);
    read_table("Params_Detector.dat", t.detector);
    read_table("Params_Image.dat", t.image);
    read_table("Params_Physics.dat", t.physics);
    return t;
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
