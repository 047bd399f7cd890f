// The reference's three scatter generators from one source, selected by
// SCATTER_PARTS at compile time:
//   3  ScatterGen_CircularHole  (ScatterGen_RayTracing_CircularHole/ScatterGen_CircularHole.cpp:38-232)
//        [-PE f] [-GeoCrystal f] [-GeoCollimator f] [-cuda N]
//        writes Scatter_SysMat_shift_* if Physics[2] == 1, SysMat_withScatter_shift_* if Physics[3] == 1
//   1  ScatterGen_Crystal       (ScatterGen_Crystal/ScatterGen_Crystal.cpp)
//        [-PE f] [-GeoCrystal f] [-cuda N]
//        writes Scatter_Crystal_SysMat_shift_*, and SysMat_shift_* if Physics[3] == 1
//   2  ScatterGen_Collimator    (ScatterGen_Collimator/ScatterGen_Collimator.cpp)
//        [-PE f] [-GeoCollimator f] [-cuda N]
//        writes Scatter_SysMat_shift_*, and SysMat_shift_* if Physics[3] == 1
// -GeoCrystal / -GeoCollimator name a bitmap file to read and set Physics[8] /
// Physics[9] to 0, as the reference does; otherwise the bitmaps are computed
// and written to GeometryRelationShip_Crystal2Crystal /
// GeometryRelationShip_Collimator2Crystal.  Each rotation uses its own block
// of the PE sysmat (the reference passes rotation 0's block for every
// rotation, scatter.cu:2083-2084).
//
// -surrogate TOL (parts 3 and 1; no reference counterpart): the crystal part
// through the scatter surrogate (physics baseline, exact re-check, exact
// recompute of rows whose estimated relative error exceeds TOL), the
// collimator part exact; one scatter point per crystal as above; the bitmaps
// are computed on the device and no bitmap file is read or written.
#include <cstring>

#include <cuda_runtime.h>

#include "cli_common.h"
#include "sysmat_b200.h"

#ifndef SCATTER_PARTS
#define SCATTER_PARTS 3
#endif

static void usage(const char* argv0) {
    if (SCATTER_PARTS == 3)
        std::printf("Usage: %s [-PE PE_SysMat_path] [-GeoCrystal GeometryRelationShip_Crystal2Crystal_path] "
                    "[-GeoCollimator GeometryRelationShip_Collimator2Crystal_path] [-cuda GPU_ID] [-surrogate TOL]\n",
                    argv0);
    else if (SCATTER_PARTS == 1)
        std::printf("Usage: %s [-PE PE_SysMat_path] [-GeoCrystal GeometryRelationShip_Crystal2Crystal_path] [-cuda GPU_ID] "
                    "[-surrogate TOL]\n",
                    argv0);
    else
        std::printf("Usage: %s [-PE PE_SysMat_path] [-GeoCollimator GeometryRelationShip_Collimator2Crystal_path] "
                    "[-cuda GPU_ID]\n", argv0);
}

static int write_file(const std::string& name, const std::vector<float>& v) {
    FILE* f = std::fopen(name.c_str(), "wb+");
    if (!f || !cli::write_all(f, v.data(), v.size())) {
        std::fprintf(stderr, "ERROR: writing %s failed\n", name.c_str());
        if (f) std::fclose(f);
        return 1;
    }
    std::fclose(f);
    return 0;
}

// The crystal part (and, for parts 3, the exact collimator part) of every
// rotation through sm_scatter_surrogate.
static int run_surrogate(const cli::Tables& t, const cli::Grid& g, const std::vector<float>& pe, std::vector<float>& out,
                         size_t block, int cuda_id, float tol) {
    sm_context* ctx = nullptr;
    sm_geometry* geo = nullptr;
    float* d_pe = nullptr;
    float* d_out = nullptr;
    int rc = sm_context_create(cuda_id, &ctx);
    if (rc == SM_OK)
        rc = sm_geometry_create(ctx, t.collimator.data(), t.collimator.size(), t.detector.data(), t.detector.size(),
                                t.image.data(), t.image.size(), t.physics.data(), t.physics.size(), &geo);
    if (rc == SM_OK && (cudaMalloc(&d_pe, block * sizeof(float)) != cudaSuccess ||
                        cudaMalloc(&d_out, block * sizeof(float)) != cudaSuccess)) {
        std::fprintf(stderr, "ERROR: device allocation of %zu floats failed\n", 2 * block);
        rc = SM_ERR_ALLOC;
    }
    sm_surrogate_options so;
    sm_surrogate_options_default(&so);
    so.sp[0] = so.sp[1] = so.sp[2] = 1;
    so.parts = SCATTER_PARTS;
    so.tol = tol;
    for (int rot = 0; rc == SM_OK && rot < g.n_rotations; ++rot) {
        std::printf("########################\nRotation (%d) processing (surrogate, tol %g) ...\n########################\n",
                    rot, tol);
        sm_surrogate_stats st;
        if (cudaMemcpy(d_pe, pe.data() + rot * block, block * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
            rc = SM_ERR_CUDA;
            break;
        }
        rc = sm_scatter_surrogate(ctx, geo, &so, rot, d_pe, (int64_t)g.voxels, d_out, (int64_t)g.voxels, nullptr, nullptr,
                                  &st, nullptr);
        if (rc != SM_OK) break;
        if (cudaMemcpy(out.data() + rot * block, d_out, block * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
            rc = SM_ERR_CUDA;
            break;
        }
        std::printf("rows recomputed %d of %d, estimated row error median %.4g, %.1f ms\n", st.rows_recomputed,
                    g.n_crystals, st.holdout_median, st.ms_total);
    }
    if (rc != SM_OK) std::fprintf(stderr, "ERROR: %s\n", sm_last_error());
    if (d_pe) cudaFree(d_pe);
    if (d_out) cudaFree(d_out);
    sm_geometry_destroy(geo);
    sm_context_destroy(ctx);
    return rc == SM_OK ? 0 : 3;
}

int main(int argc, char* argv[]) {
    cli::Tables t = cli::read_params();
    cli::print_collimator(t);
    if (!cli::check_params(t)) return 1;
    std::string pe_name, geo_crystal = "GeometryRelationShip_Crystal2Crystal",
                         geo_collimator = "GeometryRelationShip_Collimator2Crystal";
    int cuda_id = 0;
    float surrogate_tol = 0.0f;
    for (int i = 1; i < argc; ++i) {
        if (std::strcmp(argv[i], "-PE") == 0 && i + 1 < argc) {
            pe_name = argv[++i];
        } else if ((SCATTER_PARTS & 1) && std::strcmp(argv[i], "-GeoCrystal") == 0 && i + 1 < argc) {
            geo_crystal = argv[++i];
            t.physics[8] = 0.0f;
        } else if ((SCATTER_PARTS & 2) && std::strcmp(argv[i], "-GeoCollimator") == 0 && i + 1 < argc) {
            geo_collimator = argv[++i];
            t.physics[9] = 0.0f;
        } else if (std::strcmp(argv[i], "-cuda") == 0 && i + 1 < argc) {
            cuda_id = std::atoi(argv[++i]);
        } else if ((SCATTER_PARTS & 1) && std::strcmp(argv[i], "-surrogate") == 0 && i + 1 < argc) {
            surrogate_tol = std::atof(argv[++i]);
            if (!(surrogate_tol > 0.0f)) {
                std::fprintf(stderr, "-surrogate needs a tolerance > 0\n");
                return 1;
            }
        } else if (std::strcmp(argv[i], "-h") == 0 || std::strcmp(argv[i], "--help") == 0) {
            usage(argv[0]);
            return 0;
        } else {
            std::fprintf(stderr, "Unknown parameter or missing argument: %s\n", argv[i]);
            usage(argv[0]);
            return EXIT_FAILURE;
        }
    }
    const cli::Grid g = cli::grid_of(t);
    const size_t block = (size_t)g.n_crystals * (size_t)g.voxels;
    const size_t total = block * (size_t)g.n_rotations;
    if (pe_name.empty()) pe_name = cli::sysmat_name("PE_SysMat", t);
    std::printf("Photon Electric SysMat: %s\n", pe_name.c_str());
    std::vector<float> pe(total, 0.0f);
    {
        FILE* f = std::fopen(pe_name.c_str(), "rb");
        if (!f) {
            std::fprintf(stderr, "ERROR: open %s\n", pe_name.c_str());
            return 1;
        }
        const size_t got = std::fread(pe.data(), sizeof(float), total, f);
        std::fclose(f);
        if (got < total) std::fprintf(stderr, "warning: %s holds %zu of %zu floats\n", pe_name.c_str(), got, total);
    }
    std::vector<float> out(total, 0.0f);
    std::printf("FOV dimension : %d %d %d\n", g.nx, g.ny, g.nz);
    if (surrogate_tol > 0.0f) {
        const int rc = run_surrogate(t, g, pe, out, block, cuda_id, surrogate_tol);
        if (rc != 0) return rc;
    }
    for (int rot = 0; surrogate_tol <= 0.0f && rot < g.n_rotations; ++rot) {
        std::printf("########################\nRotation (%d) processing ...\n########################\n", rot);
        t.image[20] = (float)rot;
        const int q = sm_scatter_legacy(SCATTER_PARTS, SCATTER_PARTS == 1 ? nullptr : t.collimator.data(),
                                        t.detector.data(), t.image.data(), t.physics.data(), pe.data() + rot * block,
                                        (SCATTER_PARTS & 1) ? geo_crystal.c_str() : nullptr,
                                        (SCATTER_PARTS & 2) ? geo_collimator.c_str() : nullptr,
                                        out.data() + rot * block, cuda_id);
        if (q < 0) {
            std::fprintf(stderr, "ERROR: %s\n", sm_last_error());
            return 3;
        }
        std::printf("numImagebin = %d\n", q);
        // the bitmaps written for the first rotation serve the others
        if (SCATTER_PARTS & 1) t.physics[8] = 0.0f;
        if (SCATTER_PARTS & 2) t.physics[9] = 0.0f;
    }
    int rc = 0;
    const char* scatter_prefix = SCATTER_PARTS == 1 ? "Scatter_Crystal_SysMat" : "Scatter_SysMat";
    if (SCATTER_PARTS != 3 || t.physics[2] == 1.0f) {
        rc |= write_file(cli::sysmat_name(scatter_prefix, t), out);
        std::printf("########################\nCompton Scatter Sysmat written.\n########################\n");
    }
    if (t.physics[3] == 1.0f) {
        for (size_t i = 0; i < total; ++i) out[i] += pe[i];
        rc |= write_file(cli::sysmat_name(SCATTER_PARTS == 3 ? "SysMat_withScatter" : "SysMat", t), out);
        std::printf("########################\nFull Sysmat written.\n########################\n");
    }
    return rc;
}
