// PEGen_CircularHole: photoelectric sysmat generator with the reference CLI's
// inputs, flags and output (PEGen_RayTracing_CircularHole/PEGen_CircularHole.cpp:37-237).
//
//   PEGen_CircularHole [-cuda GPU_ID] [-sv X Y Z] [-sc X Y Z]
//
// Reads Params_{Collimator,Detector,Image,Physics}.dat from the working
// directory and writes PE_SysMat_shift_<x>_<y>_<z>.sysmat: float32
// [rotation][crystal][voxel x + nx (y + ny z)].  Defaults reproduce the
// reference (voxel centre, 8 x 16 x 8 crystal sub-cells); -sv / -sc set voxel
// sub-samples and crystal sub-cells.  Several rotations run as the work items
// of one persistent launch (the reference launches once per slab and
// rotation, PEGen_CircularHole.cpp:167-223); a matrix too large for that goes
// by slabs of z-planes.  The file is written while the device computes.
#include <algorithm>
#include <cstring>
#include <thread>

#include <cuda_runtime.h>

#include "cli_common.h"
#include "sysmat_b200.h"

static void usage(const char* argv0) { std::printf("Usage: %s [-cuda GPU_ID] [-sv X Y Z] [-sc X Y Z]\n", argv0); }

int main(int argc, char* argv[]) {
    cli::Tables t = cli::read_params();
    cli::print_collimator(t);
    if (!cli::check_params(t)) return 1;
    int cuda_id = 0;
    sm_pe_options opt;
    sm_pe_options_reference(&opt);
    for (int i = 1; i < argc; ++i) {
        if (std::strcmp(argv[i], "-cuda") == 0 && i + 1 < argc) {
            cuda_id = std::atoi(argv[++i]);
        } else if ((std::strcmp(argv[i], "-sv") == 0 || std::strcmp(argv[i], "-sc") == 0) && i + 3 < argc) {
            int* dst = argv[i][2] == 'v' ? opt.sv : opt.sc;
            for (int a = 0; a < 3; ++a) dst[a] = std::atoi(argv[i + 1 + a]);
            i += 3;
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
    const int64_t total = (int64_t)g.n_crystals * g.voxels * g.n_rotations;
    std::printf("FOV dimension : %d %d %d\n", g.nx, g.ny, g.nz);
    std::printf("FOV Voxel Size(mm) : %f %f %f\n", t.image[3], t.image[4], t.image[5]);
    std::printf("numDet=%d  fullVox=%lld  rotations=%d  sysmatBytes=%lld (%.2f GB)\n", g.n_crystals,
                (long long)g.voxels, g.n_rotations, (long long)(total * 4), (double)total * 4.0 / (1 << 30));
    if (total <= 0) {
        std::fprintf(stderr, "ERROR: totalBytes invalid\n");
        return 2;
    }
    sm_context* ctx = nullptr;
    sm_geometry* geo = nullptr;
    if (sm_context_create(cuda_id, &ctx) != SM_OK ||
        sm_geometry_create(ctx, t.collimator.data(), t.collimator.size(), t.detector.data(), t.detector.size(),
                           t.image.data(), t.image.size(), t.physics.data(), t.physics.size(), &geo) != SM_OK) {
        std::fprintf(stderr, "ERROR: %s\n", sm_last_error());
        return 1;
    }
    const std::string name = cli::sysmat_name("PE_SysMat", t);
    FILE* fp = std::fopen(name.c_str(), "wb+");
    if (!fp) {
        std::fprintf(stderr, "ERROR: open sysmat output %s\n", name.c_str());
        return 1;
    }
    std::thread writer;
    bool write_ok = true;
    const int64_t plane = (int64_t)g.nx * g.ny;
    const int64_t rot_floats = (int64_t)g.n_crystals * g.voxels;
    // Whole rotations as the work items of one persistent launch (sm_pe_batch)
    // when a rotation's matrix fits the device budget: up to 64 rotations per
    // launch, at most 4 GiB of output per group, written while the next group
    // computes.  Otherwise slabs of z-planes, one sm_pe_compute per slab.
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
    const int64_t budget = std::min<int64_t>((int64_t)4 << 30, (int64_t)(free_b / 4));
    const int group = (int)std::min<int64_t>({(int64_t)g.n_rotations, 64, budget / std::max<int64_t>(1, 4 * rot_floats)});
    if (group >= 1 && g.n_rotations > 1) {
        float* d_out = nullptr;
        if (cudaMalloc(&d_out, sizeof(float) * (size_t)rot_floats * (size_t)group) != cudaSuccess) {
            std::fprintf(stderr, "ERROR: device allocation of %d rotations failed\n", group);
            return 1;
        }
        std::vector<float> host[2];
        int which = 0;
        for (int r0 = 0; r0 < g.n_rotations; r0 += group) {
            const int nr = std::min(group, g.n_rotations - r0);
            std::vector<const sm_geometry*> geos(nr, geo);
            std::vector<sm_pe_options> opts(nr, opt);
            std::vector<int> rots(nr);
            std::vector<float*> dst(nr);
            std::vector<int64_t> lds(nr, g.voxels);
            for (int i = 0; i < nr; ++i) {
                rots[i] = r0 + i;
                dst[i] = d_out + (size_t)i * (size_t)rot_floats;
            }
            std::printf("########################\nRotations (%d..%d) processing in one launch ...\n"
                        "########################\n", r0, r0 + nr - 1);
            sm_pe_batch* batch = nullptr;
            int rc = sm_pe_batch_create(ctx, nr, geos.data(), opts.data(), rots.data(), dst.data(), lds.data(), &batch);
            if (rc == SM_OK) rc = sm_pe_batch_run(batch, nullptr);
            if (rc == SM_OK) rc = sm_context_sync(ctx, nullptr);
            sm_pe_batch_destroy(batch);
            if (rc != SM_OK) {
                std::fprintf(stderr, "ERROR: %s\n", sm_last_error());
                if (writer.joinable()) writer.join();
                return 3;
            }
            if (writer.joinable()) writer.join();
            host[which].resize((size_t)rot_floats * (size_t)nr);
            if (cudaMemcpy(host[which].data(), d_out, sizeof(float) * host[which].size(), cudaMemcpyDeviceToHost) !=
                cudaSuccess) {
                std::fprintf(stderr, "ERROR: copying rotations %d..%d to the host failed\n", r0, r0 + nr - 1);
                return 3;
            }
            // rotations r0 .. r0 + nr - 1 are contiguous in the file ([rotation][crystal][voxel])
            const float* src = host[which].data();
            const size_t n = host[which].size();
            writer = std::thread([=, &write_ok] {
                if (fseeko(fp, (off_t)((int64_t)r0 * rot_floats * 4), SEEK_SET) != 0 || !cli::write_all(fp, src, n))
                    write_ok = false;
            });
            which ^= 1;
        }
        if (writer.joinable()) writer.join();
        cudaFree(d_out);
    } else {
        // slabs of whole z-planes, at most 1 GiB of host buffer each, two buffers
        int slab = (int)std::max<int64_t>(1, ((int64_t)1 << 28) / std::max<int64_t>(1, (int64_t)g.n_crystals * plane));
        slab = std::min(slab, g.nz);
        std::vector<float> buf[2];
        buf[0].resize((size_t)g.n_crystals * plane * slab);
        buf[1].resize(buf[0].size());
        int which = 0;
        for (int rot = 0; rot < g.n_rotations; ++rot) {
            std::printf("########################\nRotation (%d) processing ...\n########################\n", rot);
            for (int z0 = 0; z0 < g.nz; z0 += slab) {
                const int nz = std::min(slab, g.nz - z0);
                const int64_t cols = plane * nz;
                float* out = buf[which].data();
                if (sm_pe_compute(ctx, geo, &opt, rot, 0, g.n_crystals, z0, nz, out, cols, 0, nullptr) != SM_OK) {
                    std::fprintf(stderr, "ERROR: %s\n", sm_last_error());
                    if (writer.joinable()) writer.join();
                    return 3;
                }
                if (writer.joinable()) writer.join();
                // rows of this slab go to [rot][det][z0 * plane ...] (PEGen_CircularHole.cpp:202-216)
                writer = std::thread([=, &write_ok] {
                    for (int d = 0; d < g.n_crystals; ++d) {
                        const int64_t off = (((int64_t)rot * g.n_crystals + d) * g.voxels + (int64_t)z0 * plane) * 4;
                        if (fseeko(fp, (off_t)off, SEEK_SET) != 0 ||
                            !cli::write_all(fp, out + (int64_t)d * cols, (size_t)cols))
                            write_ok = false;
                    }
                });
                std::printf("WROTE slab z0=%d slabZ=%d bins=%lld\n", z0, nz, (long long)cols);
                which ^= 1;
            }
        }
    }
    if (writer.joinable()) writer.join();
    std::fclose(fp);
    sm_geometry_destroy(geo);
    sm_context_destroy(ctx);
    if (!write_ok) {
        std::fprintf(stderr, "ERROR: writing %s failed\n", name.c_str());
        return 1;
    }
    std::printf("########################\nPhoton Electric 3D Sysmat Written (slabbed, exact).\n########################\n");
    return 0;
}
