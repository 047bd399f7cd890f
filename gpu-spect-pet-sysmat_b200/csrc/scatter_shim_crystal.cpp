// `scatter` of the reference's crystal-only generator (ScatterGen_Crystal/scatter.h:4,
// body ScatterGen_Crystal/scatter.cu:1528-1738): primary Compton scatter in the
// crystals only, one bitmap file.  Built as libsysmat_b200_scatter_crystal.so
// because its signature differs from the combined generator's `scatter`.
#include <cstdio>

#define SYSMAT_B200_SINGLE_PART_SCATTER
#include "sysmat_b200.h"

extern "C" int scatter(float* parameter_Detector, float* parameter_Image, float* parameter_Physics, float* PE_SysMat,
                       const char* FnameGeo, float* dst, int cuda_id) {
    if (!parameter_Detector || !parameter_Image || !parameter_Physics || !PE_SysMat || !dst) {
        std::fprintf(stderr, "scatter: null argument\n");
        return -1;
    }
    const int rc = sm_scatter_legacy(1, nullptr, parameter_Detector, parameter_Image, parameter_Physics, PE_SysMat,
                                     FnameGeo, nullptr, dst, cuda_id);
    if (rc < 0) {
        std::fprintf(stderr, "scatter: %s\n", sm_last_error());
        return -1;
    }
    return rc;
}
