// `scatter` of the reference's collimator-only generator
// (ScatterGen_Collimator/scatter.h:4-5, body ScatterGen_Collimator/scatter.cu:1511-1747):
// primary Compton scatter in the plate-0 holes only, one bitmap file.  Built as
// libsysmat_b200_scatter_collimator.so because its signature differs from the
// combined generator's `scatter`.
#include <cstdio>

#define SYSMAT_B200_SINGLE_PART_SCATTER
#include "sysmat_b200.h"

extern "C" int scatter(float* parameter_Collimator, float* parameter_Detector, float* parameter_Image,
                       float* parameter_Physics, float* PE_SysMat, const char* FnameGeo, float* dst, int cuda_id) {
    if (!parameter_Collimator || !parameter_Detector || !parameter_Image || !parameter_Physics || !dst) {
        std::fprintf(stderr, "scatter: null argument\n");
        return -1;
    }
    const int rc = sm_scatter_legacy(2, parameter_Collimator, parameter_Detector, parameter_Image, parameter_Physics,
                                     PE_SysMat, nullptr, FnameGeo, dst, cuda_id);
    if (rc < 0) {
        std::fprintf(stderr, "scatter: %s\n", sm_last_error());
        return -1;
    }
    return rc;
}
