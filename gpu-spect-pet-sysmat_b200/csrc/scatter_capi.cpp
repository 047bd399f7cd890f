// Legacy `scatter` drop-in (ScatterGen_RayTracing_CircularHole/scatter.h:4-5).
#include <cstdio>

#include "sysmat_b200.h"

extern "C" int scatter(float*, float*, float*, float*, float*, const char*, const char*, float*, int) {
    std::fprintf(stderr, "scatter: not available in this build\n");
    return -1;
}
