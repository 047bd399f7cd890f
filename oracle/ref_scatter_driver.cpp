/* TEST INFRASTRUCTURE ONLY -- part of the oracle, never linked into the product.
 *
 * OpenMP driver around the reference's own scatter kernel code compiled for
 * the host (ref_shim.h and the recipe in oracle/Makefile), built with
 * REF_REAL=float (the reference's arithmetic) and REF_REAL=double (the same
 * source with `float` read as `double`).  Inputs are the float32 Params
 * tables and PE matrix; the FP64 build widens them exactly.
 *
 * Entry points (C ABI, called through ctypes by tests/ and bench.py only):
 *   ref_bitmap_crystal      geometryRelationShip_Crystal2Crystal   (scatter.cu:1440-1540)
 *   ref_bitmap_collimator   geometryRelationShip_Collimator2Crystal (scatter.cu:1939-2009)
 *   ref_crystal_scatter_entries     crystalScatterSysMatCuda     (scatter.cu:1077-1437),
 *                                   summed over every scatter crystal (grid z)
 *   ref_collimator_scatter_entries  collimatorScatterSysMatCuda  (scatter.cu:1544-1936),
 *                                   summed over every layer-0 hole (grid z)
 *   ref_compton_integral_batch      computeComptonIntegral       (scatter.cu:981-995)
 */
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

#ifndef REF_REAL
#define REF_REAL float
#endif
typedef REF_REAL real;

struct ref_uint3 { unsigned int x, y, z; };
thread_local ref_uint3 blockIdx;
thread_local ref_uint3 threadIdx;
thread_local ref_uint3 blockDim;
thread_local unsigned int ref_div[3] = {1u, 1u, 1u};

/* Defined in the extracted reference source (oracle/_ref/scatter_kernel.cpp). */
void crystalScatterSysMatCuda(real* dst, real* det, real* img, real* phys, real* pe, unsigned int* bitmap,
                              int numProjectionSingle, int numImagebin);
void collimatorScatterSysMatCuda(real* dst, real* col, real* det, real* img, real* phys, unsigned int* bitmap,
                                 int numProjectionSingle, int numImagebin);
void geometryRelationShip_Crystal2Crystal(unsigned int* dst, real* det);
void geometryRelationShip_Collimator2Crystal(unsigned int* dst, real* det, real* col);
real computeComptonIntegral(real E0, real lo, real hi, real delta);

static std::vector<real> widen(const float* src, int64_t n, int64_t min_len) {
    std::vector<real> out((size_t)(n > min_len ? n : min_len), (real)0);
    for (int64_t i = 0; i < n; ++i) out[(size_t)i] = (real)src[i];
    return out;
}

/* Points the kernel's write of dst[index] at `cell`. */
static real* cell_base(real* cell, int64_t index) {
    return reinterpret_cast<real*>(reinterpret_cast<uintptr_t>(cell) - (uintptr_t)(index * (int64_t)sizeof(real)));
}

extern "C" {

/* Runs the bitmap kernel for every (i, j, k) thread of the reference's
 * 1-D launch (256 threads per block); `words` must be zeroed by the caller. */
int ref_bitmap_crystal(const float* det, int64_t ndet, unsigned int* words) {
    std::vector<real> d = widen(det, ndet, 80000);
    const int64_t N = (int64_t)det[0];
    const int64_t total = N * N * N;
    blockDim = {256u, 1u, 1u};
    for (int64_t idx = 0; idx < total; ++idx) {
        blockIdx = {(unsigned)(idx / 256), 0u, 0u};
        threadIdx = {(unsigned)(idx % 256), 0u, 0u};
        geometryRelationShip_Crystal2Crystal(words, d.data());
    }
    return 0;
}

int ref_bitmap_collimator(const float* det, int64_t ndet, const float* col, int64_t ncol, unsigned int* words) {
    std::vector<real> d = widen(det, ndet, 80000), c = widen(col, ncol, 80000);
    const int64_t N = (int64_t)det[0];
    const int64_t H = (int64_t)col[10];
    const int64_t total = H * N * N;
    blockDim = {256u, 1u, 1u};
    for (int64_t idx = 0; idx < total; ++idx) {
        blockIdx = {(unsigned)(idx / 256), 0u, 0u};
        threadIdx = {(unsigned)(idx % 256), 0u, 0u};
        geometryRelationShip_Collimator2Crystal(words, d.data(), c.data());
    }
    return 0;
}

/* Entries (rows[i], cols[i]) of the crystal-scatter sysmat: the kernel run
 * for every scatter crystal z in [0, N) of that cell, accumulated in z order.
 * pe is the [N][V] PE sysmat of the rotation (float32). */
int ref_crystal_scatter_entries(const float* det, int64_t ndet, const float* img, const float* phys,
                                const float* pe, const unsigned int* bitmap, const int64_t* rows,
                                const int64_t* cols, int64_t n, double* out, int nthreads) {
    std::vector<real> d = widen(det, ndet, 80000), im = widen(img, 100, 100), ph = widen(phys, 100, 100);
    const int N = (int)det[0];
    const int nx = (int)img[0], ny = (int)img[1], nz = (int)img[2];
    const int V = nx * ny * nz;
    std::vector<real> P = widen(pe, (int64_t)N * V, 0);
    unsigned int* bm = const_cast<unsigned int*>(bitmap);
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int64_t i = 0; i < n; ++i) {
        blockDim = {1u, 1u, 1u};
        threadIdx = {0u, 0u, 0u};
        real cell = (real)0;
        real* base = cell_base(&cell, rows[i] * (int64_t)V + cols[i]);
        for (int s = 0; s < N; ++s) {
            blockIdx = {(unsigned)rows[i], (unsigned)cols[i], (unsigned)s};
            crystalScatterSysMatCuda(base, d.data(), im.data(), ph.data(), P.data(), bm, N, V);
        }
        out[i] = (double)cell;
    }
    return 0;
}

int ref_collimator_scatter_entries(const float* col, int64_t ncol, const float* det, int64_t ndet, const float* img,
                                   const float* phys, const unsigned int* bitmap, const int64_t* rows,
                                   const int64_t* cols, int64_t n, double* out, int nthreads) {
    std::vector<real> c = widen(col, ncol, 80000), d = widen(det, ndet, 80000), im = widen(img, 100, 100),
                      ph = widen(phys, 100, 100);
    const int N = (int)det[0];
    const int H = (int)col[10];
    const int nx = (int)img[0], ny = (int)img[1], nz = (int)img[2];
    const int V = nx * ny * nz;
    unsigned int* bm = const_cast<unsigned int*>(bitmap);
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int64_t i = 0; i < n; ++i) {
        blockDim = {1u, 1u, 1u};
        threadIdx = {0u, 0u, 0u};
        real cell = (real)0;
        real* base = cell_base(&cell, rows[i] * (int64_t)V + cols[i]);
        for (int h = 0; h < H; ++h) {
            blockIdx = {(unsigned)rows[i], (unsigned)cols[i], (unsigned)h};
            collimatorScatterSysMatCuda(base, c.data(), d.data(), im.data(), ph.data(), bm, N, V);
        }
        out[i] = (double)cell;
    }
    return 0;
}

/* args: n x 3 floats (E0, theta_low, theta_high); step 0.01 as the kernels pass it. */
int ref_compton_integral_batch(const float* args, int64_t n, double* out) {
    for (int64_t i = 0; i < n; ++i) {
        const float* a = args + 3 * i;
        out[i] = (double)computeComptonIntegral((real)a[0], (real)a[1], (real)a[2], 0.01);
    }
    return 0;
}

int ref_scatter_real_bytes(void) { return (int)sizeof(real); }

}  /* extern "C" */
