/* TEST INFRASTRUCTURE ONLY -- part of the oracle, never linked into the product.
 *
 * OpenMP driver around the reference's own kernel code compiled for the host
 * (see ref_shim.h and the recipe in oracle/Makefile).  Built twice: with
 * REF_REAL=float (the reference's arithmetic, IEEE single, no fused
 * multiply-add) and REF_REAL=double (the same source with `float` redefined
 * to `double`).  Inputs are always the float32 Params tables; the FP64 build
 * widens them exactly.  Results are returned as double.
 *
 * Entry points (C ABI, called through ctypes by tests/ and bench.py only):
 *   ref_pe_entries         photodetectorCudaMe (PESysMatGen.cu:375-764) for a list
 *                          of (crystal row, voxel column) cells
 *   ref_box_ray_batch      length_box_ray        (PESysMatGen.cu:19-151)
 *   ref_box_inside_batch   length_box_ray_inside (PESysMatGen.cu:153-307)
 *   ref_cylinder_batch     length_cylinder_ray   (PESysMatGen.cu:309-373)
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
thread_local unsigned int ref_div[3] = {8u, 16u, 8u};

/* Defined in the extracted reference source (oracle/_ref/pe_kernel.cpp). */
void photodetectorCudaMe(real* dst, real* col, real* det, real* img, int numProjectionSingle, int numImagebin);
real length_box_ray(real, real, real, real, real, real, real, real, real, real, real, real);
real length_box_ray_inside(real, real, real, real, real, real, real, real, real, real, real, real);
real length_cylinder_ray(real, real, real, real, real, real, real, real, real, real, real);

static std::vector<real> widen(const float* src, int64_t n, int64_t min_len) {
    std::vector<real> out((size_t)(n > min_len ? n : min_len), (real)0);
    for (int64_t i = 0; i < n; ++i) out[(size_t)i] = (real)src[i];
    return out;
}

extern "C" {

/* Evaluate the reference PE kernel for cells (rows[i], cols[i]), where
 * cols[i] indexes the full volume described by img[0..2].  Each cell is run
 * as the reference CLI runs it: as part of the one-plane slab that contains
 * it (img[2] = 1, img[30] = full nz, img[31] = the cell's z), so the
 * kernel's 32-bit index row * numImagebin + col stays in range
 * (PEGen_CircularHole.cpp:181-194, PESysMatGen.cu:424). */
int ref_pe_entries(const float* col, int64_t ncol, const float* det, int64_t ndet,
                   const float* img, int divx, int divy, int divz,
                   int n_rows_total, int n_cols_total,
                   const int64_t* rows, const int64_t* cols, int64_t n,
                   double* out, int nthreads)
{
    (void)n_cols_total;
    std::vector<real> c = widen(col, ncol, 80000), d = widen(det, ndet, 80000);
    const int nx = (int)img[0], ny = (int)img[1], nz = (int)img[2];
    const int plane = nx * ny;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<real> im = widen(img, 100, 100);
        im[2] = (real)1.0f;
        im[30] = (real)(float)nz;
#pragma omp for schedule(dynamic, 8)
        for (int64_t i = 0; i < n; ++i) {
            ref_div[0] = (unsigned)divx; ref_div[1] = (unsigned)divy; ref_div[2] = (unsigned)divz;
            const int64_t z = cols[i] / plane;
            const int64_t in_plane = cols[i] % plane;
            im[31] = (real)(float)z;
            blockDim = {1u, 1u, 1u};
            threadIdx = {0u, 0u, 0u};
            blockIdx = {(unsigned)rows[i], (unsigned)in_plane, 0u};
            real cell = (real)0;
            /* The kernel writes dst[row * plane + in_plane]; point that slot at `cell`. */
            int64_t dst_index = rows[i] * (int64_t)plane + in_plane;
            real* base = reinterpret_cast<real*>(reinterpret_cast<uintptr_t>(&cell) - (uintptr_t)(dst_index * (int64_t)sizeof(real)));
            photodetectorCudaMe(base, c.data(), d.data(), im.data(), n_rows_total, plane);
            out[i] = (double)cell;
        }
    }
    return 0;
}

/* args: n x 12 floats (x_in, y_in, z_in, x_out, y_out, z_out, x1, y1, z1, x2, y2, z2). */
int ref_box_ray_batch(const float* args, int64_t n, double* out) {
    for (int64_t i = 0; i < n; ++i) {
        const float* a = args + 12 * i;
        out[i] = (double)length_box_ray(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11]);
    }
    return 0;
}

int ref_box_inside_batch(const float* args, int64_t n, double* out) {
    for (int64_t i = 0; i < n; ++i) {
        const float* a = args + 12 * i;
        out[i] = (double)length_box_ray_inside(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11]);
    }
    return 0;
}

/* args: n x 11 floats (x_in, y_in, z_in, x_out, y_out, z_out, x_c, y1, y2, z_c, R). */
int ref_cylinder_batch(const float* args, int64_t n, double* out) {
    for (int64_t i = 0; i < n; ++i) {
        const float* a = args + 11 * i;
        out[i] = (double)length_cylinder_ray(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10]);
    }
    return 0;
}

int ref_real_bytes(void) { return (int)sizeof(real); }

}  /* extern "C" */
