/* TEST INFRASTRUCTURE ONLY -- the reference's scatter kernels built for sm_100a.
 *
 * Compiles the reference's ScatterGen_RayTracing_CircularHole/scatter.cu as it
 * is and adds C entry points for the tests and bench.py, each launching one
 * reference kernel with the reference's own launch shape on device buffers
 * and reporting the kernel time from CUDA events:
 *   ref_cuda_bitmap_crystal      geometryRelationShip_Crystal2Crystal (scatter.cu:2123-2132)
 *   ref_cuda_bitmap_collimator   geometryRelationShip_Collimator2Crystal (:2253-2263)
 *   ref_cuda_crystal_scatter     crystalScatterSysMatCuda on rows [0, n_rows) (:2169-2194)
 *   ref_cuda_collimator_scatter  collimatorScatterSysMatCuda on rows [0, n_rows) (:2303-2308)
 * Restricting the grid's x extent to n_rows crystals computes exactly those
 * rows of the reference's matrix (each thread owns one (row, voxel, source)).
 */
#include "scatter.cu"

static float ref_time_ms(cudaEvent_t e0, cudaEvent_t e1) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
}

extern "C" int ref_cuda_bitmap_crystal(unsigned int* d_words, float* d_det, int n_crystals, float* ms_out) {
    long long total = (long long)n_crystals * n_crystals * n_crystals;
    long long blocks = (total + 255) / 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    geometryRelationShip_Crystal2Crystal<<<(unsigned)blocks, 256>>>(d_words, d_det);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    if (ms_out) *ms_out = ref_time_ms(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err == cudaSuccess) err = cudaGetLastError();
    return (int)err;
}

extern "C" int ref_cuda_bitmap_collimator(unsigned int* d_words, float* d_det, float* d_col, int n_crystals,
                                          int n_holes, float* ms_out) {
    long long total = (long long)n_holes * n_crystals * n_crystals;
    long long blocks = (total + 255) / 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    geometryRelationShip_Collimator2Crystal<<<(unsigned)blocks, 256>>>(d_words, d_det, d_col);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    if (ms_out) *ms_out = ref_time_ms(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err == cudaSuccess) err = cudaGetLastError();
    return (int)err;
}

extern "C" int ref_cuda_crystal_scatter(float* d_dst, float* d_det, float* d_img, float* d_phys, float* d_pe,
                                        unsigned int* d_bitmap, int n_crystals, int n_voxels, int n_rows,
                                        float* ms_out) {
    dim3 block(16, 16, 1);
    dim3 grid((n_rows + 15) / 16, (n_voxels + 15) / 16, n_crystals);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    crystalScatterSysMatCuda<<<grid, block>>>(d_dst, d_det, d_img, d_phys, d_pe, d_bitmap, n_crystals, n_voxels);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    if (ms_out) *ms_out = ref_time_ms(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err == cudaSuccess) err = cudaGetLastError();
    return (int)err;
}

extern "C" int ref_cuda_collimator_scatter(float* d_dst, float* d_col, float* d_det, float* d_img, float* d_phys,
                                           unsigned int* d_bitmap, int n_crystals, int n_voxels, int n_holes,
                                           int n_rows, float* ms_out) {
    dim3 block(16, 16, 1);
    dim3 grid((n_rows + 15) / 16, (n_voxels + 15) / 16, n_holes);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    collimatorScatterSysMatCuda<<<grid, block>>>(d_dst, d_col, d_det, d_img, d_phys, d_bitmap, n_crystals,
                                                 n_voxels);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    if (ms_out) *ms_out = ref_time_ms(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err == cudaSuccess) err = cudaGetLastError();
    return (int)err;
}
