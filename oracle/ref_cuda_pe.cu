/* TEST INFRASTRUCTURE ONLY -- the reference's PE kernel built for sm_100a.
 *
 * Compiles the reference's PESysMatGen.cu (with the crystal sub-cell counts of
 * PESysMatGen.cu:435 turned into REF_DIVX/Y/Z macros by the recipe in
 * oracle/Makefile) and adds two C entry points for the tests and bench.py:
 *   ref_cuda_pe_kernel   launches photodetectorCudaMe with the reference's own
 *                        launch shape (PESysMatGen.cu:806-807) on device buffers
 *                        and reports the kernel time from CUDA events;
 *   ref_cuda_PESysMatGen the reference's own host entry point (allocates,
 *                        copies, launches, copies back and frees per call).
 */
#include "pe_cuda_src.cu"

extern "C" int ref_cuda_pe_kernel(float* d_col, float* d_det, float* d_img, float* d_dst,
                                  int n_rows, int n_imagebin, int iters, float* ms_out) {
    dim3 block(16, 32);
    dim3 grid((n_rows + 15) / block.x, (n_imagebin + 31) / block.y);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (int i = 0; i < iters; ++i)
        photodetectorCudaMe<<<grid, block>>>(d_dst, d_col, d_det, d_img, n_rows, n_imagebin);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms_out) *ms_out = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err == cudaSuccess) err = cudaGetLastError();
    return (int)err;
}

extern "C" int ref_cuda_PESysMatGen(float* col, float* det, float* img, float* dst, int cuda_id) {
    return PESysMatGen(col, det, img, dst, cuda_id);
}
