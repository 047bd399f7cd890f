// Scatter surrogate: physics baseline (anchor-interpolated transfer x PE on the
// tensor cores), learned correction (coordinate MLP), exact verification and
// recompute.  Internal declarations shared by the surrogate sources.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "sysmat_b200.h"

namespace smb {

// ---- anchor grid ------------------------------------------------------------------
// Per axis k anchors at c_i = (i + 0.5) n / k - 0.5.  A voxel coordinate x lies
// in slab j (0..k): between anchors lo = max(j - 1, 0) and hi = min(j, k - 1)
// with weight t on hi and 1 - t on lo (t = 0 when lo == hi, outside the
// first / last centre).  AxisTable holds that per coordinate.
struct AxisTable {
    std::vector<int> lo, hi;
    std::vector<float> t;
    std::vector<int> slab;      // slab of each coordinate
    std::vector<int> first, count;   // per anchor: coordinates where it carries weight
    int k = 1;
};
AxisTable make_axis(int n, int k);

// A cell: the voxels of one slab per axis (a box), with up to 8 corner anchors.
struct BaseCell {
    int x0, y0, z0;             // box origin (voxel indices)
    int nx, ny, nz;             // box size
    int n_seg;                  // distinct corner anchors (1, 2, 4 or 8)
    int anchor[8];              // anchor index a = (ix * ky + iy) * kz + iz
    int side[8];                // bits 0-2: hi anchor on x, y, z; bits 4-6: that axis has two anchors
};

// PE [N][ld_pe] fp32 -> PEt [V][N] bf16 (voxel-major, source contiguous).
cudaError_t launch_pe_transpose(const float* pe, int64_t ld_pe, int N, int64_t V, __nv_bfloat16* pet, cudaStream_t s);

// For every source s and anchor a: the PE-weighted centroid (fractional voxel
// indices) of the source's voxels under anchor a's trilinear weight;
// vbar[a * N + s] = (x, y, z, 1) or (0, 0, 0, 0) where the weight sums to 0.
// d_box: per axis and anchor the [first, count] coordinates of its support.
cudaError_t launch_anchor_centroids(const float* pe, int64_t ld_pe, int N, int nx, int ny, int nz, const int* d_lo,
                                    const int* d_hi, const float* d_t, const int* d_box, int kx, int ky, int kz,
                                    float4* vbar, cudaStream_t s);

// dst[d * ld + v] = sum over the cell's corner anchors a of w_a(v) * sum_s K[a][r][s] PEt[v][s]
// for every cell and K row r < N, d = row_map[r] (r when null).  K bf16 [A][N][N].
struct BaseItem {
    int cell;                   // index into the cell array
    int n0;                     // first voxel (cell-local) of this item's column tile
};
cudaError_t launch_baseline_gemm(const __nv_bfloat16* K, const __nv_bfloat16* pet, int N, int nx, int ny,
                                 const BaseCell* cells, const BaseItem* items, int n_items, const float* tx,
                                 const float* ty, const float* tz, const int* row_map, float* dst, int64_t ld,
                                 int* error, cudaStream_t s);

// dst[r][c * ny + y] <-> full[r][voxel(cols[c], y)] for rows r < N.
cudaError_t launch_gather_columns(const float* full, int64_t ld_full, int N, const int2* cols, int n_cols, int nx,
                                  int ny, float* out, int64_t ld_out, cudaStream_t s);
cudaError_t launch_scatter_columns(const float* sub, int64_t ld_sub, int N, const int2* cols, int n_cols, int nx,
                                   int ny, float* full, int64_t ld_full, cudaStream_t s);

// Per-row squared error and squared norm over a column block:
// err2[r] = sum_j (pred[r][j] - ref[r][j])^2, norm2[r] = sum_j ref[r][j]^2 (double).
cudaError_t launch_row_error(const float* pred, int64_t ld_pred, const float* ref, int64_t ld_ref, int N, int n,
                             double* err2, double* norm2, cudaStream_t s);

// rho[d][j] = log(Y / B), wgt[d][j] = Y^2 / (norm2[d] / n) where Y, B > 0 (else 0), j < n.
cudaError_t launch_prep_targets(const float* Y, const float* Bm, int64_t ld, int N, int n, const double* norm2, float* rho,
                                float* wgt, int64_t ld_out, cudaStream_t s);
// Batch j: col[j] = fit[hash(seed, step, j) mod n_fit], vox[j] = col_vox[col[j]].
cudaError_t launch_sample_batch(uint64_t seed, int step, int B, const int* fit, int n_fit, const int* col_vox, int* col,
                                int* vox, cudaStream_t s);
// out[d][j] = in[d][idx[j]], j < n.
cudaError_t launch_gather_idx(const float* in, int64_t ld_in, int N, const int* idx, int n, float* out, int64_t ld_out,
                              cudaStream_t s);

// ---- the learned correction ---------------------------------------------------------
// rho(d, v) = g(d) . h(v): trunk h = MLP over Fourier features of the voxel
// centre (sin, cos of w_j c per axis, w_j = pi/2 min(n/2, 8)^(j / (F - 1)), c in
// [-1, 1]), `layers` linear layers of `width` with SiLU between them; crystal
// branch g(d) = P e_d + b_P.  Parameters are fp32 masters with bf16 copies.
struct NetShape {
    int layers = 6, width = 256, freqs = 16, emb = 64;
    int n_crystals = 0, nx = 0, ny = 0, nz = 0;
    int in_dim(int l) const { return l == 0 ? 6 * freqs : width; }
};

class SurrogateNet {
public:
    NetShape shape;
    // parameter blocks: for l < layers: W_l [width][in_l], b_l [width]; then E [N][emb], P [width][emb], b_P [width]
    std::vector<int64_t> off, len;
    int64_t n_params = 0;
    float* w = nullptr;             // fp32 masters
    float* grad = nullptr;
    float* m1 = nullptr;
    float* m2 = nullptr;
    __nv_bfloat16* wb = nullptr;    // bf16 copies
    int* error = nullptr;           // GEMM bounded-wait flag
    double* loss = nullptr;
    int step = 0;

    int init(const NetShape& s, uint64_t seed, cudaStream_t st);
    void release();
    int set_params(const float* host, cudaStream_t st);
    // One forward + backward over batch voxels vox[0..B) against targets
    // rho[d][col[j]], weights wgt[d][col[j]] (row pitch ld); gradients into
    // `grad`; loss = sum w (pred - rho)^2 / (N B) accumulated into *loss.
    int forward_backward(const int* vox, const int* col, int B, const float* rho, const float* wgt, int64_t ld,
                         cudaStream_t st);
    int adam(float lr, cudaStream_t st);
    // out[d][j] = rho(d, vox[j]) for j < n (row pitch ld), or with epilogue 1:
    // out[d][j] *= exp(gate[d] * rho(d, vox[j])).  vox null: voxels 0..n-1.
    int predict(const int* vox, int n, float* out, int64_t ld, const float* gate, cudaStream_t st);
    ~SurrogateNet() { release(); }

private:
    int reserve(int rows, cudaStream_t st);
    int trunk_forward(const int* vox, int rows, bool keep_t, cudaStream_t st);
    int crystal_forward(bool keep_t, cudaStream_t st);
    int transpose_weights(cudaStream_t st);
    int gemm(int m, int n, int k, const __nv_bfloat16* a, int64_t ams, const __nv_bfloat16* b, int64_t bns, float* c,
             int64_t ldc, const float* bias, const float* row_scale, int epilogue, cudaStream_t st);
    __nv_bfloat16* wbt = nullptr;   // transposed bf16 copies of W_l [in][width], E [emb][N], P [emb][width]
    void* ws = nullptr;
    int ws_rows = 0;
    int64_t o[24] = {};             // workspace slices (bytes)
};

}  // namespace smb
