// The scatter surrogate's learned correction: a coordinate MLP trained and run
// on the sm_100a tensor cores.
//
// rho(d, v) = g(d) . h(v) with
//   h(v) = trunk over Fourier features of the voxel centre: 6 F inputs
//          (sin, cos of w_j c, c in [-1, 1] per axis, w_j = pi/2 r^(j/(F-1)),
//          r = min(n/2, 8): the highest frequency spans a quarter of the
//          field, so the learned correction stays smooth between the sparse
//          training columns instead of inventing detail there),
//          `layers` linear layers of `width` with SiLU between them (the last
//          one linear);
//   g(d) = P e_d + b_P, e_d the crystal's learned `emb`-dimensional embedding.
// Every product (trunk layers forward and backward, the crystal projection and
// its gradients, the bilinear head and its gradients, inference over all
// voxels) is the BF16 tcgen05 GEMM of gemm_tc.cu with FP32 accumulation.  All
// GEMM operands are K-major: the kernels below also write the transposed bf16
// copies the backward products read.  Weights are fp32 masters with bf16
// copies, updated by Adam.
#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.h"
#include "gemm_tc.h"
#include "surrogate.h"

namespace smb {
namespace {

constexpr int kEw = 256;

int blocks_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + kEw - 1) / kEw, 148LL * 16)); }
int n_tile_for(int n) { return n >= 192 ? 256 : (n > 64 ? 128 : 64); }

// out [n][6F] and, when set, outT [6F][n]
__global__ void fourier_kernel(const int* __restrict__ vox, int n, int nx, int ny, int nz, int F,
                               __nv_bfloat16* __restrict__ out, __nv_bfloat16* __restrict__ outT) {
    const int dim = 6 * F;
    const long long total = (long long)n * dim;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / dim), f = (int)(i - (long long)r * dim);
        const int v = vox[r];
        const int axis = f / (2 * F), rem = f - axis * 2 * F, j = rem >> 1;
        const int ix = v % nx, iy = (v / nx) % ny, iz = v / (nx * ny);
        const int idx = axis == 0 ? ix : (axis == 1 ? iy : iz);
        const int nn = axis == 0 ? nx : (axis == 1 ? ny : nz);
        const float c = 2.0f * ((float)idx + 0.5f) / (float)nn - 1.0f;
        const float w = 1.57079632679489662f * powf(fminf(0.5f * (float)nn, 8.0f), F > 1 ? (float)j / (float)(F - 1) : 0.0f);
        const float a = c * w;
        const __nv_bfloat16 q = __float2bfloat16((rem & 1) ? cosf(a) : sinf(a));
        out[i] = q;
        if (outT) outT[(long long)f * n + r] = q;
    }
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }

// Tiled [R][C] fp32 -> bf16 (optional, same layout) and bf16 transposed [C][R]
// (optional), with an optional SiLU applied first.
__global__ void convert_kernel(const float* __restrict__ x, int R, int C, int act, __nv_bfloat16* __restrict__ y,
                               __nv_bfloat16* __restrict__ yt) {
    __shared__ float tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        float v = 0.0f;
        if (r < R && c < C) {
            v = x[(long long)r * C + c];
            if (act) v = silu(v);
            if (y) y[(long long)r * C + c] = __float2bfloat16(v);
        }
        tile[i][threadIdx.x] = v;
    }
    if (!yt) return;
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (r < R && c < C) yt[(long long)c * R + r] = __float2bfloat16(tile[threadIdx.x][i]);
    }
}

// dz = da * silu'(z) (in place into da's slot `dz`)
__global__ void silu_bwd_kernel(const float* __restrict__ da, const float* __restrict__ z, long long n,
                                float* __restrict__ dz) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float s = 1.0f / (1.0f + __expf(-z[i]));
        dz[i] = da[i] * s * (1.0f + z[i] * (1.0f - s));
    }
}

// r = yhat - rho, loss += w r^2, dY = 2 w r / (N B): bf16 [N][B] and transposed [B][N]
__global__ void residual_kernel(const float* __restrict__ yhat, const float* __restrict__ rho,
                                const float* __restrict__ wgt, long long ld, const int* __restrict__ col, int N, int B,
                                float inv_count, __nv_bfloat16* __restrict__ dy, __nv_bfloat16* __restrict__ dyt,
                                double* __restrict__ loss) {
    __shared__ double part[kEw / 32];
    double acc = 0.0;
    const long long total = (long long)N * B;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int d = (int)(i / B), j = (int)(i - (long long)d * B);
        const long long src = (long long)d * ld + col[j];
        const float w = wgt[src];
        const float r = yhat[i] - rho[src];
        acc += (double)w * r * r;
        const __nv_bfloat16 g = __float2bfloat16(2.0f * w * r * inv_count);
        dy[i] = g;
        dyt[(long long)j * N + d] = g;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kEw / 32; ++w) s += part[w];
        atomicAdd(loss, s * (double)inv_count);
    }
}

// out[c] = sum_r x[r][c]
__global__ void colsum_kernel(const float* __restrict__ x, int rows, int cols, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (int r = 0; r < rows; ++r) s += x[(long long)r * cols + c];
    out[c] = s;
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                            float c2, __nv_bfloat16* __restrict__ wb) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        w[i] = wi;
        wb[i] = __float2bfloat16(wi);
    }
}

__global__ void to_bf16_kernel(const float* __restrict__ x, long long n, __nv_bfloat16* __restrict__ y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16(x[i]);
}

__global__ void iota_kernel(int base, int n, int* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = base + i;
}

cudaError_t convert(const float* x, int R, int C, int act, __nv_bfloat16* y, __nv_bfloat16* yt, cudaStream_t s) {
    dim3 grid((C + 31) / 32, (R + 31) / 32);
    convert_kernel<<<grid, dim3(32, 8), 0, s>>>(x, R, C, act, y, yt);
    return cudaGetLastError();
}

// workspace slice indices
enum {
    W_X0, W_X0T, W_Z, W_A, W_AT, W_DZ, W_DZB, W_DZT, W_DA, W_G, W_GB, W_GT, W_DG, W_DGB, W_DGT, W_YHAT, W_DY, W_DYT,
    W_VOX, W_END
};

}  // namespace

int SurrogateNet::init(const NetShape& s, uint64_t seed, cudaStream_t st) {
    release();
    shape = s;
    off.clear();
    len.clear();
    int64_t at = 0;
    auto add = [&](int64_t n) {
        off.push_back(at);
        len.push_back(n);
        at += (n + 63) / 64 * 64;
    };
    for (int l = 0; l < s.layers; ++l) {
        add((int64_t)s.width * s.in_dim(l));
        add(s.width);
    }
    add((int64_t)s.n_crystals * s.emb);
    add((int64_t)s.width * s.emb);
    add(s.width);
    n_params = at;
    SM_CUDA(cudaMalloc(&w, sizeof(float) * n_params));
    SM_CUDA(cudaMalloc(&grad, sizeof(float) * n_params));
    SM_CUDA(cudaMalloc(&m1, sizeof(float) * n_params));
    SM_CUDA(cudaMalloc(&m2, sizeof(float) * n_params));
    SM_CUDA(cudaMalloc(&wb, sizeof(__nv_bfloat16) * n_params));
    SM_CUDA(cudaMalloc(&wbt, sizeof(__nv_bfloat16) * n_params));
    SM_CUDA(cudaMalloc(&loss, sizeof(double)));
    SM_CUDA(cudaMalloc(&error, sizeof(int)));
    SM_CUDA(cudaMemsetAsync(grad, 0, sizeof(float) * n_params, st));
    SM_CUDA(cudaMemsetAsync(error, 0, sizeof(int), st));
    SM_CUDA(cudaMemsetAsync(loss, 0, sizeof(double), st));
    // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases, N(0, 1/emb)
    // embeddings; the projection P starts at zero so the correction starts at 0
    std::vector<float> h((size_t)n_params, 0.0f);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<float> U(-1.0f, 1.0f);
    std::normal_distribution<float> Nd(0.0f, 1.0f);
    for (int l = 0; l < s.layers; ++l) {
        const float a = 1.0f / std::sqrt((float)s.in_dim(l));
        for (int64_t i = 0; i < len[2 * l]; ++i) h[off[2 * l] + i] = U(rng) * a;
    }
    for (int64_t i = 0; i < len[2 * s.layers]; ++i) h[off[2 * s.layers] + i] = Nd(rng) / std::sqrt((float)s.emb);
    return set_params(h.data(), st);
}

void SurrogateNet::release() {
    for (void* p : {(void*)w, (void*)grad, (void*)m1, (void*)m2, (void*)wb, (void*)wbt, (void*)loss, (void*)error, ws})
        if (p) cudaFree(p);
    w = grad = m1 = m2 = nullptr;
    wb = wbt = nullptr;
    loss = nullptr;
    error = nullptr;
    ws = nullptr;
    ws_rows = 0;
}

int SurrogateNet::set_params(const float* host, cudaStream_t st) {
    SM_CUDA(cudaMemcpyAsync(w, host, sizeof(float) * n_params, cudaMemcpyHostToDevice, st));
    to_bf16_kernel<<<blocks_for(n_params), kEw, 0, st>>>(w, n_params, wb);
    SM_CUDA(cudaGetLastError());
    SM_CUDA(cudaMemsetAsync(m1, 0, sizeof(float) * n_params, st));
    SM_CUDA(cudaMemsetAsync(m2, 0, sizeof(float) * n_params, st));
    step = 0;
    SM_CUDA(cudaStreamSynchronize(st));   // `host` may be released on return
    return transpose_weights(st);
}

int SurrogateNet::transpose_weights(cudaStream_t st) {
    const NetShape& s = shape;
    for (int l = 0; l < s.layers; ++l)
        SM_CUDA(convert(w + off[2 * l], s.width, s.in_dim(l), 0, nullptr, wbt + off[2 * l], st));
    SM_CUDA(convert(w + off[2 * s.layers], s.n_crystals, s.emb, 0, nullptr, wbt + off[2 * s.layers], st));
    SM_CUDA(convert(w + off[2 * s.layers + 1], s.width, s.emb, 0, nullptr, wbt + off[2 * s.layers + 1], st));
    return SM_OK;
}

int SurrogateNet::reserve(int rows, cudaStream_t st) {
    (void)st;
    if (rows <= ws_rows) return SM_OK;
    if (ws) cudaFree(ws);
    ws = nullptr;
    ws_rows = rows;
    const int64_t R = rows, Wd = shape.width, F = shape.in_dim(0), N = shape.n_crystals, L = shape.layers;
    const int64_t sz[W_END] = {
        R * F * 2, R * F * 2,                     // X0, X0T
        L * R * Wd * 4, L * R * Wd * 2, L * R * Wd * 2,   // Z, A, AT (per layer)
        R * Wd * 4, R * Wd * 2, R * Wd * 2, R * Wd * 4,   // DZ, DZB, DZT, DA
        N * Wd * 4, N * Wd * 2, N * Wd * 2,       // G, GB, GT
        N * Wd * 4, N * Wd * 2, N * Wd * 2,       // DG, DGB, DGT
        N * R * 4, N * R * 2, N * R * 2,          // YHAT, DY, DYT
        R * 4};                                   // VOX
    int64_t at = 0;
    for (int i = 0; i < W_END; ++i) {
        o[i] = at;
        at += (sz[i] + 255) / 256 * 256;
    }
    SM_CUDA(cudaMalloc(&ws, at));
    return SM_OK;
}

int SurrogateNet::gemm(int m, int n, int k, const __nv_bfloat16* a, int64_t ams, const __nv_bfloat16* b, int64_t bns,
                       float* c, int64_t ldc, const float* bias, const float* row_scale, int epilogue, cudaStream_t st) {
    GemmArgs g{};
    g.m = m;
    g.n = n;
    g.k = k;
    g.a = a;
    g.a_ms = ams;
    g.a_ks = 1;
    g.b = b;
    g.b_ns = bns;
    g.b_ks = 1;
    g.c = c;
    g.ldc = ldc;
    g.alpha = 1.0f;
    g.row_scale = row_scale;
    g.bias = bias;
    g.accumulate = 0;
    g.epilogue = epilogue;
    g.n_tile = n_tile_for(n);
    g.error = error;
    SM_CUDA(gemm_bf16_tc(g, st));
    return SM_OK;
}

#define WS(T, i) reinterpret_cast<T*>(static_cast<unsigned char*>(ws) + o[i])

int SurrogateNet::trunk_forward(const int* vox, int rows, bool keep_t, cudaStream_t st) {
    const NetShape& s = shape;
    const int64_t R = rows, Wd = s.width;
    fourier_kernel<<<blocks_for(R * s.in_dim(0)), kEw, 0, st>>>(vox, rows, s.nx, s.ny, s.nz, s.freqs, WS(__nv_bfloat16, W_X0),
                                                                 keep_t ? WS(__nv_bfloat16, W_X0T) : nullptr);
    SM_CUDA(cudaGetLastError());
    for (int l = 0; l < s.layers; ++l) {
        const __nv_bfloat16* in = l == 0 ? WS(__nv_bfloat16, W_X0) : WS(__nv_bfloat16, W_A) + (l - 1) * R * Wd;
        float* z = WS(float, W_Z) + l * R * Wd;
        SM_TRY(gemm(rows, s.width, s.in_dim(l), in, s.in_dim(l), wb + off[2 * l], s.in_dim(l), z, s.width,
                    w + off[2 * l + 1], nullptr, 0, st));
        SM_CUDA(convert(z, rows, s.width, l + 1 < s.layers ? 1 : 0, WS(__nv_bfloat16, W_A) + l * R * Wd,
                        keep_t ? WS(__nv_bfloat16, W_AT) + l * R * Wd : nullptr, st));
    }
    return SM_OK;
}

int SurrogateNet::crystal_forward(bool keep_t, cudaStream_t st) {
    const NetShape& s = shape;
    const int64_t oE = off[2 * s.layers], oP = off[2 * s.layers + 1], obP = off[2 * s.layers + 2];
    SM_TRY(gemm(s.n_crystals, s.width, s.emb, wb + oE, s.emb, wb + oP, s.emb, WS(float, W_G), s.width, w + obP, nullptr,
                0, st));
    SM_CUDA(convert(WS(float, W_G), s.n_crystals, s.width, 0, WS(__nv_bfloat16, W_GB),
                    keep_t ? WS(__nv_bfloat16, W_GT) : nullptr, st));
    return SM_OK;
}

int SurrogateNet::forward_backward(const int* vox, const int* col, int B, const float* rho, const float* wgt, int64_t ld,
                                   cudaStream_t st) {
    const NetShape& s = shape;
    const int N = s.n_crystals, Wd = s.width, L = s.layers;
    SM_TRY(reserve(B, st));
    const int64_t R = B;
    SM_TRY(trunk_forward(vox, B, true, st));
    SM_TRY(crystal_forward(true, st));
    const __nv_bfloat16* H = WS(__nv_bfloat16, W_A) + (L - 1) * R * Wd;
    const __nv_bfloat16* HT = WS(__nv_bfloat16, W_AT) + (L - 1) * R * Wd;
    // head: Yhat[d][j] = G[d] . H[j]
    SM_TRY(gemm(N, B, Wd, WS(__nv_bfloat16, W_GB), Wd, H, Wd, WS(float, W_YHAT), B, nullptr, nullptr, 0, st));
    residual_kernel<<<blocks_for((int64_t)N * B), kEw, 0, st>>>(WS(float, W_YHAT), rho, wgt, ld, col, N, B,
                                                                 1.0f / ((float)N * (float)B), WS(__nv_bfloat16, W_DY),
                                                                 WS(__nv_bfloat16, W_DYT), loss);
    SM_CUDA(cudaGetLastError());
    // dG[d][w] = sum_j dY[d][j] H[j][w];  dH[j][w] = sum_d dY[d][j] G[d][w]
    SM_TRY(gemm(N, Wd, B, WS(__nv_bfloat16, W_DY), B, HT, B, WS(float, W_DG), Wd, nullptr, nullptr, 0, st));
    SM_TRY(gemm(B, Wd, N, WS(__nv_bfloat16, W_DYT), N, WS(__nv_bfloat16, W_GT), N, WS(float, W_DZ), Wd, nullptr, nullptr,
                0, st));
    SM_CUDA(convert(WS(float, W_DG), N, Wd, 0, WS(__nv_bfloat16, W_DGB), WS(__nv_bfloat16, W_DGT), st));
    // crystal branch: dP[w][e] = sum_d dG[d][w] E[d][e]; db_P = colsum dG; dE[d][e] = sum_w dG[d][w] P[w][e]
    const int64_t oE = off[2 * L], oP = off[2 * L + 1], obP = off[2 * L + 2];
    SM_TRY(gemm(Wd, s.emb, N, WS(__nv_bfloat16, W_DGT), N, wbt + oE, N, grad + oP, s.emb, nullptr, nullptr, 0, st));
    colsum_kernel<<<(Wd + kEw - 1) / kEw, kEw, 0, st>>>(WS(float, W_DG), N, Wd, grad + obP);
    SM_TRY(gemm(N, s.emb, Wd, WS(__nv_bfloat16, W_DGB), Wd, wbt + oP, Wd, grad + oE, s.emb, nullptr, nullptr, 0, st));
    // trunk, last layer first; dZ_{L-1} = dH (no activation on the last layer)
    float* dz = WS(float, W_DZ);
    for (int l = L - 1; l >= 0; --l) {
        const int fin = s.in_dim(l);
        SM_CUDA(convert(dz, B, Wd, 0, WS(__nv_bfloat16, W_DZB), WS(__nv_bfloat16, W_DZT), st));
        const __nv_bfloat16* inT = l == 0 ? WS(__nv_bfloat16, W_X0T) : WS(__nv_bfloat16, W_AT) + (l - 1) * R * Wd;
        // dW[o][i] = sum_j dZ[j][o] In[j][i]
        SM_TRY(gemm(Wd, fin, B, WS(__nv_bfloat16, W_DZT), B, inT, B, grad + off[2 * l], fin, nullptr, nullptr, 0, st));
        colsum_kernel<<<(Wd + kEw - 1) / kEw, kEw, 0, st>>>(dz, B, Wd, grad + off[2 * l + 1]);
        SM_CUDA(cudaGetLastError());
        if (l > 0) {
            // dA[j][i] = sum_o dZ[j][o] W[o][i]; dZ_{l-1} = dA * silu'(Z_{l-1})
            SM_TRY(gemm(B, fin, Wd, WS(__nv_bfloat16, W_DZB), Wd, wbt + off[2 * l], Wd, WS(float, W_DA), fin, nullptr,
                        nullptr, 0, st));
            silu_bwd_kernel<<<blocks_for(R * fin), kEw, 0, st>>>(WS(float, W_DA), WS(float, W_Z) + (l - 1) * R * Wd,
                                                                  R * fin, dz);
            SM_CUDA(cudaGetLastError());
        }
    }
    return SM_OK;
}

int SurrogateNet::adam(float lr, cudaStream_t st) {
    ++step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f / (1.0f - std::pow(b1, (float)step)), c2 = 1.0f / (1.0f - std::pow(b2, (float)step));
    adam_kernel<<<blocks_for(n_params), kEw, 0, st>>>(w, grad, m1, m2, n_params, lr, b1, b2, 1e-8f, c1, c2, wb);
    SM_CUDA(cudaGetLastError());
    return transpose_weights(st);
}

int SurrogateNet::predict(const int* vox, int n, float* out, int64_t ld, const float* gate, cudaStream_t st) {
    const NetShape& s = shape;
    const int chunk = 8192;
    SM_TRY(reserve(std::min(n, chunk), st));
    SM_TRY(crystal_forward(false, st));
    int* ids = WS(int, W_VOX);
    const int64_t Wd = s.width;
    for (int c0 = 0; c0 < n; c0 += chunk) {
        const int rows = std::min(chunk, n - c0);
        if (vox) SM_CUDA(cudaMemcpyAsync(ids, vox + c0, sizeof(int) * rows, cudaMemcpyDeviceToDevice, st));
        else {
            iota_kernel<<<(rows + kEw - 1) / kEw, kEw, 0, st>>>(c0, rows, ids);
            SM_CUDA(cudaGetLastError());
        }
        SM_TRY(trunk_forward(ids, rows, false, st));
        const __nv_bfloat16* H = WS(__nv_bfloat16, W_A) + (int64_t)(s.layers - 1) * rows * Wd;
        SM_TRY(gemm(s.n_crystals, rows, s.width, WS(__nv_bfloat16, W_GB), s.width, H, s.width, out + c0, ld, nullptr, gate,
                    gate ? 1 : 0, st));
    }
    return SM_OK;
}

#undef WS

}  // namespace smb
