// Primary-Compton scatter kernels for sm_100a (see scatter.h for the split).
//
// Physics per (detector d, voxel I, scatter point S), as the reference's
// crystalScatterSysMatCuda / collimatorScatterSysMatCuda
// (ScatterGen_RayTracing_CircularHole/scatter.cu:1077-1437, :1544-1936):
//   W(S, I) * RangePhi / 2pi * KNfraction(theta_min, theta_max) * P_window(E')
//     * exp(-sum_k mu_k(E') L_k - mu_d(E') L_self) * (1 - exp(-mu_d(E') L_abs)) mu_pe,d(E') / mu_d(E')
// with E' = E0 / (1 + alpha (1 - cos theta)), theta the angle at S between
// I -> S and S -> D, mu_pe(E') = mu_pe (E0/E')^3, mu_c(E') = mu_c E0/E'.
// W is PE[s, I] mu_c,d / mu_pe,d (crystal scatter) or the virtual solid angle
// of the hole times mu_c / mu_t of plate 0 (collimator scatter).
//
// Differences in arithmetic (not in the quantities): the cosine and sine of
// the scatter angle come from a dot and a cross product instead of
// cos(acos(.)), the polar range from atan2 of the extreme unit-box corners
// instead of eight acos, and the reference's 0.01 rad rectangle sum of the
// Klein-Nishina integrand (up to 315 terms) from a closed form: the
// Euler-Maclaurin formula with the exact integral (a Taylor table of
// g = KN sin theta, built in double on the host) and its first two
// correction terms, whose remainder is below 1e-10.
#include <algorithm>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "scatter.h"
#include "scatter_term.cuh"
#include "tracer.cuh"

namespace smb {
namespace {


// ---- bitmaps (scatter.cu:1440-1540, :1939-2009) ------------------------------
// Single-precision expressions in the reference's order; this translation
// unit is compiled without fused multiply-add, so every bit matches.
__device__ __forceinline__ float dist3(float x1, float y1, float z1, float x2, float y2, float z2) {
    return sqrtf((x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2) + (z1 - z2) * (z1 - z2));
}

__device__ bool crystal_bit(const float4* cr, int i, int j, int k) {
    const float4 a = cr[i], b = cr[j], c = cr[k];
    const float Lij = dist3(a.x, a.y, a.z, b.x, b.y, b.z);
    const float crit_ij = a.w / Lij, crit_ji = b.w / Lij;
    const float ex_ij = (a.x - b.x) / Lij, ey_ij = (a.y - b.y) / Lij, ez_ij = (a.z - b.z) / Lij;
    const float ex_ji = (b.x - a.x) / Lij, ey_ji = (b.y - a.y) / Lij, ez_ji = (b.z - a.z) / Lij;
    const float Lik = dist3(c.x, c.y, c.z, a.x, a.y, a.z);
    const float crit_ki = c.w / Lik;
    const float Ljk = dist3(c.x, c.y, c.z, b.x, b.y, b.z);
    const float crit_kj = c.w / Ljk;
    const float ex_ki = (c.x - a.x) / Lik, ey_ki = (c.y - a.y) / Lik, ez_ki = (c.z - a.z) / Lik;
    const float ex_kj = (c.x - b.x) / Ljk, ey_kj = (c.y - b.y) / Ljk, ez_kj = (c.z - b.z) / Ljk;
    if (dist3(ex_ki, ey_ki, ez_ki, ex_ji, ey_ji, ez_ji) <= crit_ki + crit_ji) return true;
    return dist3(ex_kj, ey_kj, ez_kj, ex_ij, ey_ij, ez_ij) <= crit_kj + crit_ij;
}

__device__ bool collimator_bit(const float4* cr, const float4* hr, int i, int j, int k) {
    const float4 h = hr[i], b = cr[j], c = cr[k];
    const float Lij = dist3(h.x, h.y, h.z, b.x, b.y, b.z);
    const float crit_ji = b.w / Lij;
    const float ex_ji = (b.x - h.x) / Lij, ey_ji = (b.y - h.y) / Lij, ez_ji = (b.z - h.z) / Lij;
    const float Lik = dist3(c.x, c.y, c.z, h.x, h.y, h.z);
    const float crit_ki = c.w / Lik;
    const float ex_ki = (c.x - h.x) / Lik, ey_ki = (c.y - h.y) / Lik, ez_ki = (c.z - h.z) / Lik;
    return dist3(ex_ki, ey_ki, ez_ki, ex_ji, ey_ji, ez_ji) <= crit_ki + crit_ji;
}

// Pair index (i <= j) -> i: the largest i with i*N - i*(i-1)/2 <= pair.
__device__ __forceinline__ int pair_row(long long pair, int N) {
    const double b = 2.0 * N + 1.0;
    int i = (int)((b - sqrt(b * b - 8.0 * (double)pair)) * 0.5);
    if (i < 0) i = 0;
    auto start = [N](long long r) { return r * N - r * (r - 1) / 2; };
    while (i > 0 && start(i) > pair) --i;
    while (i + 1 < N && start(i + 1) <= pair) ++i;
    return i;
}

// One thread per 32-bit word: bits bit0 .. bit0 + 31 of the pair-major bitmap
// bit = (i N - i (i + 1) / 2 + j) N + k, i <= j; set for i < j, k != i, j.
__global__ void bitmap_crystal_kernel(uint32_t* words, long long n_words, ScatterTables T) {
    const int N = T.n_crystals;
    const long long total = ((long long)N * (N + 1) / 2) * N;
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n_words;
         w += (long long)gridDim.x * blockDim.x) {
        const long long bit0 = w * 32;
        long long pair = bit0 / N;
        int k = (int)(bit0 - pair * N);
        int i = pair_row(pair, N);
        int j = (int)(pair - ((long long)i * N - (long long)i * (i - 1) / 2)) + i;
        uint32_t word = 0u;
        for (int b = 0; b < 32 && bit0 + b < total; ++b) {
            if (i < j && k != i && k != j && crystal_bit(T.crystal_raw, i, j, k)) word |= 1u << b;
            if (++k == N) {
                k = 0;
                if (++j == N) {
                    ++i;
                    j = i;
                }
            }
        }
        words[w] = word;
    }
}

// bit = i N^2 + j N + k for layer-0 hole i, crystals j, k.
__global__ void bitmap_collimator_kernel(uint32_t* words, long long n_words, ScatterTables T) {
    const int N = T.n_crystals;
    const long long total = (long long)T.n_holes0 * N * N;
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n_words;
         w += (long long)gridDim.x * blockDim.x) {
        const long long bit0 = w * 32;
        int i = (int)(bit0 / ((long long)N * N));
        long long rem = bit0 - (long long)i * N * N;
        int j = (int)(rem / N);
        int k = (int)(rem - (long long)j * N);
        uint32_t word = 0u;
        for (int b = 0; b < 32 && bit0 + b < total; ++b) {
            if (collimator_bit(T.crystal_raw, T.hole_raw, i, j, k)) word |= 1u << b;
            if (++k == N) {
                k = 0;
                if (++j == N) {
                    j = 0;
                    ++i;
                }
            }
        }
        words[w] = word;
    }
}

// ---- per (scatter point, detector) ---------------------------------------------
// sum_k L_k mu_pe_k, sum_k L_k mu_c_k over the crystals k the bitmap flags for
// the pair (scatter.cu:1309-1367, :1832-1889), the path inside the detecting
// crystal before its unit (:1371-1382), and the absorption chord (:1385-1392).
// The detector unit is the whole crystal (the reference's divide = 1), whose
// centre is the crystal centre.
template <int KIND>
__global__ void scatter_pair_kernel(DevGeometry G, ScatterTables T, const uint32_t* __restrict__ bitmap,
                                    const int* __restrict__ perm, int r0, int r1, float4* __restrict__ pair,
                                    int n_sources) {
    const int N = T.n_crystals;
    const int r = r0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= r1) return;
    const int d = perm[r];
    const long long ld = r1 - r0;
    const float4 Dp = G.c.pos[d], Dsz = G.c.size[d], Dr = G.c.rot[d];
    for (int q = blockIdx.y; q < n_sources; q += gridDim.y) {
        float4 S;
        int s;
        if (KIND == kScatterCrystal) {
            S = T.crystal_src[q];
            s = q / T.n_points;
        } else {
            S = T.hole_src[q];
            s = q;
        }
        float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (!(KIND == kScatterCrystal && s == d)) {
            float a_pe = 0.0f, a_c = 0.0f;
            long long base;
            if (KIND == kScatterCrystal) {
                const int lo = s < d ? s : d, hi = s < d ? d : s;
                base = ((long long)lo * N - (long long)lo * (lo + 1) / 2 + hi) * N;
            } else {
                base = ((long long)s * N + d) * N;
            }
            const long long w_end = (base + N - 1) >> 5;
            for (long long wi = base >> 5; wi <= w_end; ++wi) {
                uint32_t bits = __ldg(bitmap + wi);
                const long long first = wi << 5;
                if (first < base) bits &= ~0u << (int)(base - first);
                if (first + 31 > base + N - 1) {
                    const int keep = (int)(base + N - first);
                    bits &= keep >= 32 ? ~0u : ((1u << keep) - 1u);
                }
                while (bits) {
                    const int b = __ffs(bits) - 1;
                    bits &= bits - 1u;
                    const int k = (int)(first + b - base);
                    if (k == d || (KIND == kScatterCrystal && k == s)) continue;
                    const float4 kp = G.c.pos[k], ks = G.c.size[k], kr = G.c.rot[k], kph = G.c.phys[k];
                    const float xa = (S.x - kp.x) * kr.x - (S.z - kp.z) * kr.y;
                    const float ya = S.y - kp.y;
                    const float za = (S.x - kp.x) * kr.y + (S.z - kp.z) * kr.x;
                    const float xb = (Dp.x - kp.x) * kr.x - (Dp.z - kp.z) * kr.y;
                    const float yb = Dp.y - kp.y;
                    const float zb = (Dp.x - kp.x) * kr.y + (Dp.z - kp.z) * kr.x;
                    const Box3 kb{-0.5f * ks.x, -0.5f * ks.y, -0.5f * ks.z, 0.5f * ks.x, 0.5f * ks.y, 0.5f * ks.z};
                    const float len = chord_through(xa, ya, za, xb, yb, zb, kb);
                    a_pe += len * kph.x;
                    a_c += len * kph.y;
                }
            }
            // scatter point in the detecting crystal's frame
            const float xs = (S.x - Dp.x) * Dr.x - (S.z - Dp.z) * Dr.y;
            const float ys = S.y - Dp.y;
            const float zs = (S.x - Dp.x) * Dr.y + (S.z - Dp.z) * Dr.x;
            const Box3 cb{-Dsz.x / 2.0f, -Dsz.y / 2.0f, -Dsz.z / 2.0f, Dsz.x / 2.0f, Dsz.y / 2.0f, Dsz.z / 2.0f};
            const Box3 ub{-0.5f * Dsz.x, -0.5f * Dsz.y, -0.5f * Dsz.z, 0.5f * Dsz.x, 0.5f * Dsz.y, 0.5f * Dsz.z};
            const float l1 = chord_to_end(xs, ys, zs, 0.0f, 0.0f, 0.0f, cb);
            const float l2 = chord_to_end(xs, ys, zs, 0.0f, 0.0f, 0.0f, ub);
            const float L = dist3(S.x, S.y, S.z, Dp.x, Dp.y, Dp.z);
            const float xt = 0.0f + 1000.0f * (0.0f - xs) / L;
            const float yt = 0.0f + 1000.0f * (0.0f - ys) / L;
            const float zt = 0.0f + 1000.0f * (0.0f - zs) / L;
            const float labs = chord_through(xs, ys, zs, xt, yt, zt, ub);
            out = make_float4(a_pe, a_c, l1 - l2, labs);
        }
        pair[(long long)q * ld + (r - r0)] = out;
    }
}

// Column xx (0..7) of brick b: its (x, z), first y and whether it exists.
struct BrickCol {
    int x, z, y0, ci;            // ci: index in the column list (column mode)
    bool valid;
};

__device__ __forceinline__ BrickCol brick_column(const ScatterParams& P, int b, int xx) {
    BrickCol c;
    if (P.cols) {
        const int cg = b % P.bricks_x, by = b / P.bricks_x;
        c.ci = cg * kScBrickX + xx;
        c.valid = c.ci < P.n_cols;
        const int2 xz = c.valid ? P.cols[c.ci] : make_int2(0, 0);
        c.x = xz.x;
        c.z = xz.y;
        c.y0 = by * kScBrickY;
    } else {
        const int bx = b % P.bricks_x, by = (b / P.bricks_x) % P.bricks_y, bz = b / (P.bricks_x * P.bricks_y);
        c.x = bx * kScBrickX + xx;
        c.z = bz;
        c.y0 = by * kScBrickY;
        c.ci = 0;
        c.valid = c.x < P.nx;
    }
    return c;
}

// ---- sources with PE != 0 per voxel brick -----------------------------------------
__global__ void brick_sources_kernel(ScatterParams P, int N, uint32_t* __restrict__ out) {
    const int b = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.y * kScWarps + warp;
    if (s >= N) return;
    const BrickCol bc = brick_column(P, b, lane & 7);
    bool any = false;
    for (int it = 0; it < kScBrickY / 4; ++it) {
        const int y = bc.y0 + it * 4 + (lane >> 3);
        if (bc.valid && y < P.ny) {
            const long long v = (long long)bc.x + (long long)P.nx * (y + (long long)P.ny * bc.z);
            any |= __ldg(P.pe + (long long)s * P.ld_pe + v) != 0.0f;
        }
    }
    if (__any_sync(0xffffffffu, any) && lane == 0) atomicOr(out + (long long)b * P.src_words + (s >> 5), 1u << (s & 31));
}

// Detecting crystal d: geometry, energy window, switch (scatter.cu:1189-1205);
// returns the per-detector factor of the kind (mu_c / mu_pe / points, or plate mu_c / mu_t).
template <int KIND>
__device__ __forceinline__ float setup_det(const ScatterParams& P, const DevGeometry& G, const ScatterTables& T, int d,
                                           Det& D) {
    const float4 pos = G.c.pos[d], sz = G.c.size[d], rt = G.c.rot[d], ph = G.c.phys[d];
    D.x = pos.x; D.y = pos.y; D.z = pos.z; D.cm = rt.x; D.sm = rt.y;
    D.hw = 0.5f * sz.x; D.ht = 0.5f * sz.y; D.hh = 0.5f * sz.z;
    D.r_unit = sqrtf(sz.x * sz.x / 1.0f / 1.0f + sz.z * sz.z / 1.0f / 1.0f + sz.y * sz.y / 1.0f / 1.0f) / 2.0f;
    D.mu_pe = ph.x; D.mu_c = ph.y; D.res = ph.z;
    if (P.same_window > 0) { D.lo = P.win_lo; D.hi = P.win_hi; }
    else {
        D.lo = (1.0f - D.res / 2.0f) * P.e0;
        D.hi = (1.0f + D.res / 2.0f) * P.e0;
    }
    D.on = P.use_compton == 1 && pos.w > 0.01f;   // (scatter.cu:1203-1205)
    D.c_cut = window_cos_cut(P.e0, P.alpha, D.res, D.lo);
    return KIND == kScatterCrystal ? D.mu_c / D.mu_pe / (float)T.n_points : P.plate_c_over_t;
}

// Voxel centre (world) of fractional voxel indices: FOV shift and image rotation (scatter.cu:1172-1184).
__device__ __forceinline__ float3 voxel_world(const ScatterParams& P, float x, float y, float z) {
    float xi = (x - (float)P.nx / 2.0f + 0.5f) * P.vx;
    float yi = (y - (float)P.ny / 2.0f + 0.5f) * P.vy;
    float zi = (z - (float)P.nz / 2.0f + 0.5f) * P.vz;
    xi = xi + P.shx;
    yi = yi + P.shy;
    zi = zi + P.shz;
    return make_float3(xi * P.cos_a - yi * P.sin_a, xi * P.sin_a + yi * P.cos_a, zi);
}

// ---- transfer of arrival points per source ------------------------------------------
// K[a][r][s] = scale_d * sum_p term(vbar[a][s], s_p, d) for d = perm[r] and anchor a:
// the crystal-scatter sysmat entry per unit PE of source s with every photon
// arriving from vbar[a][s] (fractional voxel indices; w <= 0: source unused).
// Thread = rank (coalesced pair reads), grid.y = source; the source point and
// its pair sums are set up once for all anchors.
constexpr int kMaxAnchorsPerPass = 8;

template <typename KT>
__global__ void scatter_transfer_kernel(ScatterParams P, DevGeometry G, ScatterTables T, const float4* __restrict__ vbar,
                                        int n_anchors, KT* __restrict__ K, long long ldk, long long anchor_stride) {
    __shared__ KnNode kn[kKnNodes + 1];
    for (int i = threadIdx.x; i < kKnNodes + 1; i += blockDim.x) kn[i] = T.kn[i];
    __syncthreads();
    const int rank = P.rank0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (rank >= P.rank1) return;
    const int d = P.perm[rank];
    Det D;
    const float scale = setup_det<kScatterCrystal>(P, G, T, d, D);
    for (int s = blockIdx.y; s < T.n_crystals; s += gridDim.y) {
        for (int a0 = 0; a0 < n_anchors; a0 += kMaxAnchorsPerPass) {
            const int na = min(kMaxAnchorsPerPass, n_anchors - a0);
            float acc[kMaxAnchorsPerPass];
            float3 I[kMaxAnchorsPerPass], Is[kMaxAnchorsPerPass];
            bool use[kMaxAnchorsPerPass];
#pragma unroll
            for (int j = 0; j < kMaxAnchorsPerPass; ++j) {
                acc[j] = 0.0f;
                use[j] = false;
                if (j < na) {
                    const float4 vb = vbar[(long long)(a0 + j) * T.n_crystals + s];
                    use[j] = D.on && s != d && vb.w > 0.0f;
                    I[j] = voxel_world(P, vb.x, vb.y, vb.z);
                    Is[j] = make_float3((I[j].x - D.x) * D.cm - (I[j].z - D.z) * D.sm, I[j].y - D.y,
                                        (I[j].x - D.x) * D.sm + (I[j].z - D.z) * D.cm);
                }
            }
            bool any = false;
#pragma unroll
            for (int j = 0; j < kMaxAnchorsPerPass; ++j) any |= use[j];
            if (any) {
                for (int p = 0; p < T.n_points; ++p) {
                    const int q = s * T.n_points + p;
                    Src C;
                    make_src_basic(D, T.crystal_src[q], C);
                    make_src_rest(D, P.pair[(long long)q * P.pair_ld + (P.pair_col ? P.pair_col[rank] : rank - P.pair_r0)], C);
#pragma unroll
                    for (int j = 0; j < kMaxAnchorsPerPass; ++j)
                        if (use[j])
                            acc[j] += scatter_term(P, D, C, kn, T.kn_inv_norm, I[j].x, I[j].y, I[j].z, Is[j].x, Is[j].y,
                                                   Is[j].z);
                }
            }
#pragma unroll
            for (int j = 0; j < kMaxAnchorsPerPass; ++j)
                if (j < na) K[(long long)(a0 + j) * anchor_stride + (long long)(rank - P.rank0) * ldk + s] = (KT)(acc[j] * scale);
        }
    }
}

// Same values as scatter_transfer_kernel, arranged for memory traffic: a CTA
// takes 16 detectors (ranks) x 8 sources, stages the pair sums of that tile
// once in shared memory (instead of reading them again for every pass of 8
// anchors), and each detector's 8 consecutive sources are stored together
// (a run of 16 or 32 bytes instead of one sector per lane).  Up to 16 scatter
// points per crystal.
constexpr int kTrRanks = 16, kTrSrcs = 8, kTrMaxPoints = 16;

struct __align__(16) TrSmem {
    KnNode kn[kKnNodes + 1];
    float4 pr[kTrMaxPoints][kTrRanks][kTrSrcs];   // pair sums of the tile: [point][detector][source]
};

template <typename KT>
__global__ void __launch_bounds__(kTrRanks * kTrSrcs) scatter_transfer_tiled_kernel(
    ScatterParams P, DevGeometry G, ScatterTables T, const float4* __restrict__ vbar, int n_anchors,
    KT* __restrict__ K, long long ldk, long long anchor_stride) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrSmem& S = *reinterpret_cast<TrSmem*>(smem_raw);
    KnNode* kn = S.kn;
    auto& pr = S.pr;
    const int tid = threadIdx.x, rl = tid / kTrSrcs, sl = tid % kTrSrcs;
    const int r0 = P.rank0 + blockIdx.x * kTrRanks, s0 = blockIdx.y * kTrSrcs;
    const int np = T.n_points;
    for (int i = tid; i < kKnNodes + 1; i += blockDim.x) kn[i] = T.kn[i];
    for (int i = tid; i < np * kTrSrcs * kTrRanks; i += blockDim.x) {
        const int r = i % kTrRanks, ss = (i / kTrRanks) % kTrSrcs, p = i / (kTrRanks * kTrSrcs);
        const int rank = r0 + r, src = s0 + ss;
        float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (rank < P.rank1 && src < T.n_crystals) {
            const long long col = P.pair_col ? (long long)P.pair_col[rank] : (long long)(rank - P.pair_r0);
            v = P.pair[(long long)(src * np + p) * P.pair_ld + col];
        }
        pr[p][r][ss] = v;
    }
    __syncthreads();
    const int rank = r0 + rl, s = s0 + sl;
    if (rank >= P.rank1 || s >= T.n_crystals) return;
    const int d = P.perm[rank];
    Det D;
    const float scale = setup_det<kScatterCrystal>(P, G, T, d, D);
    for (int a0 = 0; a0 < n_anchors; a0 += kMaxAnchorsPerPass) {
        const int na = min(kMaxAnchorsPerPass, n_anchors - a0);
        float acc[kMaxAnchorsPerPass];
        float3 I[kMaxAnchorsPerPass], Is[kMaxAnchorsPerPass];
        bool use[kMaxAnchorsPerPass];
#pragma unroll
        for (int j = 0; j < kMaxAnchorsPerPass; ++j) {
            acc[j] = 0.0f;
            use[j] = false;
            if (j < na) {
                const float4 vb = vbar[(long long)(a0 + j) * T.n_crystals + s];
                use[j] = D.on && s != d && vb.w > 0.0f;
                I[j] = voxel_world(P, vb.x, vb.y, vb.z);
                Is[j] = make_float3((I[j].x - D.x) * D.cm - (I[j].z - D.z) * D.sm, I[j].y - D.y,
                                    (I[j].x - D.x) * D.sm + (I[j].z - D.z) * D.cm);
            }
        }
        bool any = false;
#pragma unroll
        for (int j = 0; j < kMaxAnchorsPerPass; ++j) any |= use[j];
        if (any) {
            for (int p = 0; p < np; ++p) {
                Src C;
                make_src_basic(D, T.crystal_src[s * np + p], C);
                make_src_rest(D, pr[p][rl][sl], C);
#pragma unroll
                for (int j = 0; j < kMaxAnchorsPerPass; ++j)
                    if (use[j])
                        acc[j] += scatter_term(P, D, C, kn, T.kn_inv_norm, I[j].x, I[j].y, I[j].z, Is[j].x, Is[j].y,
                                               Is[j].z);
            }
        }
#pragma unroll
        for (int j = 0; j < kMaxAnchorsPerPass; ++j)
            if (j < na) K[(long long)(a0 + j) * anchor_stride + (long long)(rank - P.rank0) * ldk + s] = (KT)(acc[j] * scale);
    }
}

struct __align__(16) ScSmem {
    KnNode kn[kKnNodes + 1];
    double acc[kScBrickX][kScBrickY][kScTileD];
    float4 vox[kScBrickX][kScBrickY];          // voxel centres (world); w < 0 marks outside the grid
    float pe[kScBrickY][kScBrickX];
    float scale[kScTileD];                     // per detector: mu_c / mu_pe / points, or plate mu_c / mu_t
};

template <int KIND>
__global__ void __launch_bounds__(kScThreads, 2) scatter_main_kernel(ScatterParams P, DevGeometry G, ScatterTables T) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ScSmem& S = *reinterpret_cast<ScSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = blockIdx.x % P.n_bricks;
    const int dt = blockIdx.x / P.n_bricks;
    const BrickCol mycol = brick_column(P, b, warp);        // this warp's voxel column
    const BrickCol stcol = brick_column(P, b, tid & 7);     // the column this thread stages
    const int y0 = mycol.y0;

    for (int i = tid; i < kKnNodes + 1; i += kScThreads) S.kn[i] = T.kn[i];
    for (int i = tid; i < kScBrickX * kScBrickY * kScTileD; i += kScThreads) (&S.acc[0][0][0])[i] = 0.0;
    {
        const int xx = tid & 7, yy = tid >> 3;
        const int x = stcol.x, y = y0 + yy;
        float4 v = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        if (stcol.valid && y < P.ny) {
            const float3 w = voxel_world(P, (float)x, (float)y, (float)stcol.z);
            v = make_float4(w.x, w.y, w.z, 1.0f);
        }
        S.vox[xx][yy] = v;
    }

    const int rank = P.rank0 + dt * kScTileD + lane;
    const int d = rank < P.rank1 ? P.perm[rank] : -1;
    Det D;
    D.on = false;
    float scale = 0.0f;
    if (rank < P.rank1) scale = setup_det<KIND>(P, G, T, d, D);
    if (warp == 0) S.scale[lane] = scale;
    __syncthreads();

    const float inv_norm = T.kn_inv_norm;
    // this warp's voxel column: I0 + t e, t in [0, col_t] (image y axis, rotated)
    const float4 col0 = S.vox[warp][0];
    const float col_ex = -P.sin_a, col_ey = P.cos_a;
    const float col_t = (float)(min(kScBrickY, P.ny - y0) - 1) * P.vy;
    if (KIND == kScatterCrystal) {
        const uint32_t* srcw = P.brick_sources + (long long)b * P.src_words;
        for (int wd = 0; wd < P.src_words; ++wd) {
            uint32_t bits = srcw[wd];
            while (bits) {
                const int s = (wd << 5) + __ffs(bits) - 1;
                bits &= bits - 1u;
                __syncthreads();
                {
                    const int xx = tid & 7, yy = tid >> 3;
                    float v = 0.0f;
                    if (stcol.valid && y0 + yy < P.ny)
                        v = __ldg(P.pe + (long long)s * P.ld_pe + stcol.x +
                                  (long long)P.nx * ((y0 + yy) + (long long)P.ny * stcol.z));
                    S.pe[yy][xx] = v;
                }
                __syncthreads();
                const float my_pe = S.pe[lane][warp];
                const unsigned live = __ballot_sync(0xffffffffu, my_pe != 0.0f);
                if (!live) continue;
                for (int p = 0; p < T.n_points; ++p) {
                    const int q = s * T.n_points + p;
                    const float4 src = T.crystal_src[q];
                    Src C;
                    bool on = D.on && s != d;
                    if (on) {
                        make_src_basic(D, src, C);
                        // no voxel of the column passes the window cut: the lane sits out
                        on = column_max_cos(C, col0.x, col0.y, col0.z, col_ex, col_ey, 0.0f, col_t) > D.c_cut;
                    }
                    if (!__any_sync(0xffffffffu, on)) continue;
                    if (on) {
                        const long long pc = P.pair_col ? P.pair_col[rank] : rank - P.pair_r0;
                        make_src_rest(D, P.pair[(long long)q * P.pair_ld + pc], C);
                    }
                    unsigned m = live;
                    while (m) {
                        const int j = __ffs(m) - 1;
                        m &= m - 1u;
                        const float w = __shfl_sync(0xffffffffu, my_pe, j);
                        if (!on) continue;
                        const float4 I = S.vox[warp][j];
                        const float isx = (I.x - D.x) * D.cm - (I.z - D.z) * D.sm;
                        const float isy = I.y - D.y;
                        const float isz = (I.x - D.x) * D.sm + (I.z - D.z) * D.cm;
                        const float t = scatter_term(P, D, C, S.kn, inv_norm, I.x, I.y, I.z, isx, isy, isz);
                        S.acc[warp][j][lane] += (double)(w * t);
                    }
                }
            }
        }
    } else {
        for (int h = 0; h < T.n_holes0; ++h) {
            const float4 src = T.hole_src[h];
            Src C;
            bool on = D.on && mycol.valid;
            if (on) {
                make_src_basic(D, src, C);
                on = column_max_cos(C, col0.x, col0.y, col0.z, col_ex, col_ey, 0.0f, col_t) > D.c_cut;
            }
            if (!on) continue;
            make_src_rest(D, P.pair[(long long)h * P.pair_ld + (rank - P.pair_r0)], C);
            for (int j = 0; j < kScBrickY; ++j) {
                const float4 I = S.vox[warp][j];
                if (I.w < 0.0f) break;
                // virtual solid angle of the hole seen from the voxel (scatter.cu:1707-1713)
                const float vr = 0.1f;
                const float dx = I.x - src.x, dy = I.y - src.y, dz = I.z - src.z;
                const float L2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                const float Lih = sqrtf(L2);
                const float w = (vr * vr * 3.14159265358979323846f + src.w * vr) /
                                (4.0f * 3.14159265358979323846f * L2) * fabsf(src.y - I.y) / Lih;
                const float isx = (I.x - D.x) * D.cm - (I.z - D.z) * D.sm;
                const float isy = I.y - D.y;
                const float isz = (I.x - D.x) * D.sm + (I.z - D.z) * D.cm;
                const float t = scatter_term(P, D, C, S.kn, inv_norm, I.x, I.y, I.z, isx, isy, isz);
                S.acc[warp][j][lane] += (double)(w * t);
            }
        }
    }
    __syncthreads();

    // write the tile: (detector, y, 8 x) with x fastest
    const int n_rows = min(kScTileD, P.rank1 - (P.rank0 + dt * kScTileD));
    for (int i = tid; i < n_rows * kScBrickY * kScBrickX; i += kScThreads) {
        const int xx = i & 7, yy = (i >> 3) & 31, dl = i >> 8;
        const BrickCol oc = brick_column(P, b, xx);
        const int yv = y0 + yy;
        if (!oc.valid || yv >= P.ny) continue;
        const int rk = P.rank0 + dt * kScTileD + dl;
        const int dd = P.perm[rk];
        const float sc = S.scale[dl];
        const long long col = P.cols ? (long long)oc.ci * P.ny + yv
                                     : (long long)oc.x + (long long)P.nx * (yv + (long long)P.ny * oc.z);
        const long long orow = P.slot ? (long long)P.slot[rk] : (long long)(dd - P.dst_row0);
        float* out = P.dst + orow * P.ld + col;
        const float v = (float)S.acc[xx][yy][dl] * sc;
        *out = P.accumulate ? *out + v : v;
    }
}

// ---- crystal scatter for scattered detector rows: voxels on the lanes ----------------------
// The same entries and the same sums as scatter_main_kernel<crystal> (per
// entry the terms are added in the same (source, point) order, so results are
// bit-identical), for row lists whose 32 detectors per tile lie far apart: a
// warp is one voxel column; per source point one lane per detector runs the
// column's window cull, then the (passing detector, voxel with PE != 0) pairs
// are spread over the 32 lanes, so lanes are not left idle by detectors that
// cull or voxels the source does not see.
// Position of the n-th (from 0) set bit of m; m must have more than n set bits.
__device__ __forceinline__ int nth_set_bit(unsigned m, int n) {
    for (int i = 0; i < n; ++i) m &= m - 1u;
    return __ffs(m) - 1;
}

struct __align__(16) ScRowSmem {
    KnNode kn[kKnNodes + 1];
    double acc[kScBrickX][kScBrickY][kScTileD];
    float4 vox[kScBrickX][kScBrickY];
    float pe[kScBrickY][kScBrickX];
    float scale[kScTileD];
    Det det[kScTileD];
    int d[kScTileD];
    long long pc[kScTileD];                    // pair column of each detector
};

__global__ void __launch_bounds__(kScThreads, 2) scatter_rows_kernel(ScatterParams P, DevGeometry G, ScatterTables T) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ScRowSmem& S = *reinterpret_cast<ScRowSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = blockIdx.x % P.n_bricks;
    const int dt = blockIdx.x / P.n_bricks;
    const BrickCol mycol = brick_column(P, b, warp);
    const BrickCol stcol = brick_column(P, b, tid & 7);
    const int y0 = mycol.y0;

    for (int i = tid; i < kKnNodes + 1; i += kScThreads) S.kn[i] = T.kn[i];
    for (int i = tid; i < kScBrickX * kScBrickY * kScTileD; i += kScThreads) (&S.acc[0][0][0])[i] = 0.0;
    {
        const int xx = tid & 7, yy = tid >> 3;
        const int x = stcol.x, y = y0 + yy;
        float4 v = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        if (stcol.valid && y < P.ny) {
            const float3 w = voxel_world(P, (float)x, (float)y, (float)stcol.z);
            v = make_float4(w.x, w.y, w.z, 1.0f);
        }
        S.vox[xx][yy] = v;
    }
    if (warp == 0) {
        const int rank = P.rank0 + dt * kScTileD + lane;
        Det D;
        D.on = false;
        float scale = 0.0f;
        int d = -1;
        if (rank < P.rank1) {
            d = P.perm[rank];
            scale = setup_det<kScatterCrystal>(P, G, T, d, D);
        }
        S.det[lane] = D;
        S.d[lane] = d;
        S.scale[lane] = scale;
        S.pc[lane] = rank < P.rank1 ? (P.pair_col ? (long long)P.pair_col[rank] : (long long)(rank - P.pair_r0)) : 0;
    }
    __syncthreads();
    const int n_det = min(kScTileD, P.rank1 - (P.rank0 + dt * kScTileD));

    const float inv_norm = T.kn_inv_norm;
    const float4 col0 = S.vox[warp][0];
    const float col_ex = -P.sin_a, col_ey = P.cos_a;
    const float col_t = (float)(min(kScBrickY, P.ny - y0) - 1) * P.vy;
    const uint32_t* srcw = P.brick_sources + (long long)b * P.src_words;
    for (int wd = 0; wd < P.src_words; ++wd) {
        uint32_t bits = srcw[wd];
        while (bits) {
            const int s = (wd << 5) + __ffs(bits) - 1;
            bits &= bits - 1u;
            __syncthreads();
            {
                const int xx = tid & 7, yy = tid >> 3;
                float v = 0.0f;
                if (stcol.valid && y0 + yy < P.ny)
                    v = __ldg(P.pe + (long long)s * P.ld_pe + stcol.x +
                              (long long)P.nx * ((y0 + yy) + (long long)P.ny * stcol.z));
                S.pe[yy][xx] = v;
            }
            __syncthreads();
            const unsigned live = __ballot_sync(0xffffffffu, S.pe[lane][warp] != 0.0f);
            if (!live) continue;
            const int n_live = __popc(live);
            for (int p = 0; p < T.n_points; ++p) {
                const int q = s * T.n_points + p;
                const float4 src = T.crystal_src[q];
                // window cull of the column, one detector per lane
                bool pass = false;
                if (lane < n_det) {
                    const Det& D = S.det[lane];
                    if (D.on && s != S.d[lane]) {
                        Src C;
                        make_src_basic(D, src, C);
                        pass = column_max_cos(C, col0.x, col0.y, col0.z, col_ex, col_ey, 0.0f, col_t) > D.c_cut;
                    }
                }
                const unsigned pmask = __ballot_sync(0xffffffffu, pass);
                if (!pmask) continue;
                // (passing detector, live voxel) pairs spread over the lanes; each pair once per point
                const int n_items = __popc(pmask) * n_live;
                for (int base = 0; base < n_items; base += 32) {
                    const int item = base + lane;
                    if (item >= n_items) continue;
                    const int k = item / n_live, jj = item - k * n_live;
                    const int dl = nth_set_bit(pmask, k), j = nth_set_bit(live, jj);
                    const Det& D = S.det[dl];
                    Src C;
                    make_src_basic(D, src, C);
                    make_src_rest(D, P.pair[(long long)q * P.pair_ld + S.pc[dl]], C);
                    const float4 Iv = S.vox[warp][j];
                    const float isx = (Iv.x - D.x) * D.cm - (Iv.z - D.z) * D.sm;
                    const float isy = Iv.y - D.y;
                    const float isz = (Iv.x - D.x) * D.sm + (Iv.z - D.z) * D.cm;
                    const float t = scatter_term(P, D, C, S.kn, inv_norm, Iv.x, Iv.y, Iv.z, isx, isy, isz);
                    S.acc[warp][j][dl] += (double)(S.pe[j][warp] * t);
                }
            }
        }
    }
    __syncthreads();
    for (int i = tid; i < n_det * kScBrickY * kScBrickX; i += kScThreads) {
        const int xx = i & 7, yy = (i >> 3) & 31, dl = i >> 8;
        const BrickCol oc = brick_column(P, b, xx);
        const int yv = y0 + yy;
        if (!oc.valid || yv >= P.ny) continue;
        const int rk = P.rank0 + dt * kScTileD + dl;
        const int dd = S.d[dl];
        const long long col = P.cols ? (long long)oc.ci * P.ny + yv
                                     : (long long)oc.x + (long long)P.nx * (yv + (long long)P.ny * oc.z);
        const long long orow = P.slot ? (long long)P.slot[rk] : (long long)(dd - P.dst_row0);
        float* out = P.dst + orow * P.ld + col;
        const float v = (float)S.acc[xx][yy][dl] * S.scale[dl];
        *out = P.accumulate ? *out + v : v;
    }
}

}  // namespace

int64_t crystal_bitmap_words(int n) {
    const int64_t bits = ((int64_t)n * (n + 1) / 2) * n;
    return (bits + 31) / 32;
}

int64_t collimator_bitmap_words(int n, int h0) {
    const int64_t bits = (int64_t)h0 * n * n;
    return (bits + 31) / 32;
}

cudaError_t launch_bitmap_crystal(uint32_t* words, int64_t n_words, const ScatterTables& T, cudaStream_t s) {
    if (n_words <= 0) return cudaSuccess;
    const long long blocks = std::min<long long>((n_words + 255) / 256, 148LL * 64);
    bitmap_crystal_kernel<<<(unsigned)blocks, 256, 0, s>>>(words, n_words, T);
    return cudaGetLastError();
}

cudaError_t launch_bitmap_collimator(uint32_t* words, int64_t n_words, const ScatterTables& T, cudaStream_t s) {
    if (n_words <= 0) return cudaSuccess;
    const long long blocks = std::min<long long>((n_words + 255) / 256, 148LL * 64);
    bitmap_collimator_kernel<<<(unsigned)blocks, 256, 0, s>>>(words, n_words, T);
    return cudaGetLastError();
}

cudaError_t launch_scatter_pairs(int kind, const DevGeometry& G, const ScatterTables& T, const uint32_t* bitmap,
                                 const int* perm, int r0, int r1, float4* pair, cudaStream_t s) {
    const int n_src = kind == kScatterCrystal ? T.n_crystals * T.n_points : T.n_holes0;
    if (r1 <= r0 || n_src <= 0) return cudaSuccess;
    dim3 grid((r1 - r0 + 127) / 128, std::min(n_src, 65535));
    if (kind == kScatterCrystal)
        scatter_pair_kernel<kScatterCrystal><<<grid, 128, 0, s>>>(G, T, bitmap, perm, r0, r1, pair, n_src);
    else
        scatter_pair_kernel<kScatterCollimator><<<grid, 128, 0, s>>>(G, T, bitmap, perm, r0, r1, pair, n_src);
    return cudaGetLastError();
}

cudaError_t launch_brick_sources(const ScatterParams& P, const ScatterTables& T, uint32_t* brick_sources,
                                 cudaStream_t s) {
    dim3 grid(P.n_bricks, (T.n_crystals + kScWarps - 1) / kScWarps);
    brick_sources_kernel<<<grid, kScThreads, 0, s>>>(P, T.n_crystals, brick_sources);
    return cudaGetLastError();
}

cudaError_t launch_scatter_transfer(const ScatterParams& P, const DevGeometry& G, const ScatterTables& T,
                                    const float4* vbar, int n_anchors, void* K, bool k_bf16, long long ldk,
                                    long long anchor_stride, cudaStream_t s) {
    if (P.rank1 <= P.rank0 || T.n_crystals <= 0 || n_anchors <= 0) return cudaSuccess;
    if (T.n_points <= kTrMaxPoints && (T.n_crystals + kTrSrcs - 1) / kTrSrcs <= 65535) {
        dim3 tg((P.rank1 - P.rank0 + kTrRanks - 1) / kTrRanks, (T.n_crystals + kTrSrcs - 1) / kTrSrcs);
        const int smem = (int)sizeof(TrSmem);
        cudaError_t e;
        if (k_bf16) {
            e = cudaFuncSetAttribute(scatter_transfer_tiled_kernel<__nv_bfloat16>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess) return e;
            scatter_transfer_tiled_kernel<__nv_bfloat16><<<tg, kTrRanks * kTrSrcs, smem, s>>>(
                P, G, T, vbar, n_anchors, static_cast<__nv_bfloat16*>(K), ldk, anchor_stride);
        } else {
            e = cudaFuncSetAttribute(scatter_transfer_tiled_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     smem);
            if (e != cudaSuccess) return e;
            scatter_transfer_tiled_kernel<float><<<tg, kTrRanks * kTrSrcs, smem, s>>>(
                P, G, T, vbar, n_anchors, static_cast<float*>(K), ldk, anchor_stride);
        }
        return cudaGetLastError();
    }
    dim3 grid((P.rank1 - P.rank0 + 127) / 128, std::min(T.n_crystals, 65535));
    if (k_bf16)
        scatter_transfer_kernel<__nv_bfloat16><<<grid, 128, 0, s>>>(P, G, T, vbar, n_anchors,
                                                                   static_cast<__nv_bfloat16*>(K), ldk, anchor_stride);
    else
        scatter_transfer_kernel<float><<<grid, 128, 0, s>>>(P, G, T, vbar, n_anchors, static_cast<float*>(K), ldk,
                                                            anchor_stride);
    return cudaGetLastError();
}

cudaError_t launch_scatter_rows(const ScatterParams& P, const DevGeometry& G, const ScatterTables& T, cudaStream_t s) {
    const size_t smem = sizeof(ScRowSmem);
    const long long d_tiles = (P.rank1 - P.rank0 + kScTileD - 1) / kScTileD;
    const long long blocks = d_tiles * P.n_bricks;
    if (blocks <= 0) return cudaSuccess;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaFuncSetAttribute(scatter_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    scatter_rows_kernel<<<(unsigned)blocks, kScThreads, smem, s>>>(P, G, T);
    return cudaGetLastError();
}

cudaError_t launch_scatter_main(const ScatterParams& P, const DevGeometry& G, const ScatterTables& T,
                                cudaStream_t s) {
    const size_t smem = sizeof(ScSmem);
    const long long d_tiles = (P.rank1 - P.rank0 + kScTileD - 1) / kScTileD;
    const long long blocks = d_tiles * P.n_bricks;
    if (blocks <= 0) return cudaSuccess;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    cudaError_t e;
    if (P.kind == kScatterCrystal) {
        e = cudaFuncSetAttribute(scatter_main_kernel<kScatterCrystal>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        scatter_main_kernel<kScatterCrystal><<<(unsigned)blocks, kScThreads, smem, s>>>(P, G, T);
    } else {
        e = cudaFuncSetAttribute(scatter_main_kernel<kScatterCollimator>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        scatter_main_kernel<kScatterCollimator><<<(unsigned)blocks, kScThreads, smem, s>>>(P, G, T);
    }
    return cudaGetLastError();
}

}  // namespace smb
