// Host driver of the scatter surrogate (include/sysmat_b200.h, sm_scatter_surrogate)
// and the C ABI of the network alone.
//
// No reference counterpart: the reference computes every crystal-scatter entry
// with the nested integral of crystalScatterSysMatCuda (scatter.cu:1077-1437).
// Here that kernel (exact_scatter) computes a seeded subset of voxel columns,
// a physics baseline and a learned correction predict the rest, and the exact
// kernel re-checks held-out columns of every row and recomputes rows over
// tolerance, so it stays both the fallback and the final check.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.h"
#include "context.h"
#include "scatter.h"
#include "surrogate.h"

namespace smb {
namespace {

uint32_t morton2(int x, int z) {
    uint32_t k = 0;
    for (int b = 0; b < 16; ++b) k |= (((uint32_t)x >> b) & 1u) << (2 * b) | (((uint32_t)z >> b) & 1u) << (2 * b + 1);
    return k;
}

struct Timer {
    cudaEvent_t e[12];
    int n = 0;
    cudaStream_t s;
    explicit Timer(cudaStream_t st) : s(st) {
        for (auto& x : e) cudaEventCreate(&x);
    }
    ~Timer() {
        for (auto& x : e) cudaEventDestroy(x);
    }
    int mark() {
        cudaEventRecord(e[n], s);
        return n++;
    }
    double ms(int a, int b) {
        float t = 0.0f;
        cudaEventElapsedTime(&t, e[a], e[b]);
        return t;
    }
};

template <typename T>
int upload(DevBuf& b, const std::vector<T>& v, cudaStream_t s, const char* what) {
    SM_TRY(b.alloc(sizeof(T) * std::max<size_t>(1, v.size()), s, what));
    if (!v.empty()) SM_CUDA(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
    return SM_OK;
}

double quantile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

// Per-row relative L2 errors of pred against ref over n columns (host vector).
int row_errors(const float* pred, int64_t ld_pred, const float* ref, int64_t ld_ref, int N, int n, cudaStream_t s,
               std::vector<double>* err, std::vector<double>* norm2_out = nullptr) {
    DevBuf b;
    SM_TRY(b.alloc(sizeof(double) * 2 * (size_t)N, s, "row errors"));
    double* e2 = static_cast<double*>(b.p);
    SM_CUDA(launch_row_error(pred, ld_pred, ref, ld_ref, N, n, e2, e2 + N, s));
    std::vector<double> h(2 * (size_t)N);
    SM_CUDA(cudaMemcpyAsync(h.data(), e2, sizeof(double) * 2 * (size_t)N, cudaMemcpyDeviceToHost, s));
    SM_CUDA(cudaStreamSynchronize(s));
    err->resize(N);
    for (int d = 0; d < N; ++d) {
        const double q = h[N + d];
        (*err)[d] = q > 0.0 ? std::sqrt(h[d] / q) : (h[d] > 0.0 ? INFINITY : 0.0);
    }
    if (norm2_out) norm2_out->assign(h.begin() + N, h.end());
    return SM_OK;
}

// Per-row sums over n columns: e2[d] = sum (pred - ref)^2, q2[d] = sum ref^2.
int row_sums(const float* pred, int64_t ld_pred, const float* ref, int64_t ld_ref, int N, int64_t n, cudaStream_t s,
             std::vector<double>* e2, std::vector<double>* q2) {
    if (n > 0x7fffffff) return fail(SM_ERR_CAPACITY, "row of %lld columns", (long long)n);
    DevBuf b;
    SM_TRY(b.alloc(sizeof(double) * 2 * (size_t)N, s, "row sums"));
    double* d = static_cast<double*>(b.p);
    SM_CUDA(launch_row_error(pred, ld_pred, ref, ld_ref, N, (int)n, d, d + N, s));
    std::vector<double> h(2 * (size_t)N);
    SM_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(double) * 2 * (size_t)N, cudaMemcpyDeviceToHost, s));
    SM_CUDA(cudaStreamSynchronize(s));
    e2->assign(h.begin(), h.begin() + N);
    q2->assign(h.begin() + N, h.end());
    return SM_OK;
}

// Estimated relative L2 error of a predicted row from sampled columns: the
// squared error on `lines` sampled voxel columns out of L, scaled to the row,
// over the norm of the whole predicted row.
double row_estimate(double e2, int lines, int L, double pred_n2) {
    const double est = e2 * (double)L / (double)std::max(1, lines);
    if (pred_n2 > 0.0) return std::sqrt(est / pred_n2);
    return est > 0.0 ? INFINITY : 0.0;
}

// Baseline B = sum_a w_a(v) K_a PE into dst (crystal part).
int baseline(const sm_geometry* geo, const int sp[3], float angle, const int anchors[3], const float* d_pe,
             int64_t ld_pe, const float4* pairs, const int* d_order, float* d_dst, int64_t ld, int* d_error,
             double* ms_transfer, cudaStream_t s) {
    const HostGeometry& g = geo->host;
    const int N = g.n_crystals, nx = g.nx, ny = g.ny, nz = g.nz;
    const int64_t V = (int64_t)nx * ny * nz;
    const int kx = std::max(1, std::min(anchors[0], nx)), ky = std::max(1, std::min(anchors[1], ny)),
              kz = std::max(1, std::min(anchors[2], nz));
    const int A = kx * ky * kz;
    const AxisTable ax = make_axis(nx, kx), ay = make_axis(ny, ky), az = make_axis(nz, kz);
    std::vector<int> lo, hi;
    std::vector<float> t;
    for (const AxisTable* T : {&ax, &ay, &az}) {
        lo.insert(lo.end(), T->lo.begin(), T->lo.end());
        hi.insert(hi.end(), T->hi.begin(), T->hi.end());
        t.insert(t.end(), T->t.begin(), T->t.end());
    }
    // cells: one per (slab x, slab y, slab z) that holds voxels
    auto ranges = [](const AxisTable& T, int k) {
        std::vector<std::pair<int, int>> r(k + 1, {0, 0});   // [first, count]
        for (int j = 0; j <= k; ++j) r[j] = {-1, 0};
        for (int x = 0; x < (int)T.slab.size(); ++x) {
            auto& q = r[T.slab[x]];
            if (q.first < 0) q.first = x;
            ++q.second;
        }
        return r;
    };
    const auto rx = ranges(ax, kx), ry = ranges(ay, ky), rz = ranges(az, kz);
    std::vector<BaseCell> cells;
    std::vector<BaseItem> items;
    for (int jz = 0; jz <= kz; ++jz)
        for (int jy = 0; jy <= ky; ++jy)
            for (int jx = 0; jx <= kx; ++jx) {
                if (rx[jx].second == 0 || ry[jy].second == 0 || rz[jz].second == 0) continue;
                BaseCell c{};
                c.x0 = rx[jx].first;
                c.y0 = ry[jy].first;
                c.z0 = rz[jz].first;
                c.nx = rx[jx].second;
                c.ny = ry[jy].second;
                c.nz = rz[jz].second;
                const int lo3[3] = {ax.lo[c.x0], ay.lo[c.y0], az.lo[c.z0]};
                const int hi3[3] = {ax.hi[c.x0], ay.hi[c.y0], az.hi[c.z0]};
                c.n_seg = 0;
                for (int bits = 0; bits < 8; ++bits) {
                    bool skip = false;
                    int idx[3], side = 0;
                    for (int a = 0; a < 3; ++a) {
                        const int b = (bits >> a) & 1;
                        const bool dual = lo3[a] != hi3[a];
                        if (b && !dual) skip = true;
                        idx[a] = b ? hi3[a] : lo3[a];
                        side |= (b << a) | ((dual ? 1 : 0) << (a + 4));
                    }
                    if (skip) continue;
                    c.anchor[c.n_seg] = (idx[0] * ky + idx[1]) * kz + idx[2];
                    c.side[c.n_seg] = side;
                    ++c.n_seg;
                }
                const int n_vox = c.nx * c.ny * c.nz;
                for (int n0 = 0; n0 < n_vox; n0 += 256) items.push_back({(int)cells.size(), n0});
                cells.push_back(c);
            }
    if (items.size() > 65535) return fail(SM_ERR_CAPACITY, "baseline: %zu column tiles exceed one launch", items.size());

    DevBuf pet, tabs_i, tabs_f, vbar, K, dcells, ditems;
    SM_TRY(pet.alloc(sizeof(__nv_bfloat16) * (size_t)V * N, s, "transposed PE"));
    SM_CUDA(launch_pe_transpose(d_pe, ld_pe, N, V, static_cast<__nv_bfloat16*>(pet.p), s));
    std::vector<int> lohi(lo);
    lohi.insert(lohi.end(), hi.begin(), hi.end());
    std::vector<int> box;
    for (const AxisTable* T : {&ax, &ay, &az})
        for (int i = 0; i < T->k; ++i) {
            box.push_back(T->first[i]);
            box.push_back(T->count[i]);
        }
    const size_t box_at = lohi.size();
    lohi.insert(lohi.end(), box.begin(), box.end());
    SM_TRY(upload(tabs_i, lohi, s, "anchor tables"));
    SM_TRY(upload(tabs_f, t, s, "anchor weights"));
    SM_TRY(vbar.alloc(sizeof(float4) * (size_t)A * N, s, "anchor points"));
    const int* d_lo = static_cast<const int*>(tabs_i.p);
    const int* d_hi = d_lo + lo.size();
    const int* d_box = d_lo + box_at;
    const float* d_t = static_cast<const float*>(tabs_f.p);
    SM_CUDA(launch_anchor_centroids(d_pe, ld_pe, N, nx, ny, nz, d_lo, d_hi, d_t, d_box, kx, ky, kz,
                                    static_cast<float4*>(vbar.p), s));
    SM_TRY(K.alloc(sizeof(__nv_bfloat16) * (size_t)A * N * N, s, "transfer matrices"));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    SM_TRY(scatter_transfer(geo, sp, angle, static_cast<const float4*>(vbar.p), A, K.p, N, true, pairs, d_order, s));
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float tms = 0.0f;
    cudaEventElapsedTime(&tms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms_transfer) *ms_transfer = tms;
    SM_TRY(upload(dcells, cells, s, "baseline cells"));
    SM_TRY(upload(ditems, items, s, "baseline tiles"));
    SM_CUDA(launch_baseline_gemm(static_cast<const __nv_bfloat16*>(K.p), static_cast<const __nv_bfloat16*>(pet.p), N, nx,
                                 ny, static_cast<const BaseCell*>(dcells.p), static_cast<const BaseItem*>(ditems.p),
                                 (int)items.size(), d_t, d_t + nx, d_t + nx + ny, pairs ? d_order : nullptr, d_dst, ld,
                                 d_error, s));
    SM_CUDA(cudaStreamSynchronize(s));   // host tables are released on return
    return SM_OK;
}

}  // namespace

// The seeded voxel y-columns (x, z): n_tr train columns, then n_ho held-out
// ones, each group in Morton order of (x, z).  `rng` continues from here.
void select_columns(const HostGeometry& g, const sm_surrogate_options& o, std::mt19937_64& rng, std::vector<int2>* cols,
                    int* n_tr_out, int* n_ho_out) {
    const int nx = g.nx, L = g.nx * g.nz;
    std::vector<int> perm(L);
    std::iota(perm.begin(), perm.end(), 0);
    std::shuffle(perm.begin(), perm.end(), rng);
    const int n_tr = std::max(1, std::min(L - 2, (int)std::lround(o.train_frac * L)));
    const int n_ho = std::max(1, std::min(L - n_tr, (int)std::lround(o.holdout_frac * L)));
    auto by_morton = [&](std::vector<int> lines) {
        std::sort(lines.begin(), lines.end(),
                  [&](int a, int b) { return morton2(a % nx, a / nx) < morton2(b % nx, b / nx); });
        return lines;
    };
    const std::vector<int> tr = by_morton(std::vector<int>(perm.begin(), perm.begin() + n_tr));
    const std::vector<int> ho = by_morton(std::vector<int>(perm.begin() + n_tr, perm.begin() + n_tr + n_ho));
    cols->clear();
    for (int l : tr) cols->push_back(make_int2(l % nx, l / nx));
    for (int l : ho) cols->push_back(make_int2(l % nx, l / nx));
    *n_tr_out = n_tr;
    *n_ho_out = n_ho;
}

int scatter_surrogate(const sm_geometry* geo, const sm_surrogate_options& o, float angle, const float* d_pe,
                      int64_t ld_pe, float* d_dst, int64_t ld, float* row_error, int32_t* row_state,
                      sm_surrogate_stats* st, cudaStream_t s) {
    const HostGeometry& g = geo->host;
    const int N = g.n_crystals, nx = g.nx, ny = g.ny, nz = g.nz;
    const int64_t V = (int64_t)nx * ny * nz;
    const int L = nx * nz;
    sm_surrogate_stats S{};
    Timer tm(s);
    const int t0 = tm.mark();

    // ---- 1. voxel columns: train (fit + validation) and held-out, seeded ----
    std::mt19937_64 rng(o.seed);
    std::vector<int2> cols;
    int n_tr = 0, n_ho = 0;
    select_columns(g, o, rng, &cols, &n_tr, &n_ho);
    (void)L;
    const int64_t ldy = (int64_t)(n_tr + n_ho) * ny;   // Y: [N][train columns | held-out columns]
    const int n_trc = n_tr * ny, n_hoc = n_ho * ny;
    S.n_train_columns = n_trc;
    S.n_holdout_columns = n_hoc;

    DevBuf dcols, Y, Bv, err_flag;
    SM_TRY(upload(dcols, cols, s, "surrogate columns"));
    SM_TRY(Y.alloc(sizeof(float) * (size_t)N * ldy, s, "exact columns"));
    SM_TRY(Bv.alloc(sizeof(float) * (size_t)N * ldy, s, "baseline columns"));
    SM_TRY(err_flag.alloc(sizeof(int), s, "error flag"));
    SM_CUDA(cudaMemsetAsync(err_flag.p, 0, sizeof(int), s));
    float* dY = static_cast<float*>(Y.p);
    float* dB = static_cast<float*>(Bv.p);
    // one crystal pair table (attenuation sums per source point and detector) for every exact and transfer step
    DevBuf pairs, d_order;
    std::vector<int> order_all;
    SM_TRY(crystal_pair_table(geo, o.sp, &pairs, &order_all, &d_order, s));
    const float4* d_pairs = static_cast<const float4*>(pairs.p);
    const int tp = tm.mark();
    {
        ExactSpec spec;
        spec.row0 = 0;
        spec.row1 = N;
        spec.d_cols = static_cast<const int2*>(dcols.p);
        spec.n_cols = n_tr + n_ho;
        spec.pairs = d_pairs;
        spec.pairs_order = &order_all;
        SM_TRY(exact_scatter(geo, o.sp, 1, angle, d_pe, ld_pe, nullptr, nullptr, spec, dY, ldy, s));
    }
    const int t1 = tm.mark();

    // ---- 2. physics baseline over every voxel ----
    SM_TRY(baseline(geo, o.sp, angle, o.anchors, d_pe, ld_pe, d_pairs, static_cast<const int*>(d_order.p), d_dst, ld,
                    static_cast<int*>(err_flag.p), &S.ms_transfer, s));
    SM_CUDA(launch_gather_columns(d_dst, ld, N, static_cast<const int2*>(dcols.p), n_tr + n_ho, nx, ny, dB, ldy, s));
    const int t2 = tm.mark();
    // baseline error estimate per row: every exactly computed column samples it
    std::vector<double> tr_e2, tr_q2, ho_e2, ho_q2, dummy;
    SM_TRY(row_sums(dB, ldy, dY, ldy, N, n_trc, s, &tr_e2, &tr_q2));
    SM_TRY(row_sums(dB + n_trc, ldy, dY + n_trc, ldy, N, n_hoc, s, &ho_e2, &ho_q2));

    // ---- 3. learned correction ----
    int t3 = t2, t4 = t2;
    std::vector<float> gate_host;
    std::vector<double> val_e2;      // squared error of the corrected prediction on the validation columns
    int n_val_lines_used = 0;
    if (o.network) {
        // validation lines: a seeded val_frac share of the train lines
        std::vector<int> line_idx(n_tr);
        std::iota(line_idx.begin(), line_idx.end(), 0);
        std::shuffle(line_idx.begin(), line_idx.end(), rng);
        const int n_val_lines = std::min(n_tr - 1, std::max(1, (int)std::lround(o.val_frac * n_tr)));
        std::vector<char> is_val(n_tr, 0);
        for (int i = 0; i < n_val_lines; ++i) is_val[line_idx[i]] = 1;
        std::vector<int> fit, val, col_vox(n_trc);
        for (int c = 0; c < n_tr; ++c)
            for (int y = 0; y < ny; ++y) {
                const int j = c * ny + y;
                col_vox[j] = cols[c].x + nx * (y + ny * cols[c].y);
                (is_val[c] ? val : fit).push_back(j);
            }
        S.n_val_columns = (int)val.size();
        std::vector<int> val_vox;
        for (int j : val) val_vox.push_back(col_vox[j]);
        DevBuf dfit, dval, dcolvox, dvalvox, tgt, batch;
        SM_TRY(upload(dfit, fit, s, "fit columns"));
        SM_TRY(upload(dval, val, s, "validation columns"));
        SM_TRY(upload(dcolvox, col_vox, s, "column voxels"));
        SM_TRY(upload(dvalvox, val_vox, s, "validation voxels"));
        // targets over the train block: rho = log(Y / B), weight (Y / rms_d)^2
        std::vector<double> tr_err, tr_norm2;
        SM_TRY(row_errors(dB, ldy, dY, ldy, N, n_trc, s, &tr_err, &tr_norm2));
        DevBuf dnorm;
        SM_TRY(upload(dnorm, tr_norm2, s, "row norms"));
        SM_TRY(tgt.alloc(sizeof(float) * 2 * (size_t)N * n_trc, s, "training targets"));
        float* rho = static_cast<float*>(tgt.p);
        float* wgt = rho + (size_t)N * n_trc;
        SM_CUDA(launch_prep_targets(dY, dB, ldy, N, n_trc, static_cast<const double*>(dnorm.p), rho, wgt, n_trc, s));
        NetShape shp;
        shp.layers = o.layers;
        shp.width = o.width;
        shp.freqs = o.freqs;
        shp.emb = o.emb;
        shp.n_crystals = N;
        shp.nx = nx;
        shp.ny = ny;
        shp.nz = nz;
        SurrogateNet net;
        SM_TRY(net.init(shp, o.seed ^ 0x5eedULL, s));
        const int Bsz = o.batch;
        SM_TRY(batch.alloc(sizeof(int) * 2 * (size_t)Bsz, s, "batch"));
        int* bcol = static_cast<int*>(batch.p);
        int* bvox = bcol + Bsz;
        for (int it = 0; it < o.steps; ++it) {
            SM_CUDA(launch_sample_batch(o.seed, it, Bsz, static_cast<const int*>(dfit.p), (int)fit.size(),
                                        static_cast<const int*>(dcolvox.p), bcol, bvox, s));
            SM_CUDA(cudaMemsetAsync(net.loss, 0, sizeof(double), s));
            SM_TRY(net.forward_backward(bvox, bcol, Bsz, rho, wgt, n_trc, s));
            if (it == 0) SM_CUDA(cudaMemcpyAsync(&S.first_loss, net.loss, sizeof(double), cudaMemcpyDeviceToHost, s));
            // warm-up over the first 5 %, then cosine decay
            const double f = (double)it / std::max(1, o.steps - 1);
            const double warm = std::min(1.0, (it + 1) / std::max(1.0, 0.05 * o.steps));
            const float lr = (float)(o.lr * warm * 0.5 * (1.0 + std::cos(3.14159265358979323846 * f)));
            SM_TRY(net.adam(lr, s));
        }
        SM_CUDA(cudaMemcpyAsync(&S.final_loss, net.loss, sizeof(double), cudaMemcpyDeviceToHost, s));
        t3 = tm.mark();
        // validation: B exp(rho) vs B on the validation columns, per row
        const int nv = (int)val.size();
        DevBuf vb;
        SM_TRY(vb.alloc(sizeof(float) * 3 * (size_t)N * nv, s, "validation"));
        float* vB = static_cast<float*>(vb.p);
        float* vY = vB + (size_t)N * nv;
        float* vP = vY + (size_t)N * nv;
        SM_CUDA(launch_gather_idx(dB, ldy, N, static_cast<const int*>(dval.p), nv, vB, nv, s));
        SM_CUDA(launch_gather_idx(dY, ldy, N, static_cast<const int*>(dval.p), nv, vY, nv, s));
        SM_CUDA(cudaMemcpyAsync(vP, vB, sizeof(float) * (size_t)N * nv, cudaMemcpyDeviceToDevice, s));
        std::vector<float> ones(N, 1.0f);
        DevBuf dgate;
        SM_TRY(upload(dgate, ones, s, "gate"));
        SM_TRY(net.predict(static_cast<const int*>(dvalvox.p), nv, vP, nv, static_cast<const float*>(dgate.p), s));
        std::vector<double> e_base, q;
        SM_TRY(row_sums(vP, nv, vY, nv, N, nv, s, &val_e2, &q));
        SM_TRY(row_sums(vB, nv, vY, nv, N, nv, s, &e_base, &q));
        n_val_lines_used = n_val_lines;
        // matrix gate: the correction must lower the mean relative squared error of
        // the rows on the validation columns by a fifth; row gate: the same per row
        double rel_net = 0.0, rel_base = 0.0;
        for (int d = 0; d < N; ++d)
            if (q[d] > 0.0) {
                rel_net += val_e2[d] / q[d];
                rel_base += e_base[d] / q[d];
            }
        S.val_gain = rel_base > 0.0 ? 1.0 - rel_net / rel_base : 0.0;
        std::vector<float> gate(N, 0.0f);
        if (rel_net < 0.81 * rel_base)
            for (int d = 0; d < N; ++d)
                if (val_e2[d] < 0.81 * e_base[d]) {
                    gate[d] = 1.0f;
                    ++S.rows_corrected;
                }
        SM_CUDA(cudaMemcpyAsync(dgate.p, gate.data(), sizeof(float) * N, cudaMemcpyHostToDevice, s));
        gate_host = gate;
        if (S.rows_corrected > 0) {
            SM_TRY(net.predict(nullptr, (int)V, d_dst, ld, static_cast<const float*>(dgate.p), s));
            // the held-out columns of the prediction
            SM_CUDA(launch_gather_columns(d_dst, ld, N, static_cast<const int2*>(dcols.p) + n_tr, n_ho, nx, ny,
                                          dB + n_trc, ldy, s));
        }
        int gemm_err = 0;
        SM_CUDA(cudaMemcpyAsync(&gemm_err, net.error, sizeof(int), cudaMemcpyDeviceToHost, s));
        SM_CUDA(cudaStreamSynchronize(s));
        if (gemm_err) return fail(SM_ERR_CUDA, "surrogate network: a tensor-core wait ran out");
        t4 = tm.mark();
    }

    // corrected rows: squared error on the held-out columns; with the validation
    // columns (not fitted; they chose the correction) they sample those rows
    std::vector<double> c_e2;
    if (S.rows_corrected > 0) {
        std::vector<double> c_q2;
        SM_TRY(row_sums(dB + n_trc, ldy, dY + n_trc, ldy, N, n_hoc, s, &c_e2, &c_q2));
    }
    // exact entries replace the prediction where they exist; the collimator part is exact everywhere
    SM_CUDA(launch_scatter_columns(dY, ldy, N, static_cast<const int2*>(dcols.p), n_tr + n_ho, nx, ny, d_dst, ld, s));
    const int t5 = tm.mark();
    if (o.parts & 2) {
        ExactSpec spec;
        spec.row0 = 0;
        spec.row1 = N;
        spec.accumulate = true;
        SM_TRY(exact_scatter(geo, o.sp, 2, angle, nullptr, 0, nullptr, nullptr, spec, d_dst, ld, s));
    }
    const int t6 = tm.mark();

    // ---- 4. per-row check of the output rows ----
    // estimate = sqrt(squared error on the sampled columns scaled to the row / squared norm of the output row);
    // baseline rows are sampled by every exactly computed column (the baseline used none of them)
    std::vector<double> pn2, est(N), base_est(N);
    SM_TRY(row_sums(d_dst, ld, d_dst, ld, N, V, s, &dummy, &pn2));
    for (int d = 0; d < N; ++d) {
        base_est[d] = row_estimate(tr_e2[d] + ho_e2[d], n_tr + n_ho, nx * nz, pn2[d]);
        est[d] = (!gate_host.empty() && gate_host[d] > 0.0f)
                     ? row_estimate(c_e2[d] + val_e2[d], n_ho + n_val_lines_used, nx * nz, pn2[d])
                     : base_est[d];
    }
    S.baseline_holdout_median = quantile(base_est, 0.5);
    S.holdout_median = quantile(est, 0.5);
    S.holdout_p90 = quantile(est, 0.9);
    S.holdout_max = *std::max_element(est.begin(), est.end());
    std::vector<int> redo;
    for (int d = 0; d < N; ++d)
        if (!(est[d] <= o.tol)) redo.push_back(d);
    S.rows_recomputed = (int)redo.size();
    if (row_error)
        for (int d = 0; d < N; ++d) row_error[d] = (float)est[d];
    if (row_state) {
        for (int d = 0; d < N; ++d) row_state[d] = gate_host.empty() ? 0 : (gate_host[d] > 0.0f ? 1 : 0);
        for (int d : redo) row_state[d] = 2;
    }
    const int t7 = tm.mark();

    // ---- 5. exact recompute of the rows over tolerance (every part, in place) ----
    if (!redo.empty()) {
        ExactSpec spec;
        spec.rows = &redo;
        spec.rows_in_place = true;
        spec.pairs = d_pairs;
        spec.pairs_order = &order_all;
        SM_TRY(exact_scatter(geo, o.sp, o.parts, angle, d_pe, ld_pe, nullptr, nullptr, spec, d_dst, ld, s));
    }
    const int t8 = tm.mark();
    int base_err_flag = 0;
    SM_CUDA(cudaMemcpyAsync(&base_err_flag, err_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SM_CUDA(cudaStreamSynchronize(s));
    if (base_err_flag) return fail(SM_ERR_CUDA, "surrogate baseline: a tensor-core wait ran out");
    S.ms_pairs = tm.ms(t0, tp);
    S.ms_exact_subsets = tm.ms(tp, t1);
    S.ms_baseline = tm.ms(t1, t2);
    S.ms_train = tm.ms(t2, t3);
    S.ms_correct = tm.ms(t3, t4);
    S.ms_verify = tm.ms(t4, t5) + tm.ms(t6, t7);
    S.ms_collimator = tm.ms(t5, t6);
    S.ms_recompute = tm.ms(t7, t8);
    S.ms_total = tm.ms(t0, t8);
    if (st) *st = S;
    return SM_OK;
}

}  // namespace smb

using namespace smb;

struct sm_surrogate_net {
    sm_context* ctx = nullptr;
    SurrogateNet net;
};

extern "C" {

void sm_surrogate_options_default(sm_surrogate_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->sp[0] = 2;
    o->sp[1] = 4;
    o->sp[2] = 2;
    o->parts = 3;
    o->train_frac = 0.05f;
    o->holdout_frac = 0.005f;
    o->val_frac = 0.2f;
    o->tol = 0.01f;
    o->anchors[0] = 12;
    o->anchors[1] = 6;
    o->anchors[2] = 12;
    o->network = 1;
    o->layers = 6;
    o->width = 256;
    o->freqs = 16;
    o->emb = 64;
    o->steps = 600;
    o->batch = 512;
    o->lr = 2e-3f;
    o->seed = 1;
}

int sm_scatter_surrogate(sm_context* ctx, const sm_geometry* geo, const sm_surrogate_options* o, int rotation,
                         const float* pe, int64_t ld_pe, float* dst, int64_t ld, float* row_error, int32_t* row_state,
                         sm_surrogate_stats* stats, void* stream) {
    if (!geo || !o || !pe || !dst) return fail(SM_ERR_INVALID, "null argument");
    SM_TRY(context_bind(ctx));
    const HostGeometry& g = geo->host;
    const int64_t V = (int64_t)g.nx * g.ny * g.nz;
    if (ld < V || ld_pe < V) return fail(SM_ERR_INVALID, "ld and ld_pe must be at least the %lld voxels", (long long)V);
    for (int a = 0; a < 3; ++a)
        if (o->sp[a] < 1 || o->sp[a] > 16) return fail(SM_ERR_INVALID, "sp[%d] = %d must be in 1..16", a, o->sp[a]);
    if (o->parts != 1 && o->parts != 3) return fail(SM_ERR_INVALID, "parts must be 1 or 3");
    if (!(o->train_frac > 0.0f && o->train_frac < 1.0f) || !(o->holdout_frac > 0.0f && o->holdout_frac < 1.0f) ||
        o->train_frac + o->holdout_frac >= 1.0f)
        return fail(SM_ERR_INVALID, "train_frac and holdout_frac must be in (0, 1) with a sum below 1");
    if (!(o->tol > 0.0f)) return fail(SM_ERR_INVALID, "tol must be > 0");
    if ((int64_t)g.nx * g.nz < 3) return fail(SM_ERR_INVALID, "the image needs at least 3 voxel columns");
    for (int a = 0; a < 3; ++a)
        if (o->anchors[a] < 1 || o->anchors[a] > 64) return fail(SM_ERR_INVALID, "anchors[%d] must be in 1..64", a);
    const int64_t A = (int64_t)o->anchors[0] * o->anchors[1] * o->anchors[2];
    if (A * (int64_t)sizeof(float4) > 200 * 1024) return fail(SM_ERR_CAPACITY, "anchor grid too large (%lld)", (long long)A);
    if (o->network) {
        if (o->layers < 1 || o->layers > 16 || o->width < 16 || o->width > 1024 || o->width % 16 || o->freqs < 1 ||
            o->freqs > 64 || o->emb < 8 || o->emb > 512 || o->emb % 8 || o->steps < 0 || o->batch < 16 ||
            o->batch > 8192 || o->batch % 8 || !(o->val_frac > 0.0f && o->val_frac < 1.0f))
            return fail(SM_ERR_INVALID, "network options out of range");
    }
    if ((int64_t)g.n_crystals * g.n_crystals * 2 * A > (int64_t)64 << 30)
        return fail(SM_ERR_CAPACITY, "transfer matrices would take over 64 GB");
    const float angle = (float)rotation * g.angle_per_rotation;
    return scatter_surrogate(geo, *o, angle, pe, ld_pe, dst, ld, row_error, row_state, stats, (cudaStream_t)stream);
}

int sm_surrogate_columns(const sm_geometry* geo, const sm_surrogate_options* o, int32_t* xz, int* n_train,
                         int* n_holdout) {
    if (!geo || !o || !n_train || !n_holdout) return fail(SM_ERR_INVALID, "null argument");
    if ((int64_t)geo->host.nx * geo->host.nz < 3) return fail(SM_ERR_INVALID, "the image needs at least 3 voxel columns");
    std::mt19937_64 rng(o->seed);
    std::vector<int2> cols;
    select_columns(geo->host, *o, rng, &cols, n_train, n_holdout);
    if (xz)
        for (size_t i = 0; i < cols.size(); ++i) {
            xz[2 * i] = cols[i].x;
            xz[2 * i + 1] = cols[i].y;
        }
    return SM_OK;
}

int sm_surrogate_net_create(sm_context* ctx, int n_crystals, int nx, int ny, int nz, int layers, int width, int freqs,
                            int emb, uint64_t seed, sm_surrogate_net** out) {
    if (!out) return fail(SM_ERR_INVALID, "null argument");
    *out = nullptr;
    if (n_crystals < 1 || nx < 1 || ny < 1 || nz < 1 || layers < 1 || layers > 16 || width < 16 || width % 16 ||
        freqs < 1 || freqs > 64 || emb < 8 || emb % 8)
        return fail(SM_ERR_INVALID, "network shape out of range");
    SM_TRY(context_bind(ctx));
    auto* h = new sm_surrogate_net();
    h->ctx = ctx;
    NetShape s;
    s.layers = layers;
    s.width = width;
    s.freqs = freqs;
    s.emb = emb;
    s.n_crystals = n_crystals;
    s.nx = nx;
    s.ny = ny;
    s.nz = nz;
    const int rc = h->net.init(s, seed, nullptr);
    if (rc != SM_OK) {
        delete h;
        return rc;
    }
    *out = h;
    return SM_OK;
}

int sm_surrogate_net_layout(const sm_surrogate_net* h, int64_t* n_params, int64_t* offsets) {
    if (!h) return fail(SM_ERR_INVALID, "null argument");
    if (n_params) *n_params = h->net.n_params;
    if (offsets)
        for (size_t i = 0; i < h->net.off.size(); ++i) offsets[i] = h->net.off[i];
    return SM_OK;
}

int sm_surrogate_net_get(sm_surrogate_net* h, float* params) {
    if (!h || !params) return fail(SM_ERR_INVALID, "null argument");
    SM_TRY(context_bind(h->ctx));
    SM_CUDA(cudaMemcpy(params, h->net.w, sizeof(float) * h->net.n_params, cudaMemcpyDeviceToHost));
    return SM_OK;
}

int sm_surrogate_net_set(sm_surrogate_net* h, const float* params) {
    if (!h || !params) return fail(SM_ERR_INVALID, "null argument");
    SM_TRY(context_bind(h->ctx));
    return h->net.set_params(params, nullptr);
}

int sm_surrogate_net_loss_grad(sm_surrogate_net* h, const int32_t* vox, const int32_t* col, int B, const float* rho,
                               const float* wgt, int64_t ld, double* loss, float* grad) {
    if (!h || !vox || !col || !rho || !wgt || B < 1) return fail(SM_ERR_INVALID, "null argument or empty batch");
    SM_TRY(context_bind(h->ctx));
    const NetShape& s = h->net.shape;
    const int64_t V = (int64_t)s.nx * s.ny * s.nz;
    for (int j = 0; j < B; ++j)
        if (vox[j] < 0 || vox[j] >= V || col[j] < 0 || col[j] >= ld)
            return fail(SM_ERR_INVALID, "batch entry %d out of range", j);
    const int N = s.n_crystals;
    cudaStream_t st = nullptr;
    DevBuf idx, tg;
    SM_TRY(idx.alloc(sizeof(int) * 2 * (size_t)B, st, "batch"));
    SM_CUDA(cudaMemcpy(idx.p, vox, sizeof(int) * B, cudaMemcpyHostToDevice));
    SM_CUDA(cudaMemcpy(static_cast<int*>(idx.p) + B, col, sizeof(int) * B, cudaMemcpyHostToDevice));
    SM_TRY(tg.alloc(sizeof(float) * 2 * (size_t)N * ld, st, "targets"));
    float* drho = static_cast<float*>(tg.p);
    float* dw = drho + (size_t)N * ld;
    SM_CUDA(cudaMemcpy(drho, rho, sizeof(float) * (size_t)N * ld, cudaMemcpyHostToDevice));
    SM_CUDA(cudaMemcpy(dw, wgt, sizeof(float) * (size_t)N * ld, cudaMemcpyHostToDevice));
    SM_CUDA(cudaMemset(h->net.loss, 0, sizeof(double)));
    SM_CUDA(cudaMemset(h->net.grad, 0, sizeof(float) * h->net.n_params));
    SM_TRY(h->net.forward_backward(static_cast<const int*>(idx.p), static_cast<const int*>(idx.p) + B, B, drho, dw, ld,
                                   st));
    SM_CUDA(cudaStreamSynchronize(st));
    int e = 0;
    SM_CUDA(cudaMemcpy(&e, h->net.error, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return fail(SM_ERR_CUDA, "a tensor-core wait ran out");
    if (loss) SM_CUDA(cudaMemcpy(loss, h->net.loss, sizeof(double), cudaMemcpyDeviceToHost));
    if (grad) SM_CUDA(cudaMemcpy(grad, h->net.grad, sizeof(float) * h->net.n_params, cudaMemcpyDeviceToHost));
    return SM_OK;
}

int sm_surrogate_net_adam(sm_surrogate_net* h, float lr) {
    if (!h) return fail(SM_ERR_INVALID, "null argument");
    SM_TRY(context_bind(h->ctx));
    SM_TRY(h->net.adam(lr, nullptr));
    SM_CUDA(cudaDeviceSynchronize());
    return SM_OK;
}

int sm_surrogate_net_predict(sm_surrogate_net* h, const int32_t* vox, int n, float* out) {
    if (!h || !vox || !out || n < 1) return fail(SM_ERR_INVALID, "null argument or empty list");
    SM_TRY(context_bind(h->ctx));
    const NetShape& s = h->net.shape;
    const int64_t V = (int64_t)s.nx * s.ny * s.nz;
    for (int j = 0; j < n; ++j)
        if (vox[j] < 0 || vox[j] >= V) return fail(SM_ERR_INVALID, "voxel %d out of range", j);
    cudaStream_t st = nullptr;
    DevBuf idx, o;
    SM_TRY(idx.alloc(sizeof(int) * (size_t)n, st, "voxels"));
    SM_CUDA(cudaMemcpy(idx.p, vox, sizeof(int) * n, cudaMemcpyHostToDevice));
    SM_TRY(o.alloc(sizeof(float) * (size_t)s.n_crystals * n, st, "prediction"));
    SM_TRY(h->net.predict(static_cast<const int*>(idx.p), n, static_cast<float*>(o.p), n, nullptr, st));
    SM_CUDA(cudaStreamSynchronize(st));
    SM_CUDA(cudaMemcpy(out, o.p, sizeof(float) * (size_t)s.n_crystals * n, cudaMemcpyDeviceToHost));
    return SM_OK;
}

int sm_surrogate_net_apply(sm_surrogate_net* h, const int32_t* vox, int n, const float* gate, float* inout) {
    if (!h || !vox || !gate || !inout || n < 1) return fail(SM_ERR_INVALID, "null argument or empty list");
    SM_TRY(context_bind(h->ctx));
    const NetShape& s = h->net.shape;
    const int64_t V = (int64_t)s.nx * s.ny * s.nz;
    for (int j = 0; j < n; ++j)
        if (vox[j] < 0 || vox[j] >= V) return fail(SM_ERR_INVALID, "voxel %d out of range", j);
    cudaStream_t st = nullptr;
    DevBuf idx, o, gt;
    const size_t bytes = sizeof(float) * (size_t)s.n_crystals * n;
    SM_TRY(idx.alloc(sizeof(int) * (size_t)n, st, "voxels"));
    SM_TRY(o.alloc(bytes, st, "values"));
    SM_TRY(gt.alloc(sizeof(float) * (size_t)s.n_crystals, st, "gate"));
    SM_CUDA(cudaMemcpy(idx.p, vox, sizeof(int) * n, cudaMemcpyHostToDevice));
    SM_CUDA(cudaMemcpy(o.p, inout, bytes, cudaMemcpyHostToDevice));
    SM_CUDA(cudaMemcpy(gt.p, gate, sizeof(float) * s.n_crystals, cudaMemcpyHostToDevice));
    SM_TRY(h->net.predict(static_cast<const int*>(idx.p), n, static_cast<float*>(o.p), n,
                          static_cast<const float*>(gt.p), st));
    SM_CUDA(cudaStreamSynchronize(st));
    SM_CUDA(cudaMemcpy(inout, o.p, bytes, cudaMemcpyDeviceToHost));
    return SM_OK;
}

int sm_surrogate_net_destroy(sm_surrogate_net* h) {
    if (!h) return SM_OK;
    context_bind(h->ctx);
    delete h;
    return SM_OK;
}

}  // extern "C"
