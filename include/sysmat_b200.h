/* sysmat_b200 -- B200 (sm_100a) SPECT/PET system-matrix generator, C ABI.
 *
 * Two layers of entry points:
 *
 * 1. Legacy drop-ins with the reference's exact signatures and semantics
 *    (host buffers, tables of at least 80000 / 80000 / 100 / 100 floats,
 *    return value = voxels per row, device chosen per call):
 *      PESysMatGen   replaces PEGen_RayTracing_CircularHole/PESysMatGen.h:4-9
 *      scatter       replaces ScatterGen_RayTracing_CircularHole/scatter.h:4-5
 *    The crystal-only and collimator-only `scatter` variants of
 *    ScatterGen_Crystal/scatter.h:4 and ScatterGen_Collimator/scatter.h:4-5 share
 *    the symbol name, so they live in the two small shim libraries
 *    libsysmat_b200_scatter_crystal.so / libsysmat_b200_scatter_collimator.so.
 *    Unlike the reference, they never call exit(): on failure they print the
 *    reason to stderr and return -1.
 *
 * 2. The status-returning sm_* API: explicit table lengths, sub-sampling
 *    options, device or host outputs, a caller stream, and no process exit.
 *    Every sm_* function returns SM_OK (0) or a negative SM_ERR_* code;
 *    sm_last_error() gives the message of the calling thread's last failure.
 *
 * Conventions: tables are the reference's float32 Params layouts (Y = depth);
 * sysmat rows are crystals, columns are voxels x + nx*(y + ny*z); a "slab" is the
 * voxel range z in [z0, z0 + nz) and occupies nx*ny*nz consecutive columns.
 */
#ifndef SYSMAT_B200_H
#define SYSMAT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- legacy drop-ins ------------------------------------------------------ */

/* PEGen_RayTracing_CircularHole/PESysMatGen.h:4-9 and PESysMatGen.cu:766-833.
 * Computes the photoelectric sysmat of one z-slab for rotation Image[20]:
 * rows = all crystals, columns = the slab of Image[2] z-planes starting at
 * Image[31] in a volume of Image[30] z-planes.  dst is host memory of
 * N * nx * ny * Image[2] floats.  Crystal sub-cells 8 x 16 x 8, voxel centre
 * only, as the reference.  Returns nx * ny * Image[2], or -1 on failure. */
int PESysMatGen(float* parameter_Collimator, float* parameter_Detector, float* parameter_Image,
                float* dst, int cuda_id);

/* ScatterGen_RayTracing_CircularHole/scatter.h:4-5 and scatter.cu:2013-2378.
 * Primary Compton scatter (crystal + collimator parts) for rotation Image[20];
 * PE_SysMat is the host PE sysmat of that rotation ([N][V]); dst receives
 * [N][V].  Physics[8] / Physics[9] == 1 compute the geometry bitmaps and write
 * them to FnameGeoCrystal / FnameGeoCollimator, otherwise they are read from
 * those files.  Returns V, or -1 on failure. */
#ifndef SYSMAT_B200_SINGLE_PART_SCATTER   /* defined by the two single-part shim libraries */
int scatter(float* parameter_Collimator, float* parameter_Detector, float* parameter_Image,
            float* parameter_Physics, float* PE_SysMat, const char* FnameGeoCrystal,
            const char* FnameGeoCollimator, float* dst, int cuda_id);
#endif

/* ---- status codes ---------------------------------------------------------- */
enum {
    SM_OK = 0,
    SM_ERR_INVALID = -1,     /* bad argument or malformed table            */
    SM_ERR_CAPACITY = -2,    /* a table or tile exceeds a supported size   */
    SM_ERR_CUDA = -3,        /* CUDA runtime error                         */
    SM_ERR_ALLOC = -4,       /* device or host allocation failed           */
    SM_ERR_IO = -5,          /* file open/read/write failed                */
    SM_ERR_TIMEOUT = -6,     /* a bounded device-side wait expired         */
    SM_ERR_DEVICE = -7       /* no usable sm_100 device                    */
};

const char* sm_last_error(void);
const char* sm_version(void);

/* ---- context and geometry -------------------------------------------------- */
typedef struct sm_context sm_context;
typedef struct sm_geometry sm_geometry;

/* Binds a CUDA device (cudaSetDevice on every call that launches work). */
int sm_context_create(int device, sm_context** out);
int sm_context_destroy(sm_context* ctx);
/* Device workspaces of a context's calls come from its own memory pool, which
 * keeps freed memory mapped for the next call (no unmapping at every
 * synchronisation).  sm_context_trim returns that memory to the device;
 * sm_context_destroy does too. */
int sm_context_trim(sm_context* ctx);
/* Waits for `stream` and reports any device-side status raised by kernels of
 * this context since the last check (e.g. SM_ERR_CAPACITY). */
int sm_context_sync(sm_context* ctx, void* stream);

/* Parses and validates the four tables (lengths in floats), uploads the
 * derived structure-of-arrays geometry to the context's device once.
 * Validation errors name the offending field. */
int sm_geometry_create(sm_context* ctx, const float* collimator, size_t n_collimator,
                       const float* detector, size_t n_detector, const float* image, size_t n_image,
                       const float* physics, size_t n_physics, sm_geometry** out);
int sm_geometry_destroy(sm_geometry* geo);
/* Host only, no device needed: the parse and validation of sm_geometry_create
 * (the checks the reference's table readers never make: counts that need
 * more floats than a table holds, e.g. a truncated Params_*.dat, plate and
 * crystal sizes, grid).  out (may be NULL) as sm_geometry_info. */
int sm_tables_check(const float* collimator, size_t n_collimator, const float* detector, size_t n_detector,
                    const float* image, size_t n_image, const float* physics, size_t n_physics, int64_t out[7]);
/* n_crystals, n_holes, n_plates, nx, ny, nz, n_rotations */
int sm_geometry_info(const sm_geometry* geo, int64_t out[7]);

/* ---- photoelectric sysmat -------------------------------------------------- */
typedef struct sm_pe_options {
    int sv[3];          /* voxel sub-samples (x, y, z); the entry is their mean  */
    int sc[3];          /* crystal sub-cells (x, y = depth, z); summed           */
    int tile_voxels[3]; /* voxel brick per CTA; 0 = default (8 x 4 x 4)          */
    int flags;          /* SM_PE_AUTOTUNE: choose tile_voxels and group with sm_pe_autotune */
    int group;          /* voxel sub-points whose rays a warp traces together (each lane
                           traces group * sc[0]*sc[1]*sc[2] / 32 of them); 0 = 32 / sc[1],
                           at most 8: one warp pass then covers one column of depth
                           sub-cells.  It changes which lane sums which ray, so the
                           rounding of the sums, never a hit decision. */
} sm_pe_options;

enum { SM_PE_AUTOTUNE = 1 };

/* Reference mode: sv = 1x1x1, sc = 8x16x8 (PESysMatGen.cu:435-440). */
void sm_pe_options_reference(sm_pe_options* opt);

/* Photoelectric sysmat for rows [row0, row1) and the voxel slab z in
 * [z0, z0 + nz) of rotation `rotation`.  dst[(r - row0) * ld + c] receives
 * column c of the slab (c < nx*ny*nz); ld >= nx*ny*nz.  dst is a device
 * pointer when dst_on_device != 0 (the call is asynchronous on `stream`),
 * otherwise host memory (the call copies and synchronises).  stream may be
 * NULL (legacy default stream). */
int sm_pe_compute(sm_context* ctx, const sm_geometry* geo, const sm_pe_options* opt, int rotation,
                  int row0, int row1, int z0, int nz, float* dst, int64_t ld, int dst_on_device,
                  void* stream);

/* No counterpart in the reference.  sm_pe_compute for callers that cannot
 * allocate device memory: a host application that routes every device byte
 * through its own pool or arena and forbids other allocators, a plugin loaded
 * into such a process, or code that must not take the device-wide
 * synchronisation cudaMalloc / cudaFree can cause.  It calls no cudaMalloc,
 * cudaFree or other allocating routine: its working memory (derived geometry
 * and status word) is a fixed 4 MiB __device__ array inside the library,
 * held on every GPU that loads the library until the process exits.
 *   - Tables are host arrays (lengths in floats) as for sm_geometry_create;
 *     dst is device memory of the current device, dst[(r - row0) * ld + c]
 *     as for sm_pe_compute; the call runs on the calling thread's current
 *     device and on `stream` (NULL = legacy default stream).
 *   - Geometries whose derived tables exceed the array (about 40000 crystals
 *     with 2000 holes) are rejected with SM_ERR_CAPACITY.
 *   - The first call on a device looks up the array's device address once
 *     (set-up); make that first call before any stream capture.  The address
 *     is kept until the process exits: do not call this entry point after
 *     cudaDeviceReset of a device it has already run on.
 *   - opt->flags must be 0 (autotuning would allocate: SM_ERR_INVALID); dst
 *     that is host memory or memory of another device is SM_ERR_INVALID.
 *   - Every call shares the one array, which keeps the previous call's
 *     contents; calls overlapping on the GPU would race, so the library runs
 *     one call at a time per process and returns only after its kernel has
 *     finished (it reads back the status word). */
int sm_pe_compute_static(const float* collimator, size_t n_collimator, const float* detector, size_t n_detector,
                         const float* image, size_t n_image, const sm_pe_options* opt, int rotation, int row0,
                         int row1, int z0, int nz, float* dst, int64_t ld, void* stream);

/* Diagnostic: for each listed entry (rows[i], voxels[i] as full-volume voxel
 * index) record every ray's hits exactly as the production kernel decides
 * them.  Per ray, `record_words` int32: [plate-miss mask, n_holes, holes
 * (<= 16), n_crystals, crystals (<= 40)], ids ascending; rays in the order
 * sub-point (x fastest, then y, z) x sub-cell (depth fastest, then x, then
 * z).  out (host) holds n * rays_per_entry * record_words int32. */
int sm_pe_record_hits(sm_context* ctx, const sm_geometry* geo, const sm_pe_options* opt,
                      int rotation, const int64_t* rows, const int64_t* voxels, int64_t n,
                      int32_t* out, int* record_words);

/* Work counters: when enabled, each sm_pe_compute on the context counts rays
 * traced, exact crystal tests, exact hole tests and candidate cone tests
 * (the cone test is taken on the candidates a ray crosses) (costs a little
 * time and synchronises the call). */
int sm_pe_set_counters(sm_context* ctx, int enable);
int sm_pe_last_counters(sm_context* ctx, int64_t out[4]);

/* ---- batched photoelectric sysmats, brick autotuning ------------------------- */
/* No reference counterpart (the reference runs one geometry per process).  A
 * design sweep: many geometries of uneven size computed by one persistent
 * kernel launch that hands out (geometry, tile) work items, largest first,
 * replayed from a CUDA graph. */
typedef struct sm_pe_batch sm_pe_batch;

/* Times candidate voxel bricks and sub-points per pass (out->group) on `geo`
 * (the whole matrix when it is small, else a sample of tiles) and writes the
 * fastest into out->tile_voxels / out->group (out = *opt otherwise).  Results are cached
 * per device and geometry class for the process, and appended to the file
 * named by the environment variable SYSMAT_B200_TUNE_CACHE when it is set.
 * best_ms_per_tile (may be NULL) receives the winner's time, -1 for a cache hit. */
int sm_pe_autotune(sm_context* ctx, const sm_geometry* geo, const sm_pe_options* opt, int rotation,
                   sm_pe_options* out, double* best_ms_per_tile);

/* The whole PE sysmat of each of n geometries (all rows, all voxels, rotation
 * rotations[i] or 0 when rotations is NULL) into device buffers dst[i] with
 * row pitch ld[i].  Options with SM_PE_AUTOTUNE are autotuned here. */
int sm_pe_batch_create(sm_context* ctx, int n, const sm_geometry* const* geos, const sm_pe_options* opts,
                       const int* rotations, float* const* dst, const int64_t* ld, sm_pe_batch** out);
/* out[0] geometries, out[1] work items, out[2] persistent CTAs */
int sm_pe_batch_info(const sm_pe_batch* batch, int64_t out[3]);
/* One launch of the batch on `stream` (asynchronous; sm_context_sync reports
 * device-side capacity errors).  The first call captures the launch in a
 * CUDA graph; later calls replay it. */
int sm_pe_batch_run(sm_pe_batch* batch, void* stream);
int sm_pe_batch_destroy(sm_pe_batch* batch);

/* ---- primary-Compton scatter sysmat ------------------------------------------ */
typedef struct sm_scatter_options {
    int sp[3];   /* scatter points per scatter crystal (x, y = depth, z): sub-cell centres of
                    the crystal, each with an equal share of its Compton probability;
                    1 x 1 x 1 = the crystal centre, as the reference                        */
    int parts;   /* 1: scatter in the crystals, 2: in the plate-0 holes, 3: both (summed)    */
    int flags;   /* reserved, 0                                                              */
} sm_scatter_options;

/* Reference mode: sp = 1 x 1 x 1, both parts (ScatterGen_RayTracing_CircularHole). */
void sm_scatter_options_reference(sm_scatter_options* opt);

/* Sizes in uint32 words of the geometry-relationship bitmaps, in the
 * reference's file format (scatter.cu:2053-2056, :2224-2229): out[0] crystal
 * bitmap (N (N + 1) / 2 pairs x N bits), out[1] collimator bitmap (H0 x N x N
 * bits, H0 = holes of plate 0). */
int sm_scatter_bitmap_words(const sm_geometry* geo, int64_t out[2]);

/* 64-bit FNV-1a hashes of the table values each bitmap depends on: out[0]
 * crystal bitmap (detector records, FOV distance), out[1] collimator bitmap
 * (plate 0's record and holes, detector records, FOV distance).  The legacy
 * scatter path keeps them in "<bitmap file>.geohash" next to the files it
 * writes, and recomputes a bitmap whose .geohash names another geometry
 * instead of reading it (the reference reuses such a stale file); a bitmap
 * file without .geohash is read as the reference reads it. */
int sm_scatter_bitmap_hashes(const sm_geometry* geo, uint64_t out[2]);

/* Computes either bitmap (NULL skips it) into device (on_device != 0, async on
 * `stream`) or host buffers, bit for bit the reference's
 * geometryRelationShip_Crystal2Crystal / _Collimator2Crystal
 * (scatter.cu:1440-1540, :1939-2009). */
int sm_scatter_bitmaps(sm_context* ctx, const sm_geometry* geo, uint32_t* crystal, uint32_t* collimator,
                       int on_device, void* stream);

/* Primary-Compton scatter sysmat of rotation `rotation` for detector rows
 * [row0, row1) and every voxel: dst[(r - row0) * ld + v].  Replaces the
 * kernels crystalScatterSysMatCuda / collimatorScatterSysMatCuda
 * (scatter.cu:1077-1437, :1544-1936).  pe: that rotation's PE sysmat
 * [N][ld_pe] (needed for parts & 1; device when pe_on_device).  Bitmaps:
 * NULL = computed here; else device (bitmaps_on_device) or host words as
 * read from the reference's files.  dst on the device makes the call
 * asynchronous on `stream` when its inputs are on the device too. */
int sm_scatter_compute(sm_context* ctx, const sm_geometry* geo, const sm_scatter_options* opt, int rotation,
                       const float* pe, int64_t ld_pe, int pe_on_device, const uint32_t* crystal_bitmap,
                       const uint32_t* collimator_bitmap, int bitmaps_on_device, int row0, int row1, float* dst,
                       int64_t ld, int dst_on_device, void* stream);

/* Exact scatter on a subset of entries, device buffers: the detector rows
 * rows[0..n_rows) (host list, distinct) against either every voxel (cols
 * NULL: dst[i * ld + v]) or the voxel y-columns whose (x, z) are the host
 * pairs cols[2c], cols[2c + 1] (dst[i * ld + c * ny + y]).  The same kernels
 * and results as sm_scatter_compute on those entries; used to re-check and
 * recompute rows of the scatter surrogate.  Returns once the work is queued
 * on `stream`. */
int sm_scatter_subset(sm_context* ctx, const sm_geometry* geo, const sm_scatter_options* opt, int rotation,
                      const float* pe, int64_t ld_pe, const int32_t* rows, int n_rows, const int32_t* cols,
                      int n_cols, float* dst, int64_t ld, void* stream);

/* Crystal-scatter transfer matrices, device buffers: for each anchor
 * a < n_anchors, K[(a * N + d) * ldk + s] = the crystal-scatter sysmat entry of
 * detector d per unit PE of source crystal s when the photon arrives from the
 * point vbar[4 (a N + s) .. + 2] (fractional voxel indices x, y, z;
 * vbar[4 (a N + s) + 3] > 0 marks a source in use, else K = 0).  The same
 * scatter terms as sm_scatter_compute (scatter points of opt->sp); the
 * scatter surrogate's physics baseline.  Queued on `stream`. */
int sm_scatter_transfer(sm_context* ctx, const sm_geometry* geo, const sm_scatter_options* opt, int rotation,
                        const float* vbar, int n_anchors, float* K, int64_t ldk, void* stream);

/* The reference's three `scatter` host entry points in one:
 *   parts 3: ScatterGen_RayTracing_CircularHole/scatter.h:4-5 (geo_crystal, geo_collimator)
 *   parts 1: ScatterGen_Crystal/scatter.h:4 (collimator table may be NULL; geo_crystal)
 *   parts 2: ScatterGen_Collimator/scatter.h:4-5 (geo_collimator)
 * Host tables of 80000 / 80000 / 100 / 100 floats, PE_SysMat = [N][V] host
 * (the rotation Image[20] selects the image rotation), dst = [N][V] host.
 * Physics[8] / Physics[9] == 1 compute the bitmaps and write them to the
 * files, otherwise the files are read.  Returns V or a negative SM_ERR_*. */
int sm_scatter_legacy(int parts, float* parameter_Collimator, float* parameter_Detector, float* parameter_Image,
                      float* parameter_Physics, float* PE_SysMat, const char* geo_crystal,
                      const char* geo_collimator, float* dst, int cuda_id);

/* ---- scatter surrogate building blocks ----------------------------------------- */
/* No reference counterpart.  BF16 tensor-core GEMM (tcgen05.mma, fp32
 * accumulators in tensor memory) on device buffers of the current device:
 *   C[i][j] = s_i * sum_k A[i][k] B[j][k] (+ bias[j]) (+ C[i][j] if accumulate)
 * with A[i][k] = a[i * a_ms + k * a_ks], B[j][k] = b[j * b_ns + k * b_ks]
 * (bf16, any strides; k-contiguous operands load fastest), C fp32 row-major
 * with pitch ldc, s_i = row_scale[i] or alpha.  n_tile (64 / 128 / 256) is
 * the column width per CTA.  error (device int, may be NULL) is set to 1 if
 * the kernel's bounded wait on its own MMAs ran out.  Asynchronous on stream. */
int sm_gemm_bf16(int m, int n, int k, const void* a, int64_t a_ms, int64_t a_ks, const void* b, int64_t b_ns,
                 int64_t b_ks, float* c, int64_t ldc, float alpha, const float* row_scale, const float* bias,
                 int accumulate, int n_tile, int* error, void* stream);

/* The bound on every wait of sm_gemm_bf16 (and of the surrogate network's
 * GEMMs) for its own MMAs: mbarrier polls before the kernel gives up, sets
 * *error, skips its epilogue, waits (bounded by the default) for MMAs still in
 * flight, frees its tensor memory and returns.  Process-wide; applies to
 * launches after the call.  polls < 0 restores the default (2^26); 0 makes
 * every wait give up at once (for testing the error path).  previous (may be
 * NULL) receives the limit in force before. */
int sm_tc_wait_limit(int64_t polls, int64_t* previous);

/* ---- scatter surrogate ------------------------------------------------------------ */
/* No reference counterpart.  The crystal-scatter sysmat from a physics
 * baseline plus a learned correction, verified against the exact kernels:
 *  1. exact crystal scatter on a seeded train_frac of the voxel y-columns
 *     (x, z) and, separately, on a seeded holdout_frac of them, every row;
 *  2. baseline B[d][v] = sum_a w_a(v) sum_s K_a[d][s] PE[s][v]: transfer
 *     matrices K_a (sm_scatter_transfer) at an anchors[0] x [1] x [2] grid,
 *     each source evaluated at the PE-weighted centroid of its voxels under
 *     the anchor's trilinear weight w_a, contracted on the tensor cores;
 *  3. (network != 0) a coordinate MLP rho(d, v) = g(d) . h(v) (Fourier
 *     features of the voxel, `freqs` per axis; `layers` x `width`; crystal
 *     embedding of `emb`) trained by Adam on log(S / B) of the train columns
 *     (minus a val_frac share kept for validation), weighted by (S / rms_d)^2;
 *     if it lowers the rows' mean relative squared error on the validation
 *     columns by a fifth, row d uses B exp(rho) where that lowers its own
 *     squared error there by a fifth, else B;
 *  4. the exact train and held-out entries are written in place of the
 *     prediction; parts & 2 adds the exact collimator scatter;
 *  5. each output row's relative L2 error is estimated from exactly computed
 *     columns the prediction was not fitted to (rows with the correction: the
 *     validation and held-out ones; other rows: every one): the sampled
 *     squared error scaled to the whole row, over the squared norm of the
 *     output row; rows above `tol` are recomputed exactly (every part, all
 *     voxels).
 * pe: the rotation's PE sysmat [N][ld_pe] and dst [N][ld], device buffers.
 * Synchronous on `stream`. */
typedef struct sm_surrogate_options {
    int sp[3];             /* scatter points per scatter crystal (as sm_scatter_options)       */
    int parts;             /* 1: crystal scatter, 3: crystal + collimator                     */
    float train_frac;      /* share of voxel columns computed exactly for training (0.05)     */
    float holdout_frac;    /* share computed exactly for the per-row check (0.005)            */
    float val_frac;        /* share of the train columns kept for validation (0.2)            */
    float tol;             /* per-row relative L2 error above which a row is recomputed (0.01) */
    int anchors[3];        /* baseline anchor grid (12, 6, 12)                                 */
    int network;           /* 1: learned correction, 0: baseline only                         */
    int layers, width, freqs, emb;   /* network shape (6, 256, 16, 64)                         */
    int steps, batch;      /* Adam steps and voxels per batch (600, 512)                      */
    float lr;              /* Adam step size (2e-3)                                           */
    uint64_t seed;
} sm_surrogate_options;

typedef struct sm_surrogate_stats {
    double ms_total;       /* phases: */
    double ms_pairs;       /* the crystal pair table shared by every exact and transfer step  */
    double ms_exact_subsets, ms_baseline, ms_transfer /* part of ms_baseline */, ms_train, ms_correct, ms_verify,
        ms_recompute, ms_collimator;
    int n_train_columns, n_holdout_columns, n_val_columns;
    int rows_corrected;    /* rows that use the learned correction                         */
    int rows_recomputed;   /* rows over tol on the held-out columns, recomputed exactly    */
    double holdout_median, holdout_p90, holdout_max;     /* per-row held-out error before recompute */
    double baseline_holdout_median;                       /* ... of the baseline alone            */
    double first_loss, final_loss;   /* training loss at the first and the last step         */
    double val_gain;       /* 1 - (mean relative squared validation error with the correction / without) */
} sm_surrogate_stats;

void sm_surrogate_options_default(sm_surrogate_options* opt);
/* row_error (host, N floats, may be NULL): each row's held-out relative L2
 * error before recompute; row_state (host, N, may be NULL): 0 predicted by the
 * baseline, 1 predicted with the learned correction, 2 recomputed exactly. */
int sm_scatter_surrogate(sm_context* ctx, const sm_geometry* geo, const sm_surrogate_options* opt, int rotation,
                         const float* pe, int64_t ld_pe, float* dst, int64_t ld, float* row_error, int32_t* row_state,
                         sm_surrogate_stats* stats, void* stream);
/* The seeded voxel y-columns a run with these options computes exactly:
 * n_train train columns then n_holdout held-out ones, as (x, z) pairs in xz
 * (host, 2 (n_train + n_holdout) ints; NULL returns the counts only). */
int sm_surrogate_columns(const sm_geometry* geo, const sm_surrogate_options* opt, int32_t* xz, int* n_train,
                         int* n_holdout);

/* The network alone, for training checks: host buffers, synchronous.
 * Parameters are one fp32 vector: for l < layers W_l [width][in_l] and b_l
 * [width] (in_0 = 6 freqs), then E [N][emb], P [width][emb], b_P [width];
 * offsets[2 * layers + 3] gives each block's start. */
typedef struct sm_surrogate_net sm_surrogate_net;
int sm_surrogate_net_create(sm_context* ctx, int n_crystals, int nx, int ny, int nz, int layers, int width, int freqs,
                            int emb, uint64_t seed, sm_surrogate_net** out);
int sm_surrogate_net_layout(const sm_surrogate_net* net, int64_t* n_params, int64_t* offsets);
int sm_surrogate_net_get(sm_surrogate_net* net, float* params);
int sm_surrogate_net_set(sm_surrogate_net* net, const float* params);
/* loss = sum_{d, j} wgt[d][col[j]] (rho_hat(d, vox[j]) - rho[d][col[j]])^2 / (N B)
 * and its gradient (n_params floats) for a batch of B voxels; rho and wgt
 * are [N][ld] host arrays. */
int sm_surrogate_net_loss_grad(sm_surrogate_net* net, const int32_t* vox, const int32_t* col, int B, const float* rho,
                               const float* wgt, int64_t ld, double* loss, float* grad);
/* One Adam step (b1 0.9, b2 0.999, eps 1e-8) with the last gradient. */
int sm_surrogate_net_adam(sm_surrogate_net* net, float lr);
/* out[d][j] = rho_hat(d, vox[j]), [N][n] host. */
int sm_surrogate_net_predict(sm_surrogate_net* net, const int32_t* vox, int n, float* out);
/* The surrogate's correction step: inout[d][j] *= exp(gate[d] rho_hat(d, vox[j])),
 * [N][n] host values, gate [N] (0 leaves a row as it is). */
int sm_surrogate_net_apply(sm_surrogate_net* net, const int32_t* vox, int n, const float* gate, float* inout);
int sm_surrogate_net_destroy(sm_surrogate_net* net);

/* ---- beam masks and multiplexing of a sysmat (analysis on the device) ----------- */
/* The reference computes these on the CPU from a memory-mapped .sysmat file
 * (PEGen_RayTracing_CircularHole/extract_beam_prop_masks.py:52-87,
 * compute_mpxi_3d.py:45-52).  For one rotation's block of a PE sysmat in
 * device memory, sysmat[r * ld + v] (r < rows, v < voxels), and device
 * outputs:
 *   row_max[r], row_sum[r] (double), row_count[r] = size of the beam mask,
 *   the mask of row r being sysmat[r][v] > frac * row_max[r] (the product in
 *   single precision; threshold 1.0 when row_max[r] <= 0; the reference uses
 *   frac = 0.05);
 *   mask[r * ld_mask + v] (int8 0/1; may be NULL);
 *   mpxi[v] = number of rows whose mask holds voxel v (uint32; may be NULL).
 * Asynchronous on `stream`, on the current device.  NaN entries count as
 * below every threshold and do not raise the maximum. */
int sm_beam_metrics(const float* sysmat, int64_t rows, int64_t voxels, int64_t ld, float frac, float* row_max,
                    double* row_sum, int32_t* row_count, int8_t* mask, int64_t ld_mask, uint32_t* mpxi, void* stream);

/* Diagnostic: evaluate the tracer's ray primitives on the current device for
 * n argument rows (host arrays).  kind 0: chord through a box (12 floats:
 * segment in, out, box min, max), 1: chord from box entry to segment end
 * (12 floats), 2: chord through a hole cylinder (11 floats: in, out, x, y1,
 * y2, z, R).  Same device code as the sysmat kernel; replaces no reference
 * interface (the reference's primitives are PESysMatGen.cu:19-373). */
int sm_primitive_batch(int kind, const float* args, int64_t n, float* out);

#ifdef __cplusplus
}
#endif

#endif /* SYSMAT_B200_H */
