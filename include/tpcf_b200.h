/*
 * tpcf_b200.h -- C ABI of libtpcf_b200.so, a B200 (sm_100a) implementation of
 * the pair-summing path of tilmantroester/2pcf.
 *
 * Every entry point is plain C: scalars by value, arrays as pointers plus
 * sizes, no C++ or torch types.  Each entry point names the reference routine
 * it replaces (file:line inside the reference project).  A Fortran caller
 * binds them through an iso_c_binding interface module; Python binds them
 * through ctypes.
 *
 * Conventions
 *   - Arrays are 0-based structure-of-arrays, the memory layout of the
 *     reference's contiguous 1-based `real` arrays passed with c_loc.
 *   - 2-D outputs [n_A][n_bin] are row-major, which is the memory layout of the
 *     reference's column-major (n_bin, n_A) marks arrays.
 *   - Any input or output pointer may be host memory (pageable or pinned) or
 *     device memory of the context's GPU; the library detects which and copies
 *     only host arrays.
 *   - Nullable pointers are marked.  Outputs are written only on TPCF_OK.
 *   - The library never calls exit() or abort(): each call returns a
 *     tpcf_status and tpcf_last_error(ctx) describes the last failure.  This
 *     replaces the reference's `stop` / `error stop`.
 *   - A context binds one device and one stream; use one context per host
 *     thread.  There is no CPU fallback: without a usable GPU, tpcf_create
 *     fails with TPCF_ERR_NO_DEVICE.
 */
#ifndef TPCF_B200_H
#define TPCF_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TPCF_ABI_VERSION 1

typedef enum tpcf_status {
  TPCF_OK = 0,
  TPCF_ERR_INVALID_ARG = 1,
  TPCF_ERR_OOM = 2,
  TPCF_ERR_OVERFLOW = 3,      /* a size limit of the library was exceeded      */
  TPCF_ERR_TIMEOUT = 4,       /* a bounded device-side wait ran out            */
  TPCF_ERR_CUDA = 5,          /* a CUDA runtime call failed                    */
  TPCF_ERR_NOT_SUPPORTED = 6, /* e.g. the adjoint with spherical coordinates   */
  TPCF_ERR_NO_DEVICE = 7
} tpcf_status;

/* Bin spacings, same codes as lin_binning .. sqrt_binning (src/utils.f90:7). */
enum { TPCF_LIN = 0, TPCF_LOG = 1, TPCF_IHS = 2, TPCF_SQRT = 3 };

/* Replaces type(binning) (src/utils.f90:18-24) as built by
 * create_bins(x_min, x_max, n_bin, p, spacing) (src/utils.f90:139-230).
 * Edges are derived inside the library by the canonical FP64 rule (see
 * tpcf_canonical_edges).  1 <= n_bin <= 128.                                   */
typedef struct tpcf_bins {
  int32_t n_bin;
  int32_t spacing;
  double x_min;
  double x_max;
  double ihs_theta; /* `p` of the ihs spacing; ignored otherwise              */
} tpcf_bins;

typedef struct tpcf_opts {
  int32_t use_grid;      /* 1: cell-grid pruning at theta_max (replaces the
                            kd-tree, use_kd_tree); 0: every lens against every
                            source (the reference's --no-kd-tree)            */
  int32_t verbose;       /* print phase timings to stderr                    */
  double cell_size;      /* grid cell side in input units; 0 = autotuned     */
  int32_t spherical;     /* 1: x, y are longitude, latitude in radians and the
                            bins are angles in radians (spherical_coords,
                            src/tpcf.f90:297-359); |latitude| <= pi/2 */
  int32_t shard_index;   /* with shard_count > 1, this call computes only the
                            work items i with i % shard_count == shard_index
                            (items ordered by estimated cost): per-bin,
                            per-patch and per-lens sums are then partial and
                            must be summed over shards (one all-reduce);
                            normalised outputs are not written            */
  int32_t shard_count;   /* 0 or 1: no sharding                              */
  int32_t group_size;    /* planar pair kernel tile shape: threads per block
                            (32, 64 or 128; 0 = 128, halved while the
                            per-lens histogram would exceed 100 KB); each
                            warp takes 32-lens work items of its own         */
  int32_t tile_chunks;   /* 32-source sub-chunks per source tile (1 or 2;
                            0 = 2), in a 4 KB ring per warp                 */
  int32_t reserved[3];
} tpcf_opts;

/* Per-call results.  Replaces type(shear_2pcf_results) (src/tpcf.f90:17-22)
 * plus the raw FP64 sums behind it.  Arrays are caller-allocated. */
typedef struct tpcf_result {
  /* FP64 per-bin sums, always written, [n_bin] each:
   *   sum_dw = sum d*w_A*w_B        sum_gt = sum g_t terms (val_A-weighted)
   *   sum_gx = sum g_x terms        sum_w  = sum w_A*w_B
   *   sum_K  = sum w_A*w_B*(1+m_B)  (equals sum_w for scalar-scalar)         */
  double* sum_dw;
  double* sum_gt;
  double* sum_gx;
  double* sum_w;
  double* sum_K;
  int64_t* n_pairs;
  /* Reference-normalised outputs (src/tpcf.f90:369-376), nullable, [n_bin]:
   * theta = bin centres as create_bins computes them, mean_theta =
   * sum_dw/sum_w (NaN when sum_w == 0, as in the reference), g_t, g_x =
   * sum/K where K > 0 else 0, weights = sum_w.                              */
  float* theta;
  float* mean_theta;
  float* g_t;
  float* g_x;
  float* weights;
  /* Per-lens marks (src/tpcf.f90:354-358), nullable, [n_A][n_bin], lens order
   * of the input; marks_weight is [n_A].                                    */
  float* xi_E_marks;
  float* xi_B_marks;
  float* K_marks;
  float* w_marks;
  float* marks_weight;
  /* Per-lens FP64 sums, nullable, [n_A][6][n_bin] with the six rows
   * (sum_dw, sum_gt, sum_gx, sum_w, sum_K, n_pairs) of that lens.           */
  double* lens_sums;
  /* Per-patch FP64 sums, nullable, [n_patch][6][n_bin], same six rows, for
   * lens patches given in the call (block sums of
   * survey_marked_point_block_bootstrap, src/tpcf.f90:1130-1137).           */
  double* patch_sums;
  /* Per-lens FP64 sums without the lens factors, nullable, [n_A][6][n_bin]:
   * the same six rows with val_A*w_A (g rows) or w_A (d*w, w, K rows) left
   * out.  Input of tpcf_shear_scalar_adjoint.                               */
  double* lens_raw;
} tpcf_result;

/* Lens / scalar catalogue (lens_catalog, src/tpcf.f90:34-37).  z may be NULL
 * (all 0).  patch may be NULL (one patch); otherwise values in [0, n_patch).  */
typedef struct tpcf_lens_catalog {
  int64_t n;
  const float* x;
  const float* y;
  const float* z;
  const float* val;
  const float* w;
  const int32_t* patch;
} tpcf_lens_catalog;

/* Shear catalogue (shape_catalog, src/tpcf.f90:24-27).  z may be NULL (all 0),
 * m may be NULL (all 0). */
typedef struct tpcf_shear_catalog {
  int64_t n;
  const float* x;
  const float* y;
  const float* z;
  const float* e1;
  const float* e2;
  const float* w;
  const float* m;
} tpcf_shear_catalog;

typedef struct tpcf_ctx tpcf_ctx;

/* ---------------------------------------------------------------- context -- */
int32_t tpcf_abi_version(void);
tpcf_status tpcf_create(tpcf_ctx** ctx, int32_t device, const tpcf_opts* opts /* nullable */);
tpcf_status tpcf_destroy(tpcf_ctx* ctx);
const char* tpcf_last_error(const tpcf_ctx* ctx);
/* Use a caller stream (a cudaStream_t passed as void*) instead of the
 * context's own; NULL restores the context stream. */
tpcf_status tpcf_set_stream(tpcf_ctx* ctx, void* cuda_stream);
/* Number of kernels this context launched so far. */
int64_t tpcf_kernel_launches(const tpcf_ctx* ctx);

/* Statistics of the last pair-sum call.  pair_kernel_ms is measured with CUDA
 * events recorded on the context stream around the pair kernel when timing
 * is enabled (tpcf_set_timing), else 0; after tpcf_xi_from_marks and
 * tpcf_marks_bootstrap it is the summed time of their partial-sum kernels. */
typedef struct tpcf_stats {
  double pair_kernel_ms;
  double call_ms;
  int64_t n_pairs;          /* sum of n_pairs over all bins and tasks       */
  int64_t h2d_bytes;        /* bytes copied host->device by the last call   */
  int64_t kernel_launches;  /* kernels launched by this context so far      */
  int64_t workspace_bytes;  /* device workspace this context holds (grown by
                               cudaMalloc on demand, freed by tpcf_destroy)  */
} tpcf_stats;
tpcf_status tpcf_set_timing(tpcf_ctx* ctx, int32_t enable);
tpcf_status tpcf_last_stats(const tpcf_ctx* ctx, tpcf_stats* stats);
/* Change the grid cell side of later calls (tpcf_opts.cell_size; 0 = theta_max/16).
 * 2pcf_b200.autotune picks it by timing trial calls. */
tpcf_status tpcf_set_cell_size(tpcf_ctx* ctx, double cell_size);
/* Change the sharding of later calls (see tpcf_opts.shard_index). */
tpcf_status tpcf_set_shard(tpcf_ctx* ctx, int32_t shard_index, int32_t shard_count);
/* Tile shape of the planar pair kernel (tpcf_opts.group_size, tile_chunks;
 * 0 = default).  Results do not depend on it, only speed (the autotuner in
 * 2pcf_b200/autotune.py times the candidates).  No reference counterpart. */
tpcf_status tpcf_set_tile_shape(tpcf_ctx* ctx, int32_t group_size, int32_t tile_chunks);

/* Fault injection for tests of the failure paths; no reference counterpart
 * (the reference stops the program: src/kdtree.f90:119-122, :265-267).
 * fail_alloc >= 0: the fail_alloc-th device workspace allocation from now
 * (0 = the next) fails as if cudaMalloc had, and the call returns
 * TPCF_ERR_OOM.  skip_tile >= 0: the planar pair kernel never issues the copy
 * of the source tile with that ring index in each block (the marks kernel,
 * n_bin <= 32: the bulk copies of each block's tile with that index), so its
 * bounded waits run out after wait_polls polls (0 = the product's 2^22) and
 * the call returns TPCF_ERR_TIMEOUT; every copy that was issued has landed
 * before the kernel exits.  -1 / 0 switch them off.  The context stays
 * usable. */
tpcf_status tpcf_debug_inject(tpcf_ctx* ctx, int64_t fail_alloc, int32_t skip_tile, uint32_t wait_polls);

/* Roofline helper with no counterpart in the reference: measures this GPU's
 * FP32 FMA throughput (FLOP/s counting an FMA as 2) with a register-resident
 * FFMA loop timed by CUDA events on the context stream. */
tpcf_status tpcf_measure_fp32_peak(tpcf_ctx* ctx, double* tflops);
/* The same for FP64 FMA (a register-resident DFMA loop); no counterpart in the
 * reference.  The roofline of the FP64-bound resampling passes. */
tpcf_status tpcf_measure_fp64_peak(tpcf_ctx* ctx, double* tflops);

/* Canonical FP64 edges [n_bin+1] and squared edges [n_bin+1]: the bin rule of
 * every pair kernel.  A pair with d2 = dx*dx + dy*dy (FP64, from the FP32
 * inputs, no contraction) is in bin i when edges_sq[i] <= d2 < edges_sq[i+1],
 * in bin n_bin-1 when d2 == edges_sq[n_bin], and in no bin otherwise.  Host
 * only; mirrors the edge formulas of create_bins (src/utils.f90:202-228). */
tpcf_status tpcf_canonical_edges(const tpcf_bins* bins, double* edges, double* edges_sq);

/* Bin centres as the reference computes them in FP32 (src/utils.f90:202-229). */
tpcf_status tpcf_bin_centers(const tpcf_bins* bins, float* centers);

/* Spherical coordinates for later calls of this context (sets
 * tpcf_opts.spherical).  No reference counterpart: the reference passes
 * spherical_coords to each call (src/tpcf.f90:190). */
tpcf_status tpcf_set_spherical(tpcf_ctx* ctx, int32_t on);

/* Squared canonical chords (2 sin(e_i/2))^2 [n_bin+1] of the canonical edges
 * e_i (radians): the bin rule on the sphere.  A pair is binned by its
 * squared chord |u_B - u_A|^2 exactly as tpcf_canonical_edges bins d2, with
 * u = hi + lo of tpcf_unit_vectors in FP64 and the chord squared as
 * (dx*dx + dy*dy) + dz*dz.  The sine is the library's own fixed FP64
 * sequence (no libm), so the edges are the same on every host.  Host only;
 * no reference counterpart (the reference bins acos of the dot product in
 * FP32, src/utils.f90:512-528). */
tpcf_status tpcf_chord_edges(const tpcf_bins* bins, double* chord_sq);

/* Replaces rotate_data_from_poles_and_meridian (src/main.f90:953-1015) with
 * rotation_sphere (src/utils.f90:483-509): in place on (xA, yA) and, when
 * given, (xB, yB) (radians; host or device pointers).  When the lens field
 * plus r_max reaches a pole or the prime meridian, longitudes above pi are
 * wrapped, and both catalogues are rotated by (pi - median(xA), -median(yA));
 * *rotated says whether it happened and center (nullable) receives the
 * medians.  Decisions in FP32 as the reference takes them; the rotation is
 * evaluated in FP64 and rounded to FP32. */
tpcf_status tpcf_rotate_from_poles(tpcf_ctx* ctx, float* xA, float* yA, int64_t nA, float* xB, float* yB,
                                   int64_t nB, float r_max, int32_t* rotated, float* center);

/* ---------------------------------------------------- files and marks -- */
/* Replaces the text loaders load_standard_shape_catalog (7 columns x y z e1
 * e2 w m), load_standard_kappa_map (5: x y kappa_E kappa_B w) and
 * load_standard_lens_catalog (5: x y z val w) of src/input_formats.f90:227-333:
 * a table of ncols numbers per line separated by blanks or commas.  Lines
 * whose first non-blank character is '#' and blank lines are skipped (the
 * reference stops on them).  With cols == NULL, *n_rows receives an upper
 * bound on the rows (the data lines).  Otherwise cols is column-major
 * [ncols][capacity]; rows with column keep_pos_col <= 0 (the weight) and, if
 * keep_nonneg_col >= 0, with that column < 0 (the lens redshift) are dropped
 * as the loaders' masks do (:250-256, :316-328), and *n_rows receives the rows
 * kept, in file order.  More kept rows than capacity gives
 * TPCF_ERR_OVERFLOW.  All host threads parse (n_threads <= 0).  A malformed
 * line gives TPCF_ERR_INVALID_ARG.  Host only. */
tpcf_status tpcf_read_table(const char* path, int32_t ncols, int32_t keep_pos_col, int32_t keep_nonneg_col,
                            int32_t n_threads, float* cols, int64_t capacity, int64_t* n_rows);

/* The driver's result table (src/main.f90:699-702): one line per bin with
 * theta, g_t, g_x, weights, n_pairs, mean_theta, in that order; theta and
 * mean_theta converted from radians to degrees when to_degrees != 0 (the
 * spherical case, :690-694).  Reals as %16.7E, n_pairs as %21lld.  Host only. */
tpcf_status tpcf_write_result_table(const char* path, int32_t n_bin, const float* theta, const float* g_t,
                                    const float* g_x, const float* weights, const int64_t* n_pairs,
                                    const float* mean_theta, int32_t to_degrees);

/* Per-lens marks of one field, as save_marks / load_survey_marks hold them
 * (src/input_formats.f90:528-603): positions, marks weight and
 * [n][n_bin] marks (the Fortran (n_bin, n) arrays). */
typedef struct tpcf_marks_field {
  int64_t n;
  int64_t n_bin;
  float* x;
  float* y;
  float* w;     /* marks_weight */
  float* xi_E;  /* [n][n_bin] */
  float* xi_B;
  float* K;
} tpcf_marks_field;

/* Binary marks stream of save_marks (src/input_formats.f90:528-560): 1024-byte
 * header (int64 1024, int64 n_field, ..., int64 1024 at byte 1016), then per
 * field int64 n, n_bin, float32 x, y, w, xi_E, xi_B, K.  n_field <= 20. */
tpcf_status tpcf_marks_save(const char* path, int32_t n_field, const tpcf_marks_field* fields);
/* Sizes of a marks file: *n_field, and n[i], n_bin[i] for i < max_fields
 * (load_survey_marks' checks: n_field <= 20, n <= 5e7). */
tpcf_status tpcf_marks_info(const char* path, int32_t max_fields, int32_t* n_field, int64_t* n, int64_t* n_bin);
/* Reads a marks file into caller-allocated fields whose n and n_bin match
 * tpcf_marks_info. */
tpcf_status tpcf_marks_load(const char* path, int32_t n_field, const tpcf_marks_field* fields);

/* Replaces calculate_tpcf_from_marks (src/main.f90:1017-1139) for n_map
 * foreground maps at once: val[i] and w[i] are [n_map][n_i] for field i.
 * Lenses with marks.w * w <= 0 are left out.  Outputs (nullable):
 * g_t, g_x [n_map][n_field][n_bin] = sum xi_E val w / sum K w (plain
 * quotients, as the reference); weights [n_map][n_field] = sum marks.w w;
 * the stacked g_t_stacked, g_x_stacked [n_map][n_bin] and weights_stacked
 * [n_map] sum numerators and K over fields.  lens_x, lens_y (nullable) are
 * checked against the marks positions to 1e-5 as the reference does.  FP64
 * accumulation in a fixed order (deterministic; n_bin <= 32 on the FP64
 * tensor instruction).  Inputs may be host or device pointers.  Returns
 * TPCF_ERR_TIMEOUT when a bounded device wait for a bulk copy ran out (the
 * outputs are then not written). */
tpcf_status tpcf_xi_from_marks(tpcf_ctx* ctx, int32_t n_field, const tpcf_marks_field* marks, int32_t n_map,
                               const float* const* val, const float* const* w, const float* const* lens_x,
                               const float* const* lens_y, double* g_t, double* g_x, double* weights,
                               double* g_t_stacked, double* g_x_stacked, double* weights_stacked);

/* Resampling of per-lens marks: simple_bootstrap_foreground with marks
 * (src/tpcf.f90:547-634), survey_marked_point_bootstrap (:1194-1265) and the
 * resampling step of pair_weighted_block_bootstrap (:844-939).  The units are
 * the lenses of all fields in order (unit == NULL, n_units ignored) or the
 * labels unit[j] in [0, n_units) of the lenses (blocks, e.g. from
 * tpcf_kmeans).  Each resample draws int(n_units * supersampling) units with
 * replacement -- Philox4x32-10 with the counter layout of tpcf_bootstrap --
 * unless multiplicity [n_boot][n_units] is given.  Outputs (nullable):
 * g_t, g_x [n_boot][n_bin] = sum_j mult_j xi_E_j / sum_j mult_j K_j over all
 * fields (k_guard != 0: 0 where that K <= 0, as the point bootstraps; 0:
 * plain quotients, as the block one), weights [n_boot] = sum_j mult_j w_j,
 * and the [n_bin][n_bin] covariances of g_t and g_x over the resamples.
 * Marks may be host or device pointers.  TPCF_ERR_TIMEOUT as for
 * tpcf_xi_from_marks. */
tpcf_status tpcf_marks_bootstrap(tpcf_ctx* ctx, int32_t n_field, const tpcf_marks_field* marks,
                                 const int32_t* unit, int64_t n_units, const int32_t* multiplicity,
                                 uint64_t seed, int32_t n_boot, double supersampling, int32_t k_guard,
                                 double* g_t, double* g_x, double* weights, double* cov_gt, double* cov_gx);

/* Unit vectors of n points (lambda, phi in radians) as the spherical kernels
 * use them: u in FP64 by the library's fixed sine/cosine sequence, then
 * hi = fl32(u), lo = fl32(u - hi); hi and lo are [n][3].  Inputs and
 * outputs may be host or device pointers.  Diagnostics; no reference
 * counterpart. */
tpcf_status tpcf_unit_vectors(tpcf_ctx* ctx, const float* lam, const float* phi, int64_t n, float* hi,
                              float* lo);

/* ------------------------------------------------------------- pair sums -- */
/* Replaces tangential_shear_tpcf (src/tpcf.f90:190-378), called from
 * shear_2pcf (src/tpcf.f90:134-160).  Lenses with wA == 0 or zA < 0 and
 * sources with zB < 0 take part in no pair; a pair is skipped when zA > zB
 * (src/tpcf.f90:285, :306, :322).  zA, zB, mB and patchA may be NULL. */
tpcf_status tpcf_shear_scalar(tpcf_ctx* ctx,
                              const float* xA, const float* yA, const float* zA,
                              const float* valA, const float* wA, int64_t nA,
                              const float* xB, const float* yB, const float* zB,
                              const float* e1B, const float* e2B, const float* wB,
                              const float* mB, int64_t nB,
                              const tpcf_bins* bins,
                              const int32_t* patchA, int32_t n_patch,
                              tpcf_result* out);

/* Replaces scalar_kappa_tpcf (src/tpcf.f90:380-545), called from kappa_2pcf
 * (src/tpcf.f90:162-188): sum_gt accumulates kE*wB*valA*wA and sum_gx
 * kB*wB*valA*wA; K = weights. */
tpcf_status tpcf_scalar_scalar(tpcf_ctx* ctx,
                               const float* xA, const float* yA,
                               const float* valA, const float* wA, int64_t nA,
                               const float* xB, const float* yB,
                               const float* kE, const float* kB, const float* wB, int64_t nB,
                               const tpcf_bins* bins,
                               const int32_t* patchA, int32_t n_patch,
                               tpcf_result* out);

/* Batched tomography: n_task (lens catalogue, source catalogue) pairs, all in
 * one persistent launch.  Each task t correlates lenses[task_lens[t]] with
 * sources[task_src[t]] exactly as tpcf_shear_scalar would, writing outs[t].
 * Replaces the per-field loop around shear_2pcf (src/main.f90:585-617). */
tpcf_status tpcf_batch_shear_scalar(tpcf_ctx* ctx,
                                    int32_t n_lens_cat, const tpcf_lens_catalog* lenses,
                                    int32_t n_src_cat, const tpcf_shear_catalog* sources,
                                    int32_t n_task, const int32_t* task_lens,
                                    const int32_t* task_src,
                                    const tpcf_bins* bins, int32_t n_patch,
                                    tpcf_result* outs);

/* Scalar (kappa) catalogue of the scalar-scalar estimator (kappa_map,
 * src/tpcf.f90:29-32): kappa_E and kappa_B per object. */
typedef struct tpcf_kappa_catalog {
  int64_t n;
  const float* x;
  const float* y;
  const float* kE;
  const float* kB;
  const float* w;
} tpcf_kappa_catalog;

/* Batched scalar-scalar: n_task (scalar catalogue, kappa catalogue) pairs in
 * one persistent launch, each as tpcf_scalar_scalar would compute it (the lens
 * catalogues' z is not used).  Replaces the per-field loop around kappa_2pcf
 * (src/main.f90:638-660). */
tpcf_status tpcf_batch_scalar_scalar(tpcf_ctx* ctx,
                                     int32_t n_lens_cat, const tpcf_lens_catalog* lenses,
                                     int32_t n_kappa_cat, const tpcf_kappa_catalog* kappas,
                                     int32_t n_task, const int32_t* task_lens,
                                     const int32_t* task_kappa,
                                     const tpcf_bins* bins, int32_t n_patch,
                                     tpcf_result* outs);

/* ------------------------------------------------------------ plans ------ */
/* A prepared tpcf_batch_shear_scalar call (planar).  tpcf_plan_shear_scalar
 * takes the same arguments and builds, once, everything that depends only on
 * the catalogues' positions, weights and values as they are now: the source
 * grids and sub-chunk records, the lens groups, the sorted work items.
 * Device input arrays are used in place and must stay alive and unchanged
 * while the plan exists.  `outs` only tells which per-lens outputs each task
 * has (non-null fields; the pointers are not kept).
 *
 * tpcf_plan_launch enqueues the persistent pair kernel and the per-patch
 * reductions on the plan's stream (the context's stream when the plan was
 * made, or tpcf_plan_set_stream): no host synchronisation, no allocation and
 * no other API call, so the sequence may be recorded into a CUDA graph
 * (stream capture) and replayed.  tpcf_plan_results waits for the last launch
 * and writes the outputs of every task, as tpcf_batch_shear_scalar would
 * (same sums bit for bit); its outs must have the per-lens outputs the plan
 * was made with.  The plan keeps its own device workspace; the context it was
 * made from stays free for other calls.  Spherical contexts return
 * TPCF_ERR_NOT_SUPPORTED. */
typedef struct tpcf_plan tpcf_plan;
tpcf_status tpcf_plan_shear_scalar(tpcf_ctx* ctx,
                                   int32_t n_lens_cat, const tpcf_lens_catalog* lenses,
                                   int32_t n_src_cat, const tpcf_shear_catalog* sources,
                                   int32_t n_task, const int32_t* task_lens,
                                   const int32_t* task_src,
                                   const tpcf_bins* bins, int32_t n_patch,
                                   const tpcf_result* outs, tpcf_plan** plan);
tpcf_status tpcf_plan_launch(tpcf_plan* plan);
tpcf_status tpcf_plan_results(tpcf_plan* plan, tpcf_result* outs);
tpcf_status tpcf_plan_set_stream(tpcf_plan* plan, void* cuda_stream);
const char* tpcf_plan_last_error(const tpcf_plan* plan);
tpcf_status tpcf_plan_destroy(tpcf_plan* plan);

/* ------------------------------------------------------------ gradients -- */
/* No counterpart in the reference (it has no gradients).  Adjoint of
 * tpcf_shear_scalar: given dL/dg_t and dL/dg_x per bin (g = the normalised
 * xi of the forward call, nullable dL_dgx = 0), writes dL/dval_A, dL/dw_A
 * [nA] and dL/de1_B, dL/de2_B, dL/dw_B, dL/dm_B [nB] (each nullable).  The
 * inputs are those of the forward call plus its sum_gt, sum_gx, sum_K [n_bin]
 * and lens_raw [nA][6][n_bin] outputs (lens_raw is only read for the lens
 * gradients).  Pairs are binned exactly as in the forward call; the lens
 * gradients come from lens_raw, the source gradients from one pass over all
 * pairs with sources as owners.  Lenses and sources that take part in no pair
 * get 0. */
tpcf_status tpcf_shear_scalar_adjoint(tpcf_ctx* ctx,
                                      const float* xA, const float* yA, const float* zA,
                                      const float* valA, const float* wA, int64_t nA,
                                      const float* xB, const float* yB, const float* zB,
                                      const float* e1B, const float* e2B, const float* wB,
                                      const float* mB, int64_t nB,
                                      const tpcf_bins* bins,
                                      const double* sum_gt, const double* sum_gx, const double* sum_K,
                                      const double* lens_raw,
                                      const double* dL_dgt, const double* dL_dgx,
                                      float* grad_valA, float* grad_wA,
                                      float* grad_e1B, float* grad_e2B, float* grad_wB, float* grad_mB);

/* Gradient outputs of one catalogue of a batched backward pass (each array
 * nullable, [n] of its catalogue). */
typedef struct tpcf_lens_grad {
  float* val;
  float* w;
} tpcf_lens_grad;
typedef struct tpcf_shear_grad {
  float* e1;
  float* e2;
  float* w;
  float* m;
} tpcf_shear_grad;
/* The forward outputs and loss derivatives of one task of a batched backward
 * pass: sum_gt, sum_gx (nullable), sum_K [n_bin] and lens_raw [nA][6][n_bin]
 * of that task's forward (tpcf_batch_shear_scalar with lens_raw), dL/dg_t
 * and dL/dg_x (nullable) [n_bin]. */
typedef struct tpcf_adjoint_task {
  const double* sum_gt;
  const double* sum_gx;
  const double* sum_K;
  const double* lens_raw;
  const double* dL_dgt;
  const double* dL_dgx;
} tpcf_adjoint_task;

/* No counterpart in the reference.  Adjoint of tpcf_batch_shear_scalar: the
 * gradients of every task at once, with one persistent launch over all
 * (task, source group) work items, one lens grid per lens catalogue and one
 * sorted copy of each source catalogue.  A catalogue used by several tasks
 * receives the sum of their gradients (FP64, added in task order).  Each
 * task's gradient is the one tpcf_shear_scalar_adjoint gives for it. */
tpcf_status tpcf_batch_shear_scalar_adjoint(tpcf_ctx* ctx,
                                            int32_t n_lens_cat, const tpcf_lens_catalog* lenses,
                                            tpcf_lens_grad* lens_grads /* [n_lens_cat], nullable */,
                                            int32_t n_src_cat, const tpcf_shear_catalog* sources,
                                            tpcf_shear_grad* src_grads /* [n_src_cat], nullable */,
                                            int32_t n_task, const int32_t* task_lens, const int32_t* task_src,
                                            const tpcf_bins* bins, const tpcf_adjoint_task* task_in);

/* -------------------------------------------------- patches and errors -- */
/* Replaces partition_data (src/kmeans.f90:12-263) as called for Voronoi
 * blocks (equal_size = .false., weight_equalizer_scaling = 0,
 * src/tpcf.f90:1117-1124): fixed-grid initial centroids
 * (src/kmeans.f90:85-112), Lloyd iterations on the device until no label
 * changes, the changed fraction drops below reassign_tol, or max_iter + 1
 * passes.  Distances are FP32 sqrt(dx*dx+dy*dy) with IEEE rounding; centroid
 * sums are 64-bit fixed point, so the labels are the same on every run.
 * labels_out [n] are 0-based; centroids_out [k][2] is nullable.  The
 * stopping rule is evaluated on the device, so the host waits once per batch
 * of passes, not once per pass.  The reference's equal-weight mode (distance
 * penalty and rebalancing pass) is tpcf_kmeans_equal below. */
tpcf_status tpcf_kmeans(tpcf_ctx* ctx, const float* x, const float* y, const float* w, int64_t n,
                        int32_t k, int32_t max_iter, float reassign_tol,
                        int32_t* labels_out, float* centroids_out, int32_t* n_iter_out);

/* Replaces partition_data with equal_size = .true. (src/kmeans.f90:12-262),
 * as pair_weighted_block_bootstrap calls it (src/tpcf.f90:892-895): from
 * pass 2 on, the distance to cluster j is scaled by
 * 1 + (W_j / W_mean - 1) * weight_scaling, W_j the cluster weights after the
 * previous pass (the reference updates them during the pass, in thread
 * order); each point keeps its second-nearest cluster and the distance ratio;
 * after the Lloyd passes, if (max W - min W) / W_mean > weight_tol, clusters
 * are visited heaviest first and their members, smallest ratio first, move to
 * their second cluster (if not yet visited) until the cluster is at most
 * W_mean (1 + weight_tol) -- the greedy rebalance of :221-262.  Weights are
 * summed in 64-bit fixed point (exact, deterministic).  random_init != 0:
 * k distinct random points as centroids and random labels (Philox4x32-10
 * from seed) as kmeans_compute_random_initial_centroids; 0: the fixed grid of
 * tpcf_kmeans.  centroids_out are those of the last pass (before the
 * rebalance, as the reference); *max_dev_out (nullable) the final
 * (max W - min W) / W_mean. */
tpcf_status tpcf_kmeans_equal(tpcf_ctx* ctx, const float* x, const float* y, const float* w, int64_t n,
                              int32_t k, int32_t max_iter, float reassign_tol, float weight_scaling,
                              float weight_tol, int32_t random_init, uint64_t seed, int32_t* labels_out,
                              float* centroids_out, int32_t* n_iter_out, float* max_dev_out);

/* Replaces the resampling loop of survey_marked_point_block_bootstrap
 * (src/tpcf.f90:1166-1191) and covariance_matrix (src/utils.f90:745-764) for
 * n_task tasks at once.  patch_sums is [n_task][n_patch][6][n_bin] as the pair
 * calls write it (tpcf_result.patch_sums).  multiplicity [n_boot][n_patch]
 * may be NULL: then each resample draws int(n_patch*supersampling) patches
 * with replacement from Philox4x32-10 keyed by `seed` (a pure function of
 * seed, resample and draw; mult_out, nullable, receives the counts).
 * Outputs: g_t, g_x [n_boot][n_task][n_bin] (0 where K <= 0, as the
 * reference), weights [n_boot][n_task] (nullable), and the unbiased
 * covariances of g_t and g_x over the joint data vector, [D][D] with
 * D = n_task*n_bin (nullable). */
tpcf_status tpcf_bootstrap(tpcf_ctx* ctx, const double* patch_sums, int32_t n_task, int32_t n_patch,
                           int32_t n_bin, const int32_t* multiplicity, uint64_t seed, int32_t n_boot,
                           double supersampling, double* g_t, double* g_x, double* weights,
                           double* cov_gt, double* cov_gx, int32_t* mult_out);

/* No counterpart in the reference.  The pair sum of tpcf_shear_scalar for
 * callers that cannot allocate device memory: a framework's caching allocator
 * or a fixed pool owns the GPU's memory (an extra cudaMalloc would fail or
 * fragment it), or cudaMalloc/cudaFree, which may synchronise the whole device,
 * is unaffordable in the caller's loop.  Every scratch buffer comes from one
 * static 64 MiB device array that each GPU loading the library holds until the
 * process exits; nothing is allocated.  The first call on each device looks up
 * the array's address (cudaGetSymbolAddress) and must come before any stream
 * capture.  All calls share the array and it keeps the last call's contents
 * (what must start at zero is cleared by each call): calls that overlap on the
 * GPU, from two host threads or two streams, race.  Patches and per-lens
 * outputs are not available (those fields of `out` must be NULL).  A call that
 * needs more than the 64 MiB fails with TPCF_ERR_OVERFLOW before any pair
 * work: about 100 bytes per object of either catalogue, i.e. roughly 600
 * thousand objects in all (the cell table is kept within an eighth of the
 * array by coarsening the cells when theta_max is small against the field, so
 * the field's extent does not lower the limit).  The cached address is only
 * valid for the device context that looked it up: do not call
 * cudaDeviceReset between calls. */
tpcf_status tpcf_shear_scalar_noalloc(tpcf_ctx* ctx,
                                      const float* xA, const float* yA, const float* zA,
                                      const float* valA, const float* wA, int64_t nA,
                                      const float* xB, const float* yB, const float* zB,
                                      const float* e1B, const float* e2B, const float* wB,
                                      const float* mB, int64_t nB,
                                      const tpcf_bins* bins, tpcf_result* out);

#ifdef __cplusplus
}
#endif

#endif /* TPCF_B200_H */
