/*
 * gd_b200.h -- C ABI of the B200-native swarm collision path.
 *
 * The reference (GameDev) has no runtime plugin ABI: its collision step is compiled into the
 * `gamedev` executable from a model directory (`make MODEL=<m>`, Makefile:56-77, 131-151) and is
 * entered through the `evolve_collisions(duration)` lambda (src/swarm/swarm_runtime.cu:357-471),
 * which runs the geometry stage (col_site_init -> index build -> col_cache_get -> col_space_bin)
 * and then `evolve_local_collisions(...)` (inc/swarm/_col_chain.cuh:108-539).  Every entry point
 * below replaces one of those pieces; the comment on each names the reference code it stands in
 * for.  A model-local bridge (mod/gd_bridge/) forwards the reference's calls here.
 *
 * Conventions
 *   - Plain pointers and sizes only.  Pointers named dev_* are CUDA device pointers owned by the
 *     caller (particles, RNG states, output caches), exactly as in the reference, where
 *     swarm_runtime.cu:76-184 allocates them.  The library owns its index, workspace and scratch.
 *   - Every call is asynchronous on the handle's stream unless it reports a device-side status
 *     (non-finite input, chain error), in which case it synchronises that stream once.
 *   - No call throws or exits.  A non-zero gd_status is returned and gd_last_error() gives the
 *     message; gd_error_detail() gives the particle index or chain error code where one applies.
 *   - One handle is not re-entrant; distinct handles are independent.
 */
#ifndef GD_B200_H
#define GD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference stops the process instead (gpu.cuh:103-120 GPU_CHECK -> exit,
 * col_chain_run.cu:256-375 chain errors -> std::runtime_error in _col_chain.cuh:403-405). */
typedef enum gd_status {
    GD_OK = 0,
    GD_ERR_INVALID_ARGUMENT = 1,   /* bad size, null pointer, unsupported configuration      */
    GD_ERR_CUDA = 2,               /* a CUDA runtime call failed; detail = cudaError_t        */
    GD_ERR_NONFINITE = 3,          /* non-finite particle state; detail = particle index       */
    GD_ERR_CHAIN = 4,              /* event-chain error; detail = reference code 1..6          */
    GD_ERR_CAPACITY = 5,           /* a bounded structure (stack, queue, scratch) overflowed   */
    GD_ERR_CONTINUATION_LIMIT = 6, /* chain did not finish within its bounded event budget     */
    GD_ERR_TIME_RESOLUTION = 7,    /* scheduler needed more than 2^52 subdivisions             */
    GD_ERR_CONTROLLER = 8,         /* invalid rate or audit state seen by the bath controller   */
    GD_ERR_NOT_READY = 9,          /* geometry or model used before it was built               */
    GD_ERR_OUT_OF_MEMORY = 10,
    GD_ERR_TIMEOUT = 11,           /* a bounded device wait gave up (the kernel stopped cleanly) */
    GD_ERR_IO = 12                 /* a checkpoint file could not be opened, read or written,
                                      or its size is not the expected one                       */
} gd_status;

/* Search structure requested by the model (Makefile COLLISION_SEARCH=kdtree|morton).  Both
 * produce the same exact top-K list in canonical order (ascending float d^2, then code). */
enum { GD_SEARCH_KDTREE = 0, GD_SEARCH_MORTON = 1 };

/* Coagulation kernels (inc/swarm/_collision.cuh:22-28). */
enum { GD_KERNEL_CONSTANT = 0, GD_KERNEL_LINEAR = 1, GD_KERNEL_PRODUCT = 2, GD_KERNEL_CUSTOM = 3 };

/*
 * Model constants that the reference fixes at compile time in const_defs.cuh
 * (inc/swarm/const_defs.cuh:30-159) and flags.mk (-DCODE_UNIT, -DCONST_NU, -DHALF_DISK ...).
 * gd_config_default() fills the reference defaults; a bridge copies the model's constexprs.
 */
typedef struct gd_config {
    /* code units (const_defs.cuh:30-33) */
    double G, M_S, R_0, S_0;
    /* mesh domain (const_defs.cuh:41-51) */
    int    n_x, n_y, n_z;
    double x_min, x_max, y_min, y_max, z_min, z_max;
    /* gas (const_defs.cuh:68-88) */
    double sigma_0, aspr_0, idx_p, idx_q;
    int    const_nu;          /* 1: CONST_NU, 0: CONST_ALPHA                                  */
    double nu, alpha;
    int    code_unit;         /* 1: CODE_UNIT (Reynolds from REYNOLDS_0, no Brownian term)     */
    double reynolds_0, m_mol, x_sec;
    int    half_disk;         /* HALF_DISK: polar upper bound inclusive (_transport.cuh:39-48) */
    int    const_st;          /* CONST_ST: Stokes number without gas scaling (param_phys.cuh:202) */
    /* dust (const_defs.cuh:95-97) */
    double stokes_0, rho_0;
    /* collision (const_defs.cuh:118-140) */
    int    coag_kernel;       /* GD_KERNEL_*                                                   */
    int    n_k;               /* neighbour slots per owner, 1..256                              */
    double h_search;          /* search radius in local gas scale heights                      */
    double v_frag;            /* fragmentation threshold speed                                  */
    int    col_event_cap;
    int    col_bin_x, col_bin_y, col_bin_z, col_bin_s, col_bin_min;
    double col_bath_max, col_bath_eps, col_bath_alpha;
    /* multisize initialisation bounds, used by fragmentation (const_defs.cuh:165-168) */
    double init_smin, init_smax;
    /* search selection (Makefile COLLISION_SEARCH, const_defs.cuh:142-145) */
    int    search;            /* GD_SEARCH_*                                                    */
    int    morton_leaf_target, morton_max_level;
} gd_config;

/* One representative particle, byte-identical to the reference `struct swarm` built with
 * -DMULTISIZE (const_defs.cuh:194-203): position (azimuth, spherical radius, polar angle),
 * velocity (l_phi, v_r, l_theta), grain diameter, represented grain count.  64 bytes. */
typedef struct gd_particle {
    double position[3];
    double velocity[3];
    double par_size;
    double par_numr;
} gd_particle;

/* Size in bytes of one per-particle RNG state (cuRAND XORWOW curandState, 48 bytes), the record
 * the reference keeps in dev_rngstate and writes to rngstate_<n>.dat (swarm_host.cuh:867-899). */
size_t gd_rng_state_bytes(void);

typedef struct gd_handle gd_handle;

/* Fill *cfg with the reference's default const_defs.cuh values. */
void gd_config_default(gd_config *cfg);

/* Create a handle for n_p particles (const_defs.cuh:39 N_P) on the current CUDA device.
 * Allocates the index, neighbour cache, controller workspace (the reference's local_workspace,
 * _col_chain.cuh:36-96) and the caches the reference allocates in swarm_runtime.cu:120-184.
 * Limits (GD_ERR_INVALID_ARGUMENT, before any device work): 3 n_p <= INT_MAX (packed neighbour
 * codes, _col_image.cuh:14-15); in an azimuthal wedge, whose index holds three sites per particle,
 * 3 n_p <= 2^30. */
gd_status gd_create(const gd_config *cfg, int n_p, gd_handle **out);
void      gd_destroy(gd_handle *h);

/* Run all later work of this handle on `stream` (a cudaStream_t; NULL = legacy default stream,
 * the stream every reference launch uses, _col_chain.cuh:147-149). */
gd_status gd_set_stream(gd_handle *h, void *stream);

/* Message and numeric detail of the last failed call on this handle. */
size_t    gd_last_error(const gd_handle *h, char *buf, size_t len);
long long gd_error_detail(const gd_handle *h);

/* rngstate_init (src/swarm/rngstate_init.cu:11-18): curand_init(seed, subsequence = i, 0) for
 * i < n, written to dev_rng (n * gd_rng_state_bytes() bytes). */
gd_status gd_rng_init(void *dev_rng, int n, unsigned long long seed, void *stream);

/* Geometry stage: col_site_init (src/swarm/col_site_init.cu:17-119) + index build
 * (kdtree::buildTree, builder.h:109-152, or morton_index::build, morton_index.cuh:168-229).
 * Non-finite particle -> GD_ERR_NONFINITE with the smallest bad index as detail (the reference
 * reports the index its atomicCAS kept and exits, swarm_runtime.cu:382-393). */
gd_status gd_geometry_build(gd_handle *h, const gd_particle *dev_particle);

/* col_cache_get (inc/swarm/_col_cache.cuh:15-159): exact top-K neighbour codes (code = 3*index +
 * image, _col_image.cuh:11-35) of every active owner, owner-major [n_p][n_k], in ascending
 * (float d^2, code) order with -1 padding; inactive owners get a row of -1 and measure 0.
 * dev_codes / dev_measure / dev_kth_d2 may be NULL, in which case the handle's own cache is
 * written (and used by the collision operator).  dev_kth_d2 receives the largest kept d^2
 * (0 for an empty row).  Requires gd_geometry_build. */
gd_status gd_knn(gd_handle *h, const gd_particle *dev_particle,
                 int32_t *dev_codes, double *dev_measure, float *dev_kth_d2);

/* Radius-bounded exact top-K: the same output as gd_knn, computed by first walking each owner's
 * neighbourhood only out to min(q_i, dev_radius[i]) (a proposed radius, e.g. from the learned
 * radius model); an owner that finds fewer than K sites inside repeats the walk with q_i, so the
 * result is exact by construction.  dev_radius may be NULL (plain query).  dev_stats, when not
 * NULL, receives 4 accumulated counters: 8-site leaf groups scanned, tree nodes tested, candidate offers to a
 * top-K heap, owners that fell back to the full radius (add to existing values; zero it first). */
gd_status gd_knn_bounded(gd_handle *h, const gd_particle *dev_particle, const float *dev_radius,
                         int32_t *dev_codes, double *dev_measure, float *dev_kth_d2,
                         unsigned long long *dev_stats);

/* Speed-only settings of the neighbour search; every setting gives the same exact lists.  No
 * counterpart in the reference (whose KD/Morton parameters are compile-time constants).
 *   warps_per_block     warps per block of the top-K kernel (0: the most resident warps)
 *   prescan             Morton-neighbour buckets scanned on each side before the tree walk (0..8)
 *   walk_breadth_first  1: breadth-first walk with a pipelined leaf list; 0: depth-first walk
 *   sort_bits           top Morton key bits the index sort orders by: 0 (all, 21 per axis) or
 *                       16..21 per axis (fewer radix passes, coarser buckets)
 *   range_query         radius-bounded query (gd_knn_bounded) only: 1 (default) serves each owner
 *                       with a whole warp, collecting the sites inside min(q, r) and sorting them
 *                       with a warp-wide network, the owners it cannot serve going to the per-lane
 *                       heap query; 0: the per-lane heap query for every owner.  Used for K <= 64
 *                       outside wedges; elsewhere the heap query runs either way. */
typedef struct gd_tuning {
    int warps_per_block, prescan, walk_breadth_first, sort_bits, range_query;
} gd_tuning;
gd_status gd_get_tuning(const gd_handle *h, gd_tuning *out);
gd_status gd_set_tuning(gd_handle *h, const gd_tuning *t);

/* Autotuner: times the search on the caller's own particles (and proposed radii, or NULL for the
 * plain query) over the sort order (if tune_sort), the walk and prescan depth, then the block width
 * (greedy, best of three runs each; a setting replaces the current one only when at least 2%
 * faster), checks that every setting reproduces the starting setting's codes and kept d^2 bit for
 * bit (GD_ERR_CONTROLLER otherwise), keeps the fastest in the handle and leaves the geometry built
 * with it.  *out_best / *out_ms (may be NULL) receive the setting and its
 * query time.  Synchronises the stream; not for use under stream capture. */
gd_status gd_autotune(gd_handle *h, const gd_particle *dev_particle, const float *dev_radius, int tune_sort,
                      gd_tuning *out_best, double *out_ms);

/* Deferred non-finite screen (on != 0).  gd_geometry_build then enqueues the whole build without
 * waiting for its non-finite screen (the reference's stop on the first non-finite particle,
 * swarm_runtime.cu:382-393), so a build + query sequence makes no host synchronisation and can be
 * captured into a CUDA graph on the handle's stream.  Non-finite particles are treated as inactive
 * until gd_check_geometry reports them.  Off by default. */
gd_status gd_set_deferred_checks(gd_handle *h, int on);

/* The deferred screen of the most recent geometry build on the handle's stream (an eager
 * gd_geometry_build or its replay from a captured graph): GD_ERR_NONFINITE with the smallest bad
 * index in gd_error_detail (and the geometry invalidated), else GD_OK (and the geometry marked
 * valid: after a replay it stands for the positions the replay read).  Synchronises the stream. */
gd_status gd_check_geometry(gd_handle *h);

/* Keplerian azimuthal advance of every active particle by dt: phi += Omega_K(R) dt wrapped into
 * [x_min, x_max) (the orbital part of the reference's transport step, _transport.cuh, without drag,
 * radiation or diffusion).  Invalidates the geometry: positions changed. */
gd_status gd_drift_keplerian(gd_handle *h, gd_particle *dev_particle, double dt);

/*
 * Learned search-radius proposal.  No counterpart in the reference: it seeds gd_knn_bounded,
 * whose fallback keeps the neighbour lists identical to the plain query.
 *
 * Features (8 per owner, float32, by particle index): log2(1 + active sites in the owner's Morton
 * cell) at 3 levels, log(y/R_0), (polar angle - pi/2)/h_g, log(size/S_0), log of the owner's
 * bucket weight sum over the mean bucket weight, log(sqrt(previous K-th d^2)/R_0) (0 without one).
 * Target: log(sqrt(K-th d^2)/R_0).  Network: 8 -> 64 -> 64 -> 1 with GELU, BF16 weights, FP32
 * accumulation, standardised inputs; trained with Adam on MSE by this library's kernels.  The
 * proposed radius is R_0 exp(prediction + margin), the margin being the calibrated quantile of the
 * training residuals.
 */
typedef struct gd_radius_model gd_radius_model;
enum { GD_RADIUS_FEATURES = 8, GD_RADIUS_PARAMS = 4801 };

/* A fresh model (seeded initialisation) for a swarm whose length unit is R_0. */
gd_status gd_radius_model_create(unsigned long long seed, double R_0, gd_radius_model **out);
void      gd_radius_model_destroy(gd_radius_model *m);

/* Features of every owner of the handle's current geometry (call after gd_geometry_build).
 * dev_prev_kth_d2 (may be NULL) is the previous step's K-th d^2 by particle index; total_mass
 * is the swarm's represented mass.  dev_features is [n_p][8]. */
gd_status gd_radius_features(gd_handle *h, const gd_particle *dev_particle, const float *dev_prev_kth_d2,
                             double total_mass, float *dev_features);

/* `iterations` Adam steps (learning rate lr) on minibatches of `batch` owners drawn uniformly
 * from the n rows of (dev_features, dev_kth_d2); rows with kth_d2 <= 0 carry no weight.  The
 * first call also fixes the input standardisation from these rows.  *loss receives the mean
 * squared error of the last minibatch (host pointer, may be NULL).  Runs on `stream`. */
gd_status gd_radius_model_train(gd_radius_model *m, const float *dev_features, const float *dev_kth_d2, int n,
                                int iterations, int batch, float lr, float *loss, void *stream);

/* Mean-squared-error loss and its gradient with respect to the GD_RADIUS_PARAMS parameters over
 * all n rows (no update): dev_grad [GD_RADIUS_PARAMS], *loss on the host. */
gd_status gd_radius_model_gradient(gd_radius_model *m, const float *dev_features, const float *dev_kth_d2, int n,
                                   float *dev_grad, float *loss, void *stream);

/* Set the radius margin to the `quantile` (e.g. 0.999) of target - prediction over the rows
 * with kth_d2 > 0; *margin receives it (host pointer, may be NULL). */
gd_status gd_radius_model_calibrate(gd_radius_model *m, const float *dev_features, const float *dev_kth_d2, int n,
                                    double quantile, float *margin, void *stream);

/* Proposed radius R_0 exp(prediction + margin) per row into dev_radius [n] (float32).  The hidden
 * 64 x 64 layer runs on the tensor cores (tcgen05, BF16 operands, FP32 accumulation); asynchronous
 * on `stream`, so a failure of its bounded waits is reported by gd_radius_model_check. */
gd_status gd_radius_model_predict(gd_radius_model *m, const float *dev_features, int n, float *dev_radius,
                                  void *stream);

/* Synchronous check of the model's device error flag: GD_ERR_TIMEOUT when a tensor-core forward
 * stopped at a timed-out wait (its radii are then incomplete), else GD_OK. */
gd_status gd_radius_model_check(gd_radius_model *m);

/* Copy the FP32 master parameters (and standardisation: 8 means, 8 scales, margin) out of or into
 * the model; host buffers of GD_RADIUS_PARAMS and 17 floats. */
gd_status gd_radius_model_get(const gd_radius_model *m, float *params, float *norm17);
gd_status gd_radius_model_set(gd_radius_model *m, const float *params, const float *norm17);

/* Copy the site-init outputs of the last gd_geometry_build to caller device buffers (any may be
 * NULL): sites [gd_site_count(h)] x (x, y, z, code bits) as float4, search radius q [n_p] (0 when
 * inactive), active flags [n_p] (the reference's dev_kdtree_node cartesian / dev_search_dist /
 * dev_col_active, col_site_init.cu:44-76, 106-117).  Sites 0..n_p-1 are the particles; with an
 * azimuthal wedge, sites n_p + i and 2 n_p + i are particle i's periodic images rotated by -width
 * (code 3i + 1) and +width (code 3i + 2), as the reference's N_T = 3 N_P tree nodes are. */
gd_status gd_get_sites(gd_handle *h, float *dev_site4, float *dev_q, unsigned char *dev_active);

/* Sites of the handle's geometry: n_p, or 3 n_p for an azimuthal wedge (N_T, const_defs.cuh:240). */
int gd_site_count(const gd_handle *h);

/* The periodic-image parameters the search uses for cfg (no device work): *wedge = X_WEDGE
 * (n_x > 1 and float(x_max) - float(x_min) < 2 pi - 1e-6, const_defs.cuh:56-57); *width = the
 * rotation angle of the images (KD: float(x_max - x_min), col_site_init.cu:60; Morton:
 * float(x_max) - float(x_min), morton_ghost.cuh:62), 0 without a wedge; *image_dist_min =
 * _get_image_dist_min (param_grid.cuh:86-89), -1 without a wedge.  An owner keeps one image per
 * particle (the nearer) when image_dist_min <= 2 q, with q its own search distance for the KD
 * search (_col_cache.cuh:38-39) and the largest one for the Morton search (swarm_runtime.cu:413-415).
 * Any output may be NULL. */
gd_status gd_wedge_info(const gd_config *cfg, int *wedge, float *width, float *image_dist_min);

/* Copy the handle's neighbour cache (codes, measures) to caller device buffers. */
gd_status gd_get_cache(gd_handle *h, int32_t *dev_codes, double *dev_measure);

/* Replace the handle's neighbour cache with caller-provided codes and measures (device
 * pointers, [n_p][n_k] and [n_p]), e.g. a cache restored from a file, and mark geometry valid. */
gd_status gd_set_cache(gd_handle *h, const int32_t *dev_codes, const double *dev_measure);

/* col_space_bin (src/swarm/col_space_bin.cu:11-35): controller group of every particle. */
gd_status gd_space_bin(gd_handle *h, const gd_particle *dev_particle, int32_t *dev_spatial);

/* Geometry epoch control (swarm_runtime.cu:350-354): positions changed, rebuild on next use. */
gd_status gd_invalidate_geometry(gd_handle *h);

/* Reset the per-group bath controller memory (local.state), as the reference does at every
 * output boundary (swarm_runtime.cu:490-496).  Results of captured operators not read yet are
 * read first (gd_check_operator) and their status returned. */
gd_status gd_reset_controller(gd_handle *h);

/* COL_DIAGNOSTICS controller summary of the current output interval (since the handle was created
 * or gd_reset_controller last ran), as the JSON text save_col_controller writes
 * (inc/swarm/_col_bound.cuh:242-299, schema 2): per finished group bath its duration, limit scale
 * before and after and the audit result, and the running extrema.  Copies up to len - 1 bytes and a
 * terminating NUL into buf (buf may be NULL) and returns the full text length.  Chain launches per
 * wave are 1 (the persistent chain) where the reference counts its relaunches. */
size_t gd_controller_summary(const gd_handle *h, char *buf, size_t len);

/* COL_DIAGNOSTICS event bookkeeping (event_work / col_event_sum, inc/swarm/_col_event.cuh:9-13,
 * _col_chain.cuh:519-535).  With diagnostics on (off by default), each collision operator counts
 * its events and sums their log mass change per outcome category: 0..3 sticking with mass ratio
 * q <= 1e-6, 1e-4, 1e-2 or above; 4 catastrophic fragmentation; 5 remnant erosion; 6 debris.
 * gd_event_totals copies the last operator's 7 counts and 7 sums to host arrays (synchronous). */
gd_status gd_set_diagnostics(gd_handle *h, int on);
/* With diagnostics on, every collision operator also writes its line of the reference's
 * per-operator JSONL log (collision_local_*.jsonl, inc/swarm/_col_chain.cuh:488-535): operator
 * number, clock_sim (the device clock under gd_step, else 0), duration, waves, owner updates,
 * chain blocks and launches, the chain, audit and whole-operator seconds (device time), the finest
 * tick count, and per controller group its owners, final level and bath length, initial level,
 * coarsened / refined / neighbour-constrained updates, minimum, maximum, final and initial
 * requested bath lengths, initial binding constraint, updates, overshoots, persistent overshoots,
 * oldest linked reservoir, largest bath length over request, largest growth and predicted activity;
 * then the event counts and log-mass sums.  The lines accumulate over the handle's life (as the
 * reference's file does); gd_operator_log copies them (up to len - 1 bytes and a NUL) and returns
 * the full length.  The persistent chain is one launch per wave, so chain_launches = waves and
 * chain_blocks = the owners the waves queued; the reference counts each capped relaunch. */
size_t gd_operator_log(const gd_handle *h, char *buf, size_t len);
/* The device time of the operators logged so far, split as the reference's COL_PERF_VAL build
 * splits it (_col_chain.cuh:215-241): out4 = seconds of the waves' reservoir publish, bath rates
 * and bins; of the skip scans and chains; of the audits and bath finishes; of the whole operators
 * (the rest is the bath-start pass and the controller's scheduling). */
gd_status gd_operator_phase_seconds(const gd_handle *h, double *out4);
gd_status gd_event_totals(gd_handle *h, unsigned long long *counts, double *log_mass);

/* evolve_local_collisions (inc/swarm/_col_chain.cuh:108-539): advance every owner through one
 * fixed-position frozen-bath collision operator of length `duration`, mutating par_size and
 * par_numr of dev_particle and the RNG states in dev_rng.  Uses the neighbour cache built by
 * gd_knn (or set by gd_set_cache).  total_dust_mass enters lambda_0 = N_P/(N_K*M_dust)
 * (_col_chain.cuh:187).
 *
 * The operator is one CUDA graph: the bath-start pass, then a conditional WHILE node whose body
 * is one wave (chains, audit, bath finish, schedule advance, the next wave's rates and bath
 * lengths), with the controller's decisions made on the device; the host reads nothing between
 * waves.  On a stream that is not capturing, the call runs that graph and returns its status.  On
 * a stream the caller is capturing (cudaStreamBeginCapture on the handle's stream), the operator
 * joins the caller's graph and the call returns GD_OK; after the caller's graph ran,
 * gd_check_operator returns the status of the operators it held and brings their statistics and
 * bath records to the host. */
gd_status gd_collision_operator(gd_handle *h, gd_particle *dev_particle, void *dev_rng,
                                double duration, double total_dust_mass);

/* Results of the collision operators run since the last read (synchronises the handle's stream):
 * the first error any of them met, the summed statistics (gd_last_operator_stats) and their bath
 * records (gd_controller_summary).  An operator that meets an error stops after the wave that met
 * it, as the reference's host loop does, and later operators do nothing until this call. */
gd_status gd_check_operator(gd_handle *h);

/* evolve_collisions (swarm_runtime.cu:357-471): non-finite screen (colstate_flag) when the
 * geometry is valid, else geometry build + gd_knn + space bins; then the collision operator. */
gd_status gd_evolve_collisions(gd_handle *h, gd_particle *dev_particle, void *dev_rng,
                               double duration, double total_dust_mass);

/* Controller statistics of the last operator (of the operators of the last gd_check_operator
 * read, summed): waves, chain launches, owners updated, events, bath lengths. */
typedef struct gd_operator_stats {
    int    waves;
    int    chain_launches;
    long long owner_updates;
    long long events;
    double min_duration, max_duration;
} gd_operator_stats;
gd_status gd_last_operator_stats(const gd_handle *h, gd_operator_stats *out);

/* Draw `count` deviates per particle exactly as the collision chain does
 * (_get_col_uniform, _col_rates.cuh:145-149: min(curand_uniform_double, nextafter(1, 0))) from a
 * COPY of each RNG state; dev_rng is left unchanged.  dev_out is [n][count] f64. */
gd_status gd_rng_uniforms(const void *dev_rng, int n, int count, double *dev_out, void *stream);

/* Per-owner state of the last collision operator, copied to caller device buffers (any may be
 * NULL): bath-start rate moments [n_p][4] = (rate or -1 when invalid, first, second, maximum)
 * (cached_rate_moments, _col_types.cuh:366), owner clock, accepted events, and the reservoir
 * published at the start of the owner's last bath (size_old, numr_old). */
gd_status gd_get_owner_state(gd_handle *h, double *dev_cached4, double *dev_time, int32_t *dev_events,
                             double *dev_size_old, double *dev_numr_old);

/* The per-pair terms col_bath_rate folds (src/swarm/col_bath_rate.cu:30-58: _get_col_chain_rate /
 * measure times the outcome factor of _erosion_outcome_moments) for `count` owners listed in
 * dev_owner_ids, with the current particle state as reservoir and the handle's neighbour cache:
 * dev_out[count][n_k][5] = rate, rate*mean, rate*second, maximum, pair speed. */
gd_status gd_pair_rates(gd_handle *h, const gd_particle *dev_particle, const int32_t *dev_owner_ids, int count,
                        double total_dust_mass, double *dev_out);

/* col_bath_rate (src/swarm/col_bath_rate.cu:13-130) for every owner, alone: the bath-start rate
 * moments [n_p][4] = (rate or -1 when invalid, first, second, maximum) on the handle's neighbour
 * cache, with the current particle state as the published reservoir; the operator's own state is
 * left unchanged (the call uses scratch and synchronises). */
gd_status gd_bath_rates(gd_handle *h, const gd_particle *dev_particle, double total_dust_mass, double *dev_cached4);

/* One frozen bath of `bath` seconds for every owner, launched eagerly, not in a graph: col_bath_rate
 * (src/swarm/col_bath_rate.cu:13-130), col_skip_scan (src/swarm/col_skip_scan.cu:13-59) and
 * col_chain_run (src/swarm/col_chain_run.cu:21-404) on the handle's neighbour cache, with the current
 * particles as the published reservoir.  This is one wave of evolve_local_collisions
 * (inc/swarm/_col_chain.cuh:36-539) when a single bath covers the operator: the particles and the
 * RNG streams advance exactly as gd_collision_operator with that one wave advances them.  *events
 * (optional) receives the number of events.  The per-owner chain state is scratch (the call
 * synchronises); the handle's operator state is left unchanged.  Chain errors are reported as
 * GD_ERR_CHAIN / GD_ERR_CONTINUATION_LIMIT with the reference's code as detail. */
gd_status gd_bath_chain(gd_handle *h, gd_particle *dev_particle, void *dev_rngstate, double total_dust_mass,
                        double bath, unsigned long long *events);

/* Number of CUDA kernels this handle has launched since gd_create (for launch accounting). */
long long gd_launch_count(const gd_handle *h);

/*
 * Batched neighbour search: S independent swarms of uneven size n_p[s] and neighbour count n_k[s]
 * per call.  No counterpart in the reference, which runs one swarm per process.  All swarms share
 * the model constants of cfg except n_k.  Every swarm keeps its own geometry (the one-swarm build
 * kernels, run side by side on internal streams) and one persistent launch computes the top-K of
 * every bucket of every swarm; each swarm's rows are bit-identical to gd_geometry_build + gd_knn on
 * that swarm alone.
 *
 * Buffers are concatenated swarm by swarm: dev_particle [sum n_p], dev_measure and dev_kth_d2
 * [sum n_p], dev_codes [sum n_p[s] * n_k[s]] (swarm s's rows start at sum_{t<s} n_p[t] n_k[t]).
 * The non-finite screen is deferred: gd_batch_knn makes no host synchronisation (so it can be
 * captured into a CUDA graph on the batch's stream) and gd_batch_check reports a non-finite
 * particle (GD_ERR_NONFINITE, detail = its index in dev_particle).
 */
typedef struct gd_batch gd_batch;
gd_status gd_batch_create(const gd_config *cfg, int S, const int *n_p, const int *n_k, gd_batch **out);
void      gd_batch_destroy(gd_batch *b);
gd_status gd_batch_set_stream(gd_batch *b, void *stream);
gd_status gd_batch_knn(gd_batch *b, const gd_particle *dev_particle, int32_t *dev_codes, double *dev_measure,
                       float *dev_kth_d2);
gd_status gd_batch_check(gd_batch *b);
/* The collision operator of every swarm of the batch (evolve_local_collisions,
 * inc/swarm/_col_chain.cuh:108-539), on the rows of the last gd_batch_knn: swarm s advances its
 * particles (dev_particle from part offset s) and RNG states by durations[s] with
 * lambda_0 = n_p[s] / (n_k[s] total_dust_masses[s]), with its own bath controller.  Each swarm's
 * operator is one conditional-node graph (as gd_collision_operator's), and the swarms' graphs run
 * side by side on forked streams; each swarm's result is bit-identical to gd_collision_operator on
 * that swarm alone.  On a stream that is not capturing the call runs them and returns the first
 * error (detail = the swarm); inside the caller's capture of the batch's stream (after one eager
 * call, which allocates the swarms' operator state) the operators join the caller's graph, whose
 * results gd_batch_check returns after it ran.  dev_codes and dev_measure are gd_batch_knn's
 * outputs. */
gd_status gd_batch_collide(gd_batch *b, gd_particle *dev_particle, void *dev_rng, const int32_t *dev_codes,
                           const double *dev_measure, const double *durations, const double *total_dust_masses);
/* Controller statistics of swarm s's last operators (as gd_last_operator_stats). */
gd_status gd_batch_operator_stats(const gd_batch *b, int s, gd_operator_stats *out);
/* Every swarm's bath controller memory afresh (gd_reset_controller for each swarm, an output
 * boundary); results of captured operators not read yet are read first. */
gd_status gd_batch_reset_controller(gd_batch *b);
/* Positions changed without a new gd_batch_knn: the operators rebuild their owner lists. */
gd_status gd_batch_invalidate(gd_batch *b);
gd_status gd_batch_set_tuning(gd_batch *b, const gd_tuning *t);  /* walk, prescan, block width, sort */
size_t    gd_batch_last_error(const gd_batch *b, char *buf, size_t len);
long long gd_batch_error_detail(const gd_batch *b);
long long gd_batch_launch_count(const gd_batch *b);

/*
 * Handle-free exact top-K neighbour search that allocates no device memory.  No counterpart in
 * the reference (whose col_site_init / col_cache_get run on the swarm's allocated buffers).
 *
 * For callers that cannot call cudaMalloc while they run: a host that gives the whole device to its
 * own memory pool at start-up and permits no allocation outside it, or a time loop that cannot pay
 * the device-wide synchronisation cudaMalloc/cudaFree can cause.  gd_create allocates per swarm;
 * this entry point does not.
 *
 * Runs the same site init, Morton radix sort, bucket-tree build and top-K query as
 * gd_geometry_build + gd_knn, and writes the same dev_codes [n_p][n_k], dev_measure [n_p] and
 * dev_kth_d2 [n_p] (all three required, caller-allocated).  Its scratch is one fixed file-scope
 * device array of 4,407,552 bytes, which every device that loads the library holds until the
 * process exits; it bounds n_p to 65536.  A larger n_p returns GD_ERR_CAPACITY with a message,
 * before any device work.  A non-finite particle returns GD_ERR_NONFINITE with its index in
 * *detail.  detail and msg (msg_len bytes, NUL-terminated) may be NULL.
 *
 * The first call on each device, with that device current, looks up the scratch's device address
 * (this can load the library's device code on that device); make that first call before any stream
 * capture begins.  The address is kept for the life of the process, so after a cudaDeviceReset of a
 * device this entry point must not be called on that device again.  The call synchronises `stream`
 * once (the non-finite screen) and returns with the query enqueued on it.  All calls on one device share the one scratch: calls whose GPU work
 * overlaps (from several host threads, or on streams with no ordering between them) race and
 * corrupt each other's results; order them on one stream or serialise them.
 */
gd_status gd_knn_static(const gd_config *cfg, const gd_particle *dev_particle, int n_p, int32_t *dev_codes,
                        double *dev_measure, float *dev_kth_d2, void *stream, long long *detail, char *msg,
                        size_t msg_len);

/* ---- Checkpoints in the reference's on-disk formats (inc/swarm/swarm_host.cuh:776-914, 1142-1205) --
 * <prefix>particle_<frame>.dat holds n 64-byte records with the azimuthal and polar velocities as
 * linear speeds (save_sam_as_velocity); <prefix>rngstate_<frame>.dat holds the n raw 48-byte
 * cuRAND states.  <frame> is idx_file zero padded to max(5, digits of save_max) (frame_num).
 * `prefix` is prepended as is (the reference's PATH ends with '/').  Synchronous. */
gd_status gd_frame_name(int idx_file, int save_max, char *buf, size_t len);

/* In-place conversion of host particle records between the internal layout (angular velocities)
 * and the file layout, exactly as the reference converts them before writing and after reading. */
gd_status gd_particles_to_file_layout(const gd_config *cfg, gd_particle *host, int n);
gd_status gd_particles_from_file_layout(const gd_config *cfg, gd_particle *host, int n);

/* SAVE_PARTICLE_TO_FILE / LOAD_PARTICLE_TO_VRAM: particles (and, when dev_rng is not NULL, the
 * RNG states) of n particles in device memory to / from the frame's files.  A load checks the
 * exact file sizes first and returns GD_ERR_IO on any mismatch. */
gd_status gd_save_checkpoint(const gd_config *cfg, const char *prefix, int idx_file, int save_max,
                             const gd_particle *dev_particle, int n, const void *dev_rng);
gd_status gd_load_checkpoint(const gd_config *cfg, const char *prefix, int idx_file, int save_max,
                             gd_particle *dev_particle, int n, void *dev_rng);

/* ---- variables.txt (save_variable, inc/swarm/swarm_host.cuh:989-1143) ------------------------------
 * The parameter file a GameDev run writes beside its output (swarm_runtime.cu:290-291), which the
 * reference's analysis scripts read.  The collision constants come from cfg.  The rest of a model
 * directory's settings, most of them outside the collision path, come in gd_run_info: its
 * compile-time flags and the constants those flags bring in.  Without a flag, its constants are
 * not written, as in the reference.  The search written is cfg->search. */
typedef struct gd_run_info {
    int multisize, transport, diffusion, radiation, pr_effect, visc_flow, importgas;
    int log_output;     /* LOGTIMING or LOGOUTPUT: writes LOG_BASE = out_base, else LIN_BASE */
    int save_max, out_base;
    int col_bath_tpb;   /* COL_BATH_TPB of the model (the reference's bath-rate block width) */
    double metal_z, schmidt_x, schmidt_r, schmidt_z;
    double beta_0, kappa_0, t_beta, c_light;
    double dt_out, dt_max, cfl_dyn;
} gd_run_info;
/* Writes `path` as save_variable(path, total_dust_mass) does for a model with N_P = n_p, byte for
 * byte.  Host only.  GD_ERR_IO when the file cannot be written. */
gd_status gd_save_variables(const gd_config *cfg, const gd_run_info *run, int n_p, double total_dust_mass,
                            const char *path);

/* ---------------------------------------------------------------------------------------------
 * The Strang step of the reference's time loop (src/swarm/swarm_runtime.cu:504-601), for a model
 * with TRANSPORT (and DIFFUSION in 3D, optionally RADIATION, PR_EFFECT and VISC_FLOW, analytic gas):
 *     dt = min(DT_MAX, 1 / max rate, dt_out - clock_out)          dyn_rate_calc (dyn_rate_calc.cu)
 *     C(dt/2)  D(dt/2)  T(dt)  D(dt/2)  C(dt/2)
 * with C the collision operator (gd_evolve_collisions), D diffusion_pos (diffusion_pos.cu) and T
 * ssa_transport, or with RADIATION ssa_substep_1, the optical depth (optdepth_*.cu) and
 * ssa_substep_2.  The model's dynamics settings come in gd_run_info (transport, diffusion,
 * radiation, pr_effect, visc_flow, schmidt_*, beta_0, kappa_0, t_beta, c_light, dt_max, cfl_dyn);
 * importgas is not supported (GD_ERR_INVALID_ARGUMENT).  The clocks live on the device: each step
 * advances clock_sim and clock_out by its dt. */

/* Sets the device clocks: clock_sim (time since the start), clock_out (time into the current
 * output interval) and the interval length dt_out.  Enqueued on the handle's stream. */
gd_status gd_set_clock(gd_handle *h, double clock_sim, double clock_out, double dt_out);
/* Reads the clocks, the last step's dt and the steps taken since gd_set_clock.  Synchronises. */
gd_status gd_get_clock(gd_handle *h, double *clock_sim, double *clock_out, double *dt_last, int *steps);
/* One step of the dynamics alone: the timestep, D(dt/2) T(dt) D(dt/2), the clocks advanced.  No
 * host synchronisation.  Invalidates the geometry. */
gd_status gd_dynamics_step(gd_handle *h, const gd_run_info *run, gd_particle *dev_particle, void *dev_rng);
/* One full step, collisions included.  With radius_model (may be NULL) each geometry rebuild after
 * the first searches with the learned proposal seeded by the previous search's K-th distances; the
 * rows are the plain query's either way.  The collision halves read dt / 2 on the device, so the
 * step reads nothing back between its kernels except the operators' results: eagerly, the call
 * returns the first error met.  On a stream the caller is capturing, the whole step (screen or
 * geometry, learned top-K, two graph-captured collision operators, dynamics, clocks) joins the
 * caller's graph; capture it after one eager gd_step with the same arguments (the buffers are
 * allocated then), and call gd_check_step after each replay. */
gd_status gd_step(gd_handle *h, const gd_run_info *run, gd_particle *dev_particle, void *dev_rng,
                  double total_dust_mass, gd_radius_model *radius_model);
/* After a replay of captured gd_step calls: the non-finite screen of the last geometry build
 * (GD_ERR_NONFINITE with the particle index, as the eager step reports it), else the first error
 * of their collision operators; brings the operators' statistics and bath records to the host.
 * Synchronises the handle's stream. */
gd_status gd_check_step(gd_handle *h);

#ifdef __cplusplus
}
#endif

#endif /* GD_B200_H */
