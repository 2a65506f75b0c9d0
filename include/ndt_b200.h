/*
 * ndt_b200 -- C ABI of the B200 NDT scan-to-map registration library.
 *
 * This is the drop-in boundary for the DAPHNE ndt_mapping align call.  The
 * reference binds it as a C++ member function,
 *     CallbackResult ndt_mapping::partial_points_callback(
 *         PointCloud& input_cloud, Matrix4f& init_guess, PointCloud& target_cloud)
 * (src/CPU/ndt_mapping/kernel.cpp:1405; CUDA port src/Cuda/ndt_mapping/kernel.cu:1489),
 * with CallbackResult{bool converged; Matrix4f final_transformation; double fitness_score}
 * (src/CPU/ndt_mapping/datatypes.h:51-55), PointXYZI = float[4] and Matrix4f =
 * float[4][4] row major (datatypes.h:11-17).  Every entry point here takes plain
 * pointers and sizes with exactly those layouts: a cloud is `n` consecutive
 * float[4] (x, y, z, intensity) records, a transform is 16 floats row major.
 *
 * Status codes: 0 = ok, negative = error (see NDT_E_*); ndt_last_error()
 * returns a message for the last failing call on a context.  A context owns
 * its device buffers and CUDA stream; use one context per host thread.
 * There is no CPU fallback: without a usable sm_100 device every call that
 * needs the GPU returns NDT_E_CUDA.
 */
#ifndef NDT_B200_H
#define NDT_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define NDT_API __attribute__((visibility("default")))
#else
#define NDT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define NDT_OK 0
#define NDT_E_ARG (-1)       /* bad argument (NULL pointer, negative size, ...) */
#define NDT_E_CUDA (-2)      /* a CUDA runtime call failed (message in ndt_last_error) */
#define NDT_E_NOMAP (-3)     /* align called before a map was set */
#define NDT_E_GRID (-4)      /* voxel grid too large for 32-bit cell indices */
#define NDT_E_WATCHDOG (-5)  /* the iteration watchdog stopped an alignment */
#define NDT_E_CAPACITY (-6)  /* a size exceeds a fixed capacity of the call */

/* Per-alignment status bits written by the batch calls. */
#define NDT_ST_OK 0
#define NDT_ST_WATCHDOG 1  /* the evaluation budget ran out before convergence */
#define NDT_ST_OVERFLOW 2  /* more pairs with degenerate voxels than the FP64 side queue holds */

/*
 * Registration parameters.  ndt_params_reference() fills the values the
 * reference kernel hard-codes (kernel.cpp:37-57): outlier 0.55, resolution 1.0,
 * step 0.1, transformation_epsilon 0.1, max_iterations 0, compat 1.
 *
 * compat = 1 reproduces the reference kernel's behaviour bit for bit where it
 * is deterministic (dense grid scaled by the grid size, permuted quaternion
 * pose build without translation, fixed Newton step, its Hessian formula).
 * compat = 0 runs the corrected NDT (per-voxel covariance with a minimum point
 * count and eigenvalue floor, T = Trans * Rx * Ry * Rz, More-Thuente line
 * search, ||dp|| stop test) whose FP64 restatement is the accuracy oracle.
 */
typedef struct ndt_params {
    float resolution;              /* voxel edge length [m] (kernel.cpp:38) */
    int32_t copy_groups;           /* host-buffer batch calls: alignment groups whose host-to-device
                                      copy overlaps the previous group's rounds (0 = by size) */
    double outlier_ratio;          /* kernel.cpp:37 */
    double step_size;              /* More-Thuente step_max (kernel.cpp:40) */
    double transformation_epsilon; /* step_min = eps/2 and |step| < eps stop (kernel.cpp:56) */
    int32_t max_iterations;        /* Newton iterations beyond the first (kernel.cpp:57) */
    int32_t compat;                /* 1 = reference behaviour, 0 = corrected NDT */
    int32_t min_points_per_voxel;  /* compat = 0 only: voxels with fewer points are empty */
    int32_t precision;             /* per-pair arithmetic: 0 = FP32 (default), 1 = FP64 */
    double eigen_ratio;            /* compat = 0 only: covariance eigenvalue floor ratio */
    int32_t watchdog_evals;        /* max derivative evaluations per alignment (0 = 1024) */
    int32_t dense_probe;           /* 1 = FP32 pass probes the dense cell index for all 27 cells of a
                                      point; 0 = it reads the probe-window table (built with the grid when
                                      it fits, same pairs) */
} ndt_params;

typedef struct ndt_ctx ndt_ctx;

/* Parameter presets. */
NDT_API void ndt_params_reference(ndt_params *p); /* reference kernel values, compat = 1 */
NDT_API void ndt_params_corrected(ndt_params *p); /* corrected NDT: compat = 0, eps 0.01, 30 iterations */

/* Context life cycle.  device = CUDA ordinal. */
NDT_API int ndt_create(const ndt_params *params, int device, ndt_ctx **out);
NDT_API void ndt_destroy(ndt_ctx *ctx);
NDT_API const char *ndt_last_error(const ndt_ctx *ctx);

/*
 * Map (target cloud) upload + voxel grid build, once per map.  Replaces the
 * per-call grid rebuild of ndt_mapping::initCompute (kernel.cpp:1302-1373);
 * the resulting grid is identical to the one the reference builds for the
 * same cloud.  `map` is a HOST pointer to m float[4] points.
 */
NDT_API int ndt_set_map(ndt_ctx *ctx, const float *map, int m);
/* Same, but `map` is a device pointer (no host copy). */
NDT_API int ndt_set_map_device(ndt_ctx *ctx, const float *d_map, int m);

/*
 * Map growth (ndt_mapping's map grows by the aligned scans it appends; each
 * reference test case carries its map, kernel.cpp:210-229).  Appends k points
 * (HOST pointer, or DEVICE pointer for the _device form) to the current map;
 * the grid afterwards is the one ndt_set_map builds for the whole grown map,
 * bit for bit.  When the new points lie inside the bounding box of the map's
 * points the update is incremental: the new points' cells are sorted and
 * merged into the map's sorted cells and the voxel records recomputed, with no
 * new sort of the whole map; otherwise the grid is rebuilt.  The context keeps
 * its own copy of the grown map: after ndt_set_map_device the caller's map
 * buffer must still hold the map when the first append is made.
 */
NDT_API int ndt_map_append(ndt_ctx *ctx, const float *points, int k);
NDT_API int ndt_map_append_device(ndt_ctx *ctx, const float *d_points, int k);

/*
 * One alignment with host buffers: the partial_points_callback call
 * (kernel.cpp:1405-1414) against the map set by ndt_set_map.
 * out16 = final transformation, *converged, *fitness (NDT score per point;
 * the reference never fills fitness_score).  Returns NDT_E_WATCHDOG when the
 * evaluation budget (params.watchdog_evals) ran out and NDT_E_CAPACITY when
 * the FP64 side queue overflowed (NDT_ST_* of the batch calls); the outputs
 * are written in both cases.
 */
NDT_API int ndt_align(ndt_ctx *ctx, const float *scan, int n, const float guess16[16], float out16[16],
              int *converged, double *fitness);

/*
 * partial_points_callback exactly as the reference shapes it: the map comes
 * with the call and the grid is built from it (kernel.cpp:1375-1392).
 */
NDT_API int ndt_align_with_map(ndt_ctx *ctx, const float *scan, int n, const float guess16[16],
                       const float *map, int m, float out16[16], int *converged,
                       double *fitness);

/*
 * B independent alignments against the current map in one batched GPU pass
 * (the loop of ndt_mapping::run, kernel.cpp:1425-1429, for one map).
 * scans[b] -> ns[b] points (HOST pointers), guesses = B x 16 floats,
 * out = B x 16 floats, converged/fitness/status = B entries (status may be NULL).
 */
NDT_API int ndt_align_batch(ndt_ctx *ctx, int B, const float *const *scans, const int *ns,
                    const float *guesses, float *out, int *converged, double *fitness,
                    int *status);

/*
 * Device-resident batch: scans concatenated in d_points (sum(ns) float[4]),
 * d_offsets = B+1 prefix offsets (int32, device), d_guesses = B x 16 floats
 * (device); results to device buffers d_out (B x 16), d_conv (B), d_fit (B),
 * d_status (B).  Enqueued on the context stream; call ndt_synchronize().
 */
NDT_API int ndt_align_batch_device(ndt_ctx *ctx, int B, const float *d_points, const int *d_offsets,
                           int total_points, const float *d_guesses, float *d_out, int *d_conv,
                           double *d_fit, int *d_status);
NDT_API int ndt_synchronize(ndt_ctx *ctx);

/*
 * Host batch with the scans packed in one HOST buffer: points = sum(ns)
 * float[4], offsets = B+1 prefix offsets (int32).  One host-to-device copy;
 * the call returns when the results are in `out`, `converged`, `fitness`,
 * `status` (status may be NULL).  The batch form of ndt_mapping::run's loop
 * (kernel.cpp:1425-1429) for one map.
 */
NDT_API int ndt_align_batch_packed(ndt_ctx *ctx, int B, const float *points, const int *offsets,
                                   const float *guesses, float *out, int *converged, double *fitness,
                                   int *status);

/*
 * The same with the batch's map, as the reference's align call takes the map
 * every time (partial_points_callback(scan, guess, map), kernel.cpp:1405,
 * which rebuilds the grid: ndt_align, :1375-1392): map = m float[4] points
 * (HOST).  The map is uploaded first and its grid built while the scans are
 * copied, so the build overlaps the copies; the grid then stays set as after
 * ndt_set_map.
 */
NDT_API int ndt_align_batch_packed_with_map(ndt_ctx *ctx, const float *map, int m, int B, const float *points,
                                            const int *offsets, const float *guesses, float *out, int *converged,
                                            double *fitness, int *status);

/* The context's CUDA stream (cudaStream_t), for callers that time or order work. */
NDT_API void *ndt_stream(ndt_ctx *ctx);

/*
 * Work counters of the last batch call (reset by each batch / set_map call):
 * alignment-evaluations, derivative-pass work (scan points visited, in-bounds
 * cell probes, probes that found a voxel, accepted (point, voxel) pairs),
 * kernel launches, lockstep rounds and, with profiling on (ndt_set_profiling),
 * the summed derivative-pass time and the grid-build time measured with CUDA
 * events on the context stream.  No reference counterpart.
 */
typedef struct ndt_counters {
    int64_t evaluations;
    int64_t points;
    int64_t probes;
    int64_t occupied_probes;
    int64_t pairs;
    int64_t tiles;
    int64_t launches;
    int64_t rounds;
    int64_t deriv_launches;
    double deriv_ms;
    double grid_ms;
} ndt_counters;
NDT_API int ndt_set_profiling(ndt_ctx *ctx, int on);
NDT_API int ndt_get_counters(ndt_ctx *ctx, ndt_counters *out);

/*
 * Batch execution as CUDA graphs (default on): each batch call launches one
 * cached graph (tile lists, initialisation, a device-side loop of rounds that
 * ends when no alignment asks for another evaluation or the evaluation
 * watchdog is spent, results), so the host neither polls nor synchronises
 * between rounds.  Off, or with profiling on, the rounds are launched one by
 * one from the host (profiling times each derivative pass with events).  No
 * reference counterpart.
 */
NDT_API int ndt_set_batch_graphs(ndt_ctx *ctx, int on);

/*
 * NDT score of B scans at given poses (one derivative pass, no iteration):
 * d_score[b] = the score of computeDerivatives (kernel.cpp:651-705; the
 * corrected mode's objective when compat = 0), higher = better fit.  Device
 * arrays as ndt_align_batch_device (d_poses: B x 16 row major).  Used to judge
 * a learned pose proposal against the raw guess.  No reference counterpart.
 */
NDT_API int ndt_score_batch_device(ndt_ctx *ctx, int B, const float *d_points, const int *d_offsets,
                                   int total_points, const float *d_poses, double *d_score);

/*
 * Launch shape of the FP32 derivative pass (points per tile = threads per
 * block, resident blocks per SM).  A new context starts with variant 6
 * (128 x 6), the fastest on B200 for the corrected-mode benchmark workload.  ndt_autotune_batch_device times a caller's batch with every
 * variant (one warm call, then `repeats` timed calls each, CUDA events on the
 * context stream, minimum taken), selects the fastest on the context and
 * returns it in *best, with the times in ms_per_variant (optional,
 * ndt_kernel_variants() entries), then times the chosen shape with 4, 6 and 8
 * tiles per chunk and keeps the fastest (ndt_get_chunk_tiles reads it);
 * ndt_autotune_batch takes the batch in host buffers (packed as
 * ndt_align_batch_packed).  The variant and the chunk size change only the
 * FP32 summation order, never which pairs are evaluated; with both fixed, an
 * alignment's result does not depend on the rest of its batch.  No reference
 * counterpart (the reference has no GPU derivative pass).
 *
 * ndt_set_chunk_tiles: tiles of consecutive points per unit of work the FP32
 * pass hands out (1..64; default 8).  Larger chunks pay the per-chunk hand-out
 * and block reduction less often; smaller ones balance the end of a pass over
 * fewer tiles better.
 */
NDT_API int ndt_kernel_variants(void);
NDT_API int ndt_kernel_variant_shape(int variant, int *tile, int *blocks_per_sm);
NDT_API int ndt_set_kernel_variant(ndt_ctx *ctx, int variant);
NDT_API int ndt_get_kernel_variant(ndt_ctx *ctx);
NDT_API int ndt_set_chunk_tiles(ndt_ctx *ctx, int tiles);
NDT_API int ndt_get_chunk_tiles(ndt_ctx *ctx);
NDT_API int ndt_autotune_batch_device(ndt_ctx *ctx, int B, const float *d_points, const int *d_offsets,
                                      int total_points, const float *d_guesses, int repeats, int *best,
                                      float *ms_per_variant);
NDT_API int ndt_autotune_batch(ndt_ctx *ctx, int B, const float *points, const int *offsets, const float *guesses,
                               int repeats, int *best, float *ms_per_variant);

/*
 * Capacity of the FP64 side queue, in (point, voxel) pairs per derivative
 * pass (0 = the default, 2^20; at most 2^24; 16 bytes of device memory per
 * pair).  The queue holds the pairs whose voxel has a non-finite or huge
 * inverse covariance (the reference's inf / NaN voxels, kept bit for bit by
 * evaluating them in FP64).  Alignments of a pass that queued more pairs get
 * status NDT_ST_OVERFLOW and results that leave out the pairs beyond the
 * capacity.  No reference counterpart (the reference evaluates every pair in
 * FP64).
 */
NDT_API int ndt_set_side_queue_capacity(ndt_ctx *ctx, int pairs);

/*
 * Grid inspection (tests): bbox (min xyz, max xyz), dims, number of occupied
 * cells, and for each occupied cell its linear index, point count, mean[3]
 * (FP64) and inverse covariance[9] (FP64) as the reference stores them.
 * Pass NULL arrays to query sizes only.
 */
NDT_API int ndt_grid_info(ndt_ctx *ctx, float *bbox6, int *dims3, int *occupied);
NDT_API int ndt_grid_cells(ndt_ctx *ctx, int cap, int *cell_index, int *count, double *mean3,
                   double *icov9);

/*
 * Probe-window table of the current map (built with the grid unless
 * params.dense_probe = 1 or it would exceed 2^28 windows or entries): number
 * of windows and of entries; both 0 when the FP32 pass probes the dense index.
 * No reference counterpart (a lookup structure of this library).
 */
NDT_API int ndt_window_info(ndt_ctx *ctx, long long *windows, long long *entries);

/*
 * One derivative evaluation (computeDerivatives, kernel.cpp:651-705) of a
 * scan already transformed by the caller, at pose vector p6 (for the angle
 * terms), against the current map.  HOST buffers.  Returns score via *score.
 */
NDT_API int ndt_derivatives(ndt_ctx *ctx, const float *scan, const float *trans, int n,
                    const double p6[6], double *score, double g6[6], double H36[36]);

/*
 * ndt_derivatives_noalloc -- no counterpart in the reference.  The same
 * evaluation as ndt_derivatives, for callers that cannot allocate device
 * memory while they run (a real-time loop with a fixed memory budget, where
 * cudaMalloc can block and take unbounded time, or code running while
 * another component owns all of the device's memory): it allocates nothing.  Inputs are DEVICE pointers: d_scan and d_trans (n float[4] each,
 * the original and the already transformed scan, both 16-byte aligned), p6
 * is a host array (the pose vector for the angle terms); d_out (8-byte
 * aligned) receives 44 doubles: score, gradient[6], Hessian[36] row major,
 * pair count.  Misaligned pointers give NDT_E_ARG before any work.
 * Scratch is one static device array per GPU (at most 256 KB, held until
 * exit), which fixes two limits: n <= 65536 (NDT_E_CAPACITY beyond), and at
 * most 2048 (point, voxel) pairs evaluated on the FP64 side path (voxels with
 * non-finite or huge inverse covariance, points beyond ~1e6 m) per call --
 * beyond that the pair count d_out[43] is -1 and the other outputs are not
 * valid (ndt_derivatives holds 2^20 such pairs).  The first call on a device
 * looks the array up (cudaGetSymbolAddress); make it before any stream
 * capture.  The call leaves the caller's current device as it found it.
 * Work is enqueued on the context stream (call ndt_synchronize before
 * reading d_out); calls whose work overlaps on one GPU race on the shared
 * scratch.
 */
NDT_API int ndt_derivatives_noalloc(ndt_ctx *ctx, const float *d_scan, const float *d_trans, int n,
                                    const double p6[6], double *d_out);

/*
 * Learned initial pose (no counterpart in the reference): a point-feature
 * network that reads a scan transformed by its guess and proposes a pose
 * correction for the NDT to refine.  Per point u (3) -> 64 -> 128 (shared
 * layers, ReLU; the 64 -> 128 layer in BF16 on the tensor cores with FP32
 * accumulation), max-pool over up to max_points evenly strided points of the
 * scan, then 128 -> 64 -> 6 (both head layers, and in training every GEMM of
 * the head's backward, in BF16 on the tensor cores over tiles of 128 scans).  u = (T_guess x - center) / scale; the output y
 * is the correction of the pose vector (x, y, z, roll, pitch, yaw of the
 * corrected parametrisation T = Trans Rx Ry Rz) in units of delta_scale6.
 * Weights: ndt_mlp_num_weights() FP32 values (W1[64][3], b1[64], W2[128][64],
 * b2[128], W3[64][128], b3[64], W4[6][64], b4[6]).  All arrays passed to the
 * *_device calls are device pointers; work is ordered on the network's own
 * stream (ndt_mlp_stream).  ndt_mlp_synchronize reports a tensor-core wait
 * that gave up (*tc_error != 0; the outputs are then invalid).
 */
typedef struct ndt_mlp ndt_mlp;
NDT_API int ndt_mlp_num_weights(void);
NDT_API int ndt_mlp_create(int device, ndt_mlp **out);
NDT_API void ndt_mlp_destroy(ndt_mlp *mlp);
NDT_API const char *ndt_mlp_last_error(const ndt_mlp *mlp);
NDT_API int ndt_mlp_set_input_frame(ndt_mlp *mlp, const float center3[3], float scale, const float delta_scale6[6]);
NDT_API int ndt_mlp_set_weights(ndt_mlp *mlp, const float *w, int n);  /* host array; resets Adam state */
NDT_API int ndt_mlp_get_weights(ndt_mlp *mlp, float *w, int n);        /* host array */
/* y6: B x 6 corrections (normalised units) for B scans (points: float4, offsets: B + 1, guesses: B x 16). */
NDT_API int ndt_mlp_forward_device(ndt_mlp *mlp, int B, const float *d_points, const int *d_offsets,
                                   const float *d_guesses, int max_points, float *d_y6);
/* One training step on B scans with targets (B x 6, normalised units): loss = mean over scans of
 * mean over the 6 outputs of (y - target)^2.  update = 1 applies Adam (lr, beta 0.9 / 0.999) to the
 * weights; update = 0 only computes.  h_loss (1 float) and h_grad (num_weights floats, the batch
 * gradient) are optional host outputs. */
NDT_API int ndt_mlp_train_step_device(ndt_mlp *mlp, int B, const float *d_points, const int *d_offsets,
                                      const float *d_guesses, const float *d_target6, int max_points, float lr,
                                      int update, float *h_loss, float *h_grad);
/* Max-pool of the last forward: B x 128 packed (float bits << 32 | 0xffffffff - argmax sample). */
NDT_API int ndt_mlp_maxpool_device(ndt_mlp *mlp, unsigned long long *d_out, int B);
/* Waits for the network's stream; *tc_error (optional) = 1 when a tensor-core wait gave up in a call since the
 * last ndt_mlp_synchronize (the outputs of those calls are then invalid); the flag is cleared once reported. */
NDT_API int ndt_mlp_synchronize(ndt_mlp *mlp, int *tc_error);
/* Polls of the tensor-core completion barrier before a wait gives up and sets the error flag (< 0: the default,
 * 2^26, which no healthy MMA reaches; 0 gives up before the first poll, which exercises the error path).  A wait
 * that gave up still waits, with the default limit, for the MMAs in flight before the kernel frees its tensor
 * memory and returns. */
NDT_API int ndt_mlp_set_wait_limit(ndt_mlp *mlp, int polls);
NDT_API void *ndt_mlp_stream(ndt_mlp *mlp);
/* Run the network's work on a caller's stream (e.g. ndt_stream of an NDT context, so that proposals, the
 * judge's scores and the refinement are ordered without host synchronisation); NULL = its own stream. */
NDT_API int ndt_mlp_set_stream(ndt_mlp *mlp, void *stream);
/* Proposals: `passes` times, y = network(scan at the current pose) and pose <- T(pose(current) + y *
 * delta_scale), starting from the guesses; d_prop16 receives the last poses (B x 16), d_y6 the last y. */
NDT_API int ndt_mlp_propose_device(ndt_mlp *mlp, int B, const float *d_points, const int *d_offsets,
                                   const float *d_guesses, int max_points, int passes, float *d_y6,
                                   float *d_prop16);
/* The NDT judge: d_start16[b] = proposal b where d_score_prop[b] >= d_score_guess[b] (scores of
 * ndt_score_batch_device), the raw guess otherwise; d_used[b] (optional) = 1 where the proposal won. */
NDT_API int ndt_mlp_judge_device(ndt_mlp *mlp, int B, const float *d_prop16, const float *d_guesses,
                                 const double *d_score_prop, const double *d_score_guess, float *d_start16,
                                 int *d_used);

/*
 * Learned-init batched alignment (no counterpart in the reference, whose align
 * call starts the NDT at the caller's guess: partial_points_callback,
 * src/CPU/ndt_mapping/kernel.cpp:1405-1414).  For B scans (d_points,
 * d_offsets: B + 1 prefix offsets) with guesses (B x 16), against contexts
 * levels[0 .. n_levels) that hold the same map at coarse-to-fine resolutions
 * (compat = 0):
 *   1. starts: each guess moved by a fixed pattern of K = grid_xy^2 x grid_yaw
 *      offsets (translations step_xy apart in the guess's heading frame, yaw
 *      offsets step_yaw_deg apart, centred on the guess);
 *   2. proposals: the network runs `passes` times from every start, each pass
 *      from the previous proposal (max_points points per scan);
 *   3. the judge: the NDT score of the K proposals and of the raw guess, on
 *      judge_points evenly strided points of the scan (0 = all), with the map
 *      of levels[judge_level]; each scan starts from its best-scoring
 *      candidate, the raw guess whenever no proposal scores higher;
 *   4. refinement: the plain NDT from that start through every level in order
 *      (level l reads level_points[l] evenly strided points per scan, 0 =
 *      all); the last level's result is the output.
 * Outputs (device): d_out (B x 16), d_conv, d_fit as ndt_align_batch_device;
 * d_status (optional) = OR of the levels' NDT_ST_* bits; d_choice (optional)
 * = the winning candidate per scan: k < K for the proposal from start k, K
 * for the raw guess; d_start16 (optional, B x 16) = the winning candidate's
 * pose, where the refinement started.  Work is enqueued on the network's and the contexts'
 * streams, ordered by events; the results are ready after
 * ndt_synchronize(levels[n_levels - 1]).  Inputs must be ready when called.
 * The pipeline's buffers belong to the network object: consecutive calls on
 * one network are ordered by the events, but one network must not be used
 * from two host threads at once (as a context must not).
 */
#define NDT_LEARNED_MAX_LEVELS 8
typedef struct ndt_learned_params {
    int32_t max_points;    /* network: points read per scan */
    int32_t passes;        /* network passes per start (0: the starts themselves are the candidates) */
    int32_t grid_xy;       /* starts: grid_xy x grid_xy translations ... */
    int32_t grid_yaw;      /* ... times grid_yaw yaw offsets */
    float step_xy;         /* translation spacing of the starts [m] */
    float step_yaw_deg;    /* yaw spacing of the starts [deg] */
    int32_t judge_level;   /* index of the level whose map scores the candidates */
    int32_t judge_points;  /* points per scan in the score pass (0 = all) */
    int32_t level_points[NDT_LEARNED_MAX_LEVELS];  /* points per scan at each refinement level (0 = all) */
} ndt_learned_params;
/* Defaults: 1024 points, 2 passes, a 3 x 3 x 3 grid of starts 2.5 m and 10 deg apart (for guesses within
 * +-3 m / +-15 deg), judge at level 0 on 2048 points. */
NDT_API void ndt_learned_params_default(ndt_learned_params *p);
NDT_API int ndt_align_batch_learned_device(ndt_mlp *mlp, ndt_ctx *const *levels, int n_levels,
                                           const ndt_learned_params *lp, int B, const float *d_points,
                                           const int *d_offsets, int total_points, const float *d_guesses,
                                           float *d_out, int *d_conv, double *d_fit, int *d_status, int *d_choice,
                                           float *d_start16);
/* The same with HOST buffers (the scans packed as ndt_align_batch_packed takes them: points = sum(ns)
 * float[4], offsets = B + 1 prefix offsets): copies in, the pipeline, copies out; returns when the results
 * are in out, converged, fitness, status, choice and start16 (the last three may be NULL). */
NDT_API int ndt_align_batch_learned(ndt_mlp *mlp, ndt_ctx *const *levels, int n_levels, const ndt_learned_params *lp,
                                    int B, const float *points, const int *offsets, const float *guesses, float *out,
                                    int *converged, double *fitness, int *status, int *choice, float *start16);

/*
 * The input file on the fast path (replaces the reference's one-value-at-a-
 * time reads of ndt_input.dat, parseInitGuess / parseFilteredScan,
 * kernel.cpp:143-173, read_next_testcases :192-229; same format).
 * ndt_dat_open maps the file read-only and indexes its test cases (a
 * truncated or malformed file gives NDT_E_ARG; *out is set even then, so that
 * ndt_dat_last_error can say why; close it with ndt_dat_close).
 * ndt_dat_case returns pointers into the mapping (valid until close).
 * ndt_dat_map_relation tells how case i's map relates to case i - 1's.
 * ndt_dat_align aligns cases [first, first + count) as the reference's run
 * loop would (each scan against its own case's map) and returns the results
 * in case order: the mapping is registered with the driver, so scans and maps
 * go to the device by asynchronous DMA from it; cases are aligned in chunks
 * of cases that share a map, the next chunk's upload overlapping the current
 * chunk's alignments; a map equal to the previous one reuses the grid, one
 * that extends it grows the grid (ndt_map_append), any other is built.
 */
#define NDT_DAT_MAP_NEW 0    /* a map unlike the previous case's */
#define NDT_DAT_MAP_SAME 1   /* byte-identical to the previous case's map */
#define NDT_DAT_MAP_GROWN 2  /* the previous case's map followed by more points */
typedef struct ndt_dat ndt_dat;
NDT_API int ndt_dat_open(const char *path, ndt_dat **out);
NDT_API void ndt_dat_close(ndt_dat *dat);
NDT_API const char *ndt_dat_last_error(const ndt_dat *dat);
NDT_API int ndt_dat_count(const ndt_dat *dat);
NDT_API int ndt_dat_case(const ndt_dat *dat, int i, const float **guess16, const float **scan, int *n,
                         const float **map, int *m);
NDT_API int ndt_dat_map_relation(const ndt_dat *dat, int i);
NDT_API int ndt_dat_align(ndt_ctx *ctx, ndt_dat *dat, int first, int count, float *out16, int *converged,
                          double *fitness, int *status);

/*
 * Scan pre-filter (no counterpart in the reference kernel: it is the
 * voxel-grid downsampling that produces the "filtered scan" inputs of the
 * align call upstream).  For each of B scans (d_points: float4 x, y, z,
 * intensity; d_offsets: B + 1 prefix offsets, d_offsets[B] = total_points)
 * the points with finite x, y, z fall into leaves (floor(x * r),
 * floor(y * r), floor(z * r)), r = 1 / leaf and each product rounded to float; every
 * occupied leaf yields one point, the mean of its points (all four
 * components, summed in double precision in input order, rounded to float).
 * A scan's output points are ordered by leaf, x fastest, then y, then z.
 * d_out: room for total_points float4; d_out_offsets: B + 1 output offsets;
 * *out_total (host) = number of output points.  NDT_E_CAPACITY when a scan
 * spans 2^31 leaves or more, or the batch 2^31 - 1 leaves or more.  The call
 * blocks until the result is ready (it reads the key range back once).
 */
typedef struct ndt_filter ndt_filter;
NDT_API int ndt_filter_create(int device, ndt_filter **out);
NDT_API void ndt_filter_destroy(ndt_filter *f);
NDT_API const char *ndt_filter_last_error(const ndt_filter *f);
NDT_API void *ndt_filter_stream(ndt_filter *f);
NDT_API int ndt_voxel_filter_device(ndt_filter *f, int B, const float *d_points, const int *d_offsets,
                                    int total_points, float leaf, float *d_out, int *d_out_offsets, int *out_total);

/*
 * Euclidean clustering (DAPHNE's euclidean_cluster kernel, whose radius
 * search builds an N x N distance matrix: src/CPU/euclidean_cluster/
 * kernel.cpp:512-647, CUDA port src/Cuda/euclidean_cluster/kernel.cu:506-560).
 * xyz: n points, 3 floats each (HOST).  Two points are neighbours when the
 * float dx*dx + dy*dy + dz*dz is <= tolerance * tolerance, as there; clusters
 * are the connected components.  ndt_ec_labels gives each point the smallest
 * index of its cluster.  ndt_ec_extract gives extract()'s clusters
 * (:635-647): sizes in [min_size, max_size], ordered as the reference orders
 * them, each point list ascending; cluster c is cluster_indices
 * [cluster_offsets[c], cluster_offsets[c + 1]) (capacities: n + 1 and n).
 * ndt_ec_segment runs segmentByDistance (:767-814): five distance rings with
 * their tolerances, clusters of 20..100000 points, and returns the clustered
 * points (out_xyz, capacity 3n floats; the reference colours them all
 * r, g, b = 10, 20, 30), the boxes that pass the reference's size filter (10
 * doubles each: position xyz, orientation xyzw, dimensions xyz; capacity 10n)
 * and their centroids (3 doubles each; capacity 3n).  The orientation is the
 * yaw of the reference's pose estimate (:720-745): the direction of the
 * minimum-area rectangle around the cluster's xy points (convex hull and
 * rotating calipers), as ndt_ec_box_yaw gives it.  NDT_E_CAPACITY when a cloud
 * spans more than 2^28 cells of the tolerance.
 */
typedef struct ndt_ec ndt_ec;
NDT_API int ndt_ec_create(int device, ndt_ec **out);
NDT_API void ndt_ec_destroy(ndt_ec *ec);
NDT_API const char *ndt_ec_last_error(const ndt_ec *ec);
NDT_API int ndt_ec_labels(ndt_ec *ec, const float *xyz, int n, float tolerance, int *labels);
NDT_API int ndt_ec_extract(ndt_ec *ec, const float *xyz, int n, float tolerance, int min_size, int max_size,
                           int *num_clusters, int *cluster_offsets, int *cluster_indices);
NDT_API int ndt_ec_segment(ndt_ec *ec, const float *xyz, int n, float *out_xyz, int *out_n, double *boxes,
                           int *num_boxes, double *centroids, int *num_centroids);
/* Host only (no device work): the yaw quaternion (z, w; x = y = 0) of one
 * cluster's box from its n points (xyz, 3 floats each), as clusterAndColor
 * computes it (kernel.cpp:720-745, minAreaRectAngle :479-502) with one
 * difference: the reference's minAreaRectAngle hands rotatingCalipers the
 * cluster's point count as the hull's length and reads past the end of the
 * hull, which makes its yaw depend on memory contents; here the hull's own
 * length is used.  NDT_E_ARG for a non-finite x or y. */
NDT_API int ndt_ec_box_yaw(const float *xyz, int n, double *qz, double *qw);
/* The same for C clusters packed in xyz (offsets: C + 1 point offsets), spread over the host's threads (up to
 * 8; a process forked after its first parallel call runs on one thread): qz[c], qw[c] of cluster c. */
NDT_API int ndt_ec_box_yaws(int C, const float *xyz, const int *offsets, double *qz, double *qw);
/* The same for C clouds packed in xyz (offsets: C + 1 point offsets), up to 8 clouds per GPU pass: cloud c's
 * clustered points are out_xyz[out_offsets[c] .. out_offsets[c + 1]), its boxes and centroids
 * [box_offsets[c] .. box_offsets[c + 1]) (capacities as above with n = offsets[C]). */
NDT_API int ndt_ec_segment_batch(ndt_ec *ec, int C, const float *xyz, const int *offsets, float *out_xyz,
                                 int *out_offsets, double *boxes, int *box_offsets, double *centroids);

#ifdef __cplusplus
}
#endif
#endif /* NDT_B200_H */
