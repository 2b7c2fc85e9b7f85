/*
 * splat_b200: the training step of a tile-based differentiable Gaussian
 * rasterizer on one NVIDIA B200 (sm_100a), behind a plain C ABI.
 *
 * The entry points mirror the reference trainer's class API, splat::Trainer
 * (src/train/trainer.hpp:89-270), method for method, so that the reference's
 * session loop (src/train/train.cpp:474-860) can drive this library through a
 * thin shim (include/splat_trainer.hpp) instead of its Vulkan trainer. Each
 * declaration names the reference interface it replaces.
 *
 * Conventions, as in the reference:
 *   - Gaussian clouds are given as the reference's GaussianCloud arrays
 *     (src/splat/gaussian_cloud.hpp:138-151): positions 3 floats per Gaussian,
 *     scales 3 (log of the standard deviations), rotations 4 (quaternion
 *     w, x, y, z, not necessarily normalised), opacities 1 (logit), SH
 *     3 * (degree + 1)^2 floats per Gaussian, ordered [coefficient][rgb].
 *   - Cameras are the reference's Camera (src/render/camera.hpp:84-89):
 *     OpenCV pinhole (x right, y down, z forward), a world->camera matrix
 *     stored column-major (view[column * 4 + row]), pixel (0,0) the top-left
 *     corner with pixel centres at +0.5.
 *   - Targets are RGBA8, width * height * 4 bytes.
 *   - Host pointers passed in are read during the call only, except the
 *     prefetched next target (see splat_trainer_step).
 *   - Every call returns a status (SPLAT_OK or an error below); the message of
 *     the last error on this thread is splat_last_error(). The reference
 *     throws instead: BudgetExceeded (trainer.hpp:46-49) maps to
 *     SPLAT_ERR_BUDGET, std::runtime_error on bad input (trainer.cpp:174,276,
 *     281,571) to SPLAT_ERR_INVALID, std::logic_error (trainer.cpp:853) to
 *     SPLAT_ERR_STATE.
 *   - A handle is used by one thread at a time, as the reference's Trainer.
 * Options the reference has but this library has no kernel for (the Mip
 * filters, SH dropout, second-order steps, pose gradients, position noise,
 * exposure) are refused with SPLAT_ERR_UNSUPPORTED; nothing falls back to the
 * CPU.
 */
#ifndef SPLAT_B200_H
#define SPLAT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum splat_status {
  SPLAT_OK = 0,
  SPLAT_ERR_INVALID = 1,     /* bad argument: sizes, counts, mismatched target */
  SPLAT_ERR_BUDGET = 2,      /* a view needs more memory than the budget allows (BudgetExceeded) */
  SPLAT_ERR_UNSUPPORTED = 3, /* an option this library has no kernel for */
  SPLAT_ERR_DEVICE = 4,      /* a CUDA error, or a device-side check that failed */
  SPLAT_ERR_NONFINITE = 5,   /* the loss came out NaN or infinite */
  SPLAT_ERR_STATE = 6,       /* called in the wrong order (e.g. gradients before compute_gradients) */
  SPLAT_ERR_NOMEM = 7        /* device allocation failed */
};

/* How the step is computed. The reference has one form; this library keeps the
 * reference's layout and arithmetic as the default and adds the B200 forms. */
enum splat_sh_storage {
  SPLAT_SH_F32 = 0,  /* SH above degree 0 in FP32 */
  SPLAT_SH_BF16 = 1, /* in bfloat16, rounded at random after each step */
  SPLAT_SH_F16 = 2   /* in FP16 as the reference (gaussian_cloud.hpp:164-173), rounded at random */
};
enum splat_state_storage {
  SPLAT_STATE_F32 = 0,      /* Adam moments in two FP32 words per parameter */
  SPLAT_STATE_BF16_PAIR = 1 /* one word of two bfloat16 per parameter, as the reference (train_gradient.comp:33-35) */
};
enum splat_sort_form {
  SPLAT_SORT_DEPTH_THEN_TILE = 0, /* the reference's order: 32-bit depth sort, then a stable sort by tile */
  SPLAT_SORT_TILE_DEPTH_64 = 1    /* one sort of 64-bit (tile << 32 | depth) keys */
};

/* TrainerOptions (src/train/trainer.hpp:24-42), plus the B200 knobs. */
typedef struct splat_trainer_options {
  float lambda_ssim;          /* 0.2 */
  float background[3];        /* 0, 0, 0 */
  float near_plane;           /* 0.01 */
  int32_t force_fixed_point;  /* 0: float atomics, 1: the bit-reproducible fixed-point backward */
  int32_t selective_adam;     /* 1 */
  float opacity_reg;          /* 0 */
  float scale_reg;            /* 0 */
  float position_noise;       /* 0; anything else is SPLAT_ERR_UNSUPPORTED */
  int32_t mip_filter_2d;      /* 0; 1 is SPLAT_ERR_UNSUPPORTED */
  int32_t pose_gradients;     /* 0; 1 is SPLAT_ERR_UNSUPPORTED */
  uint64_t memory_budget;     /* bytes; UINT64_MAX for none */
  /* B200 knobs. */
  int32_t sh_storage;         /* splat_sh_storage, default SPLAT_SH_F16 (the reference's) */
  int32_t state_storage;      /* splat_state_storage, default SPLAT_STATE_BF16_PAIR (the reference's) */
  int32_t sort_form;          /* splat_sort_form, default SPLAT_SORT_DEPTH_THEN_TILE */
  int32_t exact_math;         /* 1: deterministic exp/log, bit-reproducible by the CPU restatement; 0: SFU */
  int32_t use_graph;          /* 1: capture the step as a CUDA graph, entry count kept on the device */
  int32_t digit_bits;         /* radix digit width, 6..8 (0 picks 8) */
  int32_t forward_pixels_per_thread;  /* compositing layout. 1: the reference's 2x16-pixel warps (0 picks 1);
                                         2: 8x8-pixel warps, two pixels per lane */
  int32_t backward_pixels_per_thread; /* float backward layout, 1 or 2 as above (0 picks 2). The fixed-point
                                         backward always uses 1, as its sums follow the reference's 32-lane
                                         groups. */
  int32_t split_step;         /* 0: a one-view Adam step is one fused kernel (chain rule, geometry and SH
                                 step); 1: three kernels, as for batches. The results are the same bits. */
  int32_t blend_lists;        /* 0: the backward recomputes each pixel's transmittance in a reverse sweep,
                                 keeping 8 bytes per pixel (the reference's design). 1: store everything:
                                 the forward records every blended (entry, alpha) pair per pixel, 8 bytes
                                 each, and the backward walks those lists (float sums, one view, no CUDA
                                 graph: the list total is read back before the recording pass). For
                                 comparison of memory and speed. */
  int32_t tile_size;          /* rasterizer tile edge in pixels: 16 (the reference's; 0 picks it) or 32. 32
                                 applies where both rasterizer kernels take two pixels per thread and the sums
                                 are float (not with force_fixed_point or blend_lists); elsewhere the tile stays
                                 16. Images are the same bits either way. */
  int32_t batch_depth;        /* splats the two-pixel kernels stage per round: 128 or 256 (0 picks 128) */
  int32_t persistent_raster;  /* 1: the two-pixel kernels run as persistent launches, resident blocks taking
                                 the tiles of every view of the step from one counter; 0: one block per tile */
  int32_t grouped_backward;   /* the two-pixel float backward's sums. 0: each splat's twelve sums reduced over
                                 the warp by a butterfly (the reference's way); 1: for groups of splats, the
                                 pixels' two factors kept in shared memory and the sums made splat-parallel,
                                 one lane per (splat, share of the warp's pixels). Scored views use 0. */
} splat_trainer_options;

/* LearningRates (src/train/trainer.hpp:51-61); trust_region must be 0. */
typedef struct splat_learning_rates {
  float position;      /* 1.6e-4 */
  float scale;         /* 0.005 */
  float rotation;      /* 0.001 */
  float opacity;       /* 0.05 */
  float sh;            /* 0.025 */
  float sh_rest_scale; /* 0.05 */
  float trust_region;  /* 0 */
} splat_learning_rates;

/* StepStats (src/train/trainer.hpp:63-73). */
typedef struct splat_step_stats {
  float loss;
  float l1;
  float ssim;
  uint32_t visible_splats;
  uint32_t tile_entries;
  float exposure_gradient[12];
  float pose_gradient[6];
} splat_step_stats;

/* Camera (src/render/camera.hpp:84-89). */
typedef struct splat_camera {
  float view[16];     /* world -> camera, column-major */
  float position[3];  /* camera centre in world space */
  float fx, fy, cx, cy;
  int32_t width, height;
} splat_camera;

/* GaussianCloud (src/splat/gaussian_cloud.hpp:145-162), as host arrays. */
typedef struct splat_cloud {
  int32_t count;
  int32_t sh_degree;         /* 0..3 */
  const float *positions;    /* 3 * count */
  const float *scales;       /* 3 * count */
  const float *rotations;    /* 4 * count */
  const float *opacities;    /* count */
  const float *sh;           /* 3 * (sh_degree + 1)^2 * count */
} splat_cloud;

typedef struct splat_trainer splat_trainer;

/* The message of the last failed call on this thread ("" if none). */
const char *splat_last_error(void);

/* Fills the reference's defaults (TrainerOptions{}, LearningRates{}). */
void splat_trainer_options_default(splat_trainer_options *options);
void splat_learning_rates_default(splat_learning_rates *rates);

/* Trainer::Trainer (trainer.hpp:91, trainer.cpp:157-208). Uploads the cloud. */
int splat_trainer_create(const splat_cloud *cloud, const splat_trainer_options *options, splat_trainer **out);
/* Trainer::~Trainer. */
int splat_trainer_destroy(splat_trainer *trainer);

/* Trainer::render (trainer.hpp:98): width * height * 4 floats, rgb and the log transmittance. */
int splat_trainer_render(splat_trainer *trainer, const splat_camera *camera, float *out_pixels);

/* Trainer::compute_gradients (trainer.hpp:104): forward, loss, backward, and
 * gradients stored for splat_trainer_get_gradients. */
int splat_trainer_compute_gradients(splat_trainer *trainer, const splat_camera *camera, const uint8_t *target,
                                    size_t target_bytes, splat_step_stats *stats);
/* Trainer::score_view (trainer.hpp:111, trainer.cpp:521-532): the FastGS
 * scoring pass. A statistics pass over the view that marks the pixels whose
 * mean absolute error is at least error_share of the view's worst
 * (train_loss.comp:101-107, train_error_mask.comp), then adds to each
 * Gaussian's densification statistics the marked pixels it reached, that count
 * times the view's loss, and its edge score (the target's luminance Laplacian
 * times the blending weight), all in pixels times pixel_weight
 * (train_score.comp). error_share must be above 0; not with blend_lists. */
int splat_trainer_score_view(splat_trainer *trainer, const splat_camera *camera, const uint8_t *target, size_t target_bytes,
                             float error_share, float pixel_weight, splat_step_stats *stats);
/* Trainer::collect_statistics (trainer.hpp:106). */
int splat_trainer_collect_statistics(splat_trainer *trainer, const splat_camera *camera, const uint8_t *target,
                                     size_t target_bytes, splat_step_stats *stats);
/* The same two passes with the target already in device memory (an RGBA8
 * image the caller keeps in HBM, as the session keeps its views). */
int splat_trainer_collect_statistics_device_target(splat_trainer *trainer, const splat_camera *camera, const uint8_t *device_target,
                                                   size_t target_bytes, splat_step_stats *stats);
int splat_trainer_score_view_device_target(splat_trainer *trainer, const splat_camera *camera, const uint8_t *device_target,
                                           size_t target_bytes, float error_share, float pixel_weight, splat_step_stats *stats);
/* Trainer::apply_gradients (trainer.hpp:121): one Adam step from the sums the last
 * compute_gradients left. */
int splat_trainer_apply_gradients(splat_trainer *trainer, const splat_learning_rates *rates);
/* Trainer::step (trainer.hpp:125-126). next_target (may be NULL) is copied to
 * pinned staging memory while the GPU works on this step and must stay valid
 * until the next call that uses it. */
int splat_trainer_step(splat_trainer *trainer, const splat_camera *camera, const uint8_t *target, size_t target_bytes,
                       const splat_learning_rates *rates, const uint8_t *next_target, size_t next_target_bytes,
                       splat_step_stats *stats);
/* Trainer::step with the target already in device memory (device_target is a
 * device pointer of width * height * 4 bytes, read during the call: the loss
 * reads it where it is, without a copy, when it is 4-byte aligned). For
 * callers that keep their photos resident in HBM. New in this library. */
int splat_trainer_step_device_target(splat_trainer *trainer, const splat_camera *camera, const uint8_t *device_target,
                                     size_t target_bytes, const splat_learning_rates *rates, splat_step_stats *stats);
/* The CUDA stream (cudaStream_t) the trainer's work runs on, for callers that
 * time it with events or order their own work after it. */
int splat_trainer_stream(splat_trainer *trainer, void **stream);
/* Several views (up to 8, of any sizes) in one step: their forward and backward
 * passes share one set of launches, their gradients are summed and one Adam
 * step is taken. New in this library; stats receives one entry per view. */
int splat_trainer_step_batch(splat_trainer *trainer, const splat_camera *cameras, const uint8_t *const *targets,
                             int32_t views, const splat_learning_rates *rates, splat_step_stats *stats);
/* The same with the targets in device memory. */
int splat_trainer_step_batch_device_targets(splat_trainer *trainer, const splat_camera *cameras, const uint8_t *const *device_targets,
                                            int32_t views, const splat_learning_rates *rates, splat_step_stats *stats);
/* Trainer::prefetch_target (trainer.hpp:129). */
int splat_trainer_prefetch_target(splat_trainer *trainer, const uint8_t *target, size_t target_bytes);

/* Trainer::gradients (trainer.hpp:141-144), in GaussianCloud layout. */
int splat_trainer_get_gradients(splat_trainer *trainer, float *positions, float *scales, float *rotations, float *opacities,
                                float *sh);
/* Trainer::cloud (trainer.hpp:131). Arrays sized as the cloud given to create
 * (after splat_trainer_apply_changes, as the last cloud given). */
int splat_trainer_get_cloud(splat_trainer *trainer, float *positions, float *scales, float *rotations, float *opacities,
                            float *sh);
/* Trainer::set_active_sh_degree (trainer.hpp:151). */
int splat_trainer_set_active_sh_degree(splat_trainer *trainer, int32_t degree);
/* Trainer::densify_stats (trainer.hpp:176, trainer.cpp:686-708): 8 floats per
 * Gaussian: gradient sum, visits, largest radius, contribution, absolute
 * gradient sum, marked pixels, marked loss, edge score. */
int splat_trainer_get_densify_stats(splat_trainer *trainer, float *out);
/* Trainer::reset_densify_stats (trainer.hpp:178). */
/* Replaces the densification statistics (8 floats per Gaussian, the layout
 * splat_trainer_get_densify_stats reads), as restoring a paused run or a
 * test that sets them needs. */
int splat_trainer_set_densify_stats(splat_trainer *trainer, const float *raw);
int splat_trainer_reset_densify_stats(splat_trainer *trainer);
/* Trainer::reset_opacity (trainer.hpp:163, trainer.cpp:810-819). */
int splat_trainer_reset_opacity(splat_trainer *trainer, float maximum);
/* Trainer::apply_changes (trainer.cpp:749-787): replaces the Gaussians by
 * `cloud`; source[i] is the old index whose optimiser state Gaussian i keeps,
 * or -1 for a new one (fresh, zero state); an index past the old count is
 * SPLAT_ERR_INVALID. The state is gathered on the GPU (train_gather.comp)
 * into the trainer's spare buffers, which then take the current ones' place;
 * the densification statistics start anew. */
int splat_trainer_apply_changes(splat_trainer *trainer, const splat_cloud *cloud, const int32_t *source);

/* Trainer::remove_largest_gaussians, remove_least_contributing_gaussians,
 * remove_least_opaque_gaussians (trainer.hpp:174-183, trainer.cpp:731-747;
 * remove_largest, remove_least_contributing, remove_least_opaque of
 * densify.cpp:70-113): removes ceil(share * count) Gaussians, at most
 * count - 1, the highest first by their largest log-scale, by minus their
 * contribution (densification statistics column 3) or by minus their opacity
 * logit, ties in index order. The survivors keep their order, parameters and
 * optimiser state; the densification statistics start anew. On the GPU: the
 * keys, a stable radix sort, a scan and gathers; nothing goes through the host.
 * share in [0, 1]; *removed gets the count (may be null). */
int splat_trainer_remove_largest(splat_trainer *trainer, double share, uint64_t *removed);
int splat_trainer_remove_least_contributing(splat_trainer *trainer, double share, uint64_t *removed);
int splat_trainer_remove_least_opaque(splat_trainer *trainer, double share, uint64_t *removed);

/* The random generator densification draws from: a std::mt19937, whose
 * state carries over from call to call as the reference's session keeps one
 * (TrainSession::densifyRng_, train.hpp:254) and passes it to every round. */
typedef struct splat_rng splat_rng;
int splat_rng_create(uint32_t seed, splat_rng **out);
int splat_rng_destroy(splat_rng *rng);
/* std::uniform_int_distribution<std::size_t>(0, count - 1)(rng), as the
 * session draws the views it scores (train.cpp:690-692); count >= 1. */
int splat_rng_pick(splat_rng *rng, uint64_t count, uint64_t *out);

/* DensifyOptions (densify.hpp:23-50). */
typedef struct splat_densify_options {
  float gradient_threshold;  /* 2e-4 */
  float dense_scale;         /* 0: larger than this along any axis splits, otherwise clones */
  float prune_opacity;       /* 0.005 */
  int32_t prune_large;       /* 0: also remove the oversized, below */
  float max_screen_radius;   /* 20 */
  float max_world_scale;     /* 0 */
  uint64_t max_gaussians;    /* UINT64_MAX */
  float split_threshold;     /* 0; above 0 large Gaussians split on the absolute gradient (AbsGS) */
  int32_t scored_views;      /* 0; above 0 only Gaussians in high-error pixels densify (FastGS) */
  float min_marked_pixels;   /* 5 */
  double transparent_share;  /* 1: the share of the too transparent removed, the least useful first */
  uint64_t explore_splits;   /* 0: random large Gaussians split each round */
  uint64_t explore_seeds;    /* 0: new Gaussians placed at random in the cloud's bounding box */
  int32_t edge_split;        /* 0: 1 splits candidates along their longest axis with probability edge score / best */
} splat_densify_options;
void splat_densify_options_default(splat_densify_options *options);

/* DensifyResult's counts (densify.hpp:52-62); count is the new size. */
typedef struct splat_densify_result {
  uint64_t count, cloned, split, seeded, pruned, held_back;
} splat_densify_result;

/* Trainer::densify (trainer.cpp:710-715, densify_cloud of densify.cpp:115-326
 * and apply_changes): clones, splits, prunes and seeds by the densification
 * statistics, the new cloud being the survivors in their order, then per old
 * index a copy per clone and two children per split, then the seeds. The
 * survivors keep their optimiser state, the new ones start fresh, and the
 * statistics start anew. On the GPU: the decisions, stable radix sorts for
 * the transparent share and the count limit, scans and gathers; only the
 * rows that take random draws (split children, seeds) and the lists those
 * draws pick from are made on the host, drawing from rng in the reference's
 * order. source (may be null): if source_capacity >= result->count, the old
 * index whose state each new Gaussian keeps, or -1. A result with no
 * Gaussian is SPLAT_ERR_INVALID and leaves the trainer as it was (rng has
 * drawn, as in the reference). */
int splat_trainer_densify(splat_trainer *trainer, const splat_densify_options *options, splat_rng *rng,
                          splat_densify_result *result, int64_t *source, uint64_t source_capacity);

/* RelocateOptions (densify.hpp:87-91). */
typedef struct splat_relocate_options {
  float min_opacity;      /* 0.005: at or below, dead, to be relocated */
  double growth;          /* 0.05: share of the count added per round, within max_gaussians */
  uint64_t max_gaussians; /* UINT64_MAX */
} splat_relocate_options;
void splat_relocate_options_default(splat_relocate_options *options);

/* Trainer::relocate (trainer.cpp:717-722, relocate_cloud of densify.cpp:
 * 328-420, 3DGS-MCMC): the dead (opacity at or below min_opacity, or a value
 * not finite) move onto live Gaussians drawn in proportion to opacity, then
 * the count grows by growth the same way; a target that becomes N copies
 * takes opacity 1 - (1 - o)^(1/N) and its scale times o / D (gsplat's
 * divisor). Copies and targets start with fresh optimiser state; result
 * counts the relocated as cloned and the growth as seeded. The dead/alive
 * split and the gathers run on the GPU; the draws and the opacity and scale
 * updates, a sequential chain over std::discrete_distribution, on the host
 * from rng in the reference's order. With nothing alive the cloud stays and
 * only the statistics start anew. source as splat_trainer_densify. */
int splat_trainer_relocate(splat_trainer *trainer, const splat_relocate_options *options, splat_rng *rng,
                           splat_densify_result *result, int64_t *source, uint64_t source_capacity);

/* The training session (TrainSession, src/train/train.hpp:193-270 and
 * train.cpp:474-760, with the schedule of src/train/schedule.cpp): it owns a
 * trainer made from starting points (initial_cloud, train.cpp:194-212: sizes
 * from the 3 nearest neighbours, found on the GPU) and the training views,
 * kept in HBM at full, half and quarter size (half_size, train.cpp:232-255,
 * on the GPU), and runs the reference's schedule one iteration per
 * splat_session_step: the shuffled view order, coarse to fine (quarter size
 * until coarse_until[1] of the way, half until coarse_until[0]; from the
 * photos' spectra with adaptive_schedule), the position rate's decay and the
 * SH degree's ramp, densification rounds with scored views, the growth cap
 * and opacity resets (or 3DGS-MCMC relocation), and the pruning rounds.
 * Exposure, pose refinement, second order, SH dropout and the Mip filters
 * are not offered: they have no kernel here. */
typedef struct splat_session_options {
  int32_t iterations;         /* 15000 */
  int32_t sh_degree;          /* 2 */
  uint32_t seed;              /* 1: the view order draws from mt19937(seed), densification from mt19937(seed + 1) */
  int32_t report_every;       /* 500: the probe view's PSNR every this many iterations; 0 never */
  int32_t densify;            /* 1 */
  int32_t densify_mode;       /* 0: clone, split and prune (ADC); 1: relocation (3DGS-MCMC) */
  int32_t full_adam;          /* 0 */
  int32_t full_resolution;    /* 0: start at quarter, then half size */
  int32_t adaptive_schedule;  /* 0: 1 sets the sizes from the photos' spectra and grows the cap with them */
  float gradient_threshold;   /* 2e-4 */
  float split_threshold;      /* 1.2e-3 */
  double dense_fraction;      /* 0.001 of the extent: larger Gaussians split, smaller clone */
  int32_t densify_interval;   /* 100 */
  int32_t score_views;        /* 10 */
  float score_min_pixels;     /* 5 */
  int32_t explore;            /* 0 */
  int32_t significance_prune; /* 0 */
  int32_t edge_split;         /* 0 */
  double threshold_rise;      /* 1 */
  double prune_share;         /* 0 */
  double recovery_prune;      /* 0 */
  double max_growth;          /* -1: 4 per 7000 iterations */
  uint64_t max_gaussians;     /* 0: as the memory budget allows */
  double coarse_until[2];     /* 0.35, 0.15 */
  int32_t views_per_step;     /* 1: the reference's one view per iteration; 2..8: that many views of the
                                 order in one batched step (64-bit tile|depth keys), one Adam step for all */
} splat_session_options;
void splat_session_options_default(splat_session_options *options);

/* TrainData (train.hpp:153-173) as host arrays: the starting points (3
 * doubles and 3 colour bytes each), the training views (cameras and RGBA8
 * images at full size), the scene's extent and typical depth (the near
 * plane is 0.01 of it). */
typedef struct splat_session_data {
  const double *points;
  const uint8_t *colors;
  uint64_t point_count;
  const splat_camera *cameras;
  const uint8_t *const *images;
  int32_t views;
  double extent;
  double typical_depth;
} splat_session_data;

/* What the session has done: the last iteration, its level (0 half, 1
 * quarter, 2 full size) and view, the position rate it used, the Gaussian
 * count, the losses, the last report's probe PSNR and mean loss, the
 * densification rounds, and the coarse levels' ends. */
typedef struct splat_session_state {
  int32_t iteration;
  int32_t level;
  int32_t view;               /* the last view the step trained on */
  int32_t views_in_step;
  float position_rate;
  uint64_t gaussians;
  float first_loss, last_loss;
  int32_t report_iteration;
  double probe_psnr, mean_loss;
  int32_t densify_rounds;
  double densify_seconds;
  splat_densify_result last_densify;
  uint64_t held_back_total, pruned_total;
  double coarse_until[2];
} splat_session_state;

typedef struct splat_session splat_session;
/* trainer_options may be null (the defaults); the session sets selective_adam
 * from full_adam and the near plane from the typical depth. */
int splat_session_create(const splat_session_data *data, const splat_session_options *options,
                         const splat_trainer_options *trainer_options, splat_session **out);
int splat_session_destroy(splat_session *session);
/* TrainSession::step: SPLAT_ERR_STATE once every iteration has run. */
int splat_session_step(splat_session *session, splat_step_stats *stats);
int splat_session_get_state(splat_session *session, splat_session_state *out);
/* The session's trainer, borrowed (render, cloud, save); not to be destroyed. */
int splat_session_trainer(splat_session *session, splat_trainer **out);

/* The schedule's parts on their own. frequency_energy (schedule.cpp:41-75)
 * on the GPU: per factor, the spectrum magnitude of the image's brightness
 * within the frequencies an image smaller by that factor holds (up to 8
 * factors, images up to 4096 x 4096). resolution_switches
 * (schedule.cpp:77-82). GrowthBudget (schedule.hpp:26-41) after the given
 * observations: its limit at image_factor and progress, and its final count.
 * half_size (train.cpp:232-255) and initial_cloud (train.cpp:194-212) on
 * the GPU, host arrays in and out. */
int splat_frequency_energy(const uint8_t *rgba, int32_t width, int32_t height, const int32_t *factors, int32_t count, double *out);
int splat_resolution_switches(double full, double half, double quarter, double out[2]);
int splat_growth_limit(double initial_count, double factor, const uint64_t *observed, int32_t observations, double image_factor,
                       double progress, uint64_t *limit, double *final_count);
int splat_half_size(const uint8_t *rgba, int32_t width, int32_t height, uint8_t *out);
int splat_initial_cloud(const double *points, const uint8_t *colors, uint64_t count, int32_t sh_degree, float *positions, float *scales,
                        float *rotations, float *opacities, float *sh);

/* Trainer methods with no kernel in this library, for callers that set them
 * unconditionally: the neutral setting is accepted and changes nothing, any
 * other returns SPLAT_ERR_UNSUPPORTED. set_exposure (trainer.hpp:154): the
 * identity rows {1,0,0,0, 0,1,0,0, 0,0,1,0}; set_sh_dropout: probability 0;
 * set_filter3d: count 0; add_position_noise: scaler 0; enable_second_order and
 * update_curvature: never accepted. */
int splat_trainer_set_exposure(splat_trainer *trainer, const float exposure[12]);
int splat_trainer_set_sh_dropout(splat_trainer *trainer, float probability, int32_t retained_degree, uint32_t seed);
int splat_trainer_set_filter3d(splat_trainer *trainer, const float *filter, size_t count);
int splat_trainer_add_position_noise(splat_trainer *trainer, float scaler, uint32_t iteration);
int splat_trainer_enable_second_order(splat_trainer *trainer);
int splat_trainer_update_curvature(splat_trainer *trainer);

/* Trainer::gaussian_count, sh_degree, active_sh_degree, uses_fixed_point,
 * gpu_bytes, bytes_per_gaussian (trainer.hpp:138-193). */
int splat_trainer_info(splat_trainer *trainer, int64_t *gaussians, int32_t *sh_degree, int32_t *active_sh_degree,
                       int32_t *uses_fixed_point, uint64_t *gpu_bytes, uint64_t *bytes_per_gaussian);
/* Trainer::timings (trainer.hpp:186): average milliseconds per training
 * iteration by stage, in order. Fills up to `capacity` (name, ms) pairs; names
 * are static strings. *count gets the number of stages. */
int splat_trainer_timings(splat_trainer *trainer, const char **names, double *ms, int32_t capacity, int32_t *count);
/* What splat_trainer_autotune measured and chose. */
typedef struct splat_autotune_result {
  int32_t sort_form;    /* the splat_sort_form kept */
  int32_t digit_bits;   /* the radix digit width kept */
  int32_t forward_pixels_per_thread;  /* the compositing layout kept */
  int32_t backward_pixels_per_thread; /* the backward layout kept */
  double ms[2][3];         /* milliseconds per gradient pass, [sort form][digit bits - 6], starting layouts */
  double layout_ms[2][2];  /* milliseconds per gradient pass, [forward pixels - 1][backward pixels - 1], best sort */
  int32_t tile_size;       /* the rasterizer tile kept (16 unless both layouts take two pixels per thread) */
  int32_t batch_depth;     /* the batch depth kept */
  int32_t persistent_raster; /* the launch form kept */
  double tile_ms[2][2][2]; /* milliseconds per gradient pass, [tile 16/32][batch 128/256][persistent 0/1], best
                              layouts, the backward's sums as kept (0 where not timed) */
  int32_t grouped_backward; /* the backward's sums kept */
  double grouped_ms[2][2][2]; /* the same with grouped_backward 1 (0 where not timed) */
} splat_autotune_result;

/* The autotuner (new in this library; the reference has fixed 16x16 tiles and
 * 8-bit digits): times every tile-sort form and radix digit width on this view
 * with gradient passes (which change neither the parameters, the optimiser
 * state nor the densification statistics), `repeats` passes each, then the
 * rasterizer's pixel layouts, then, where both layouts take two pixels per
 * thread and the sums are float, its tile edge (16, 32), batch depth (128,
 * 256), launch form (one block per tile, persistent) and the backward's sums
 * (per splat, grouped), and keeps the fastest for the following steps. A
 * stage keeps the trainer's configured setting unless another is more than
 * 1 % faster, so that timing noise does not flip the form between runs. */
int splat_trainer_autotune(splat_trainer *trainer, const splat_camera *camera, const uint8_t *target, size_t target_bytes,
                           int32_t repeats, splat_autotune_result *result);
/* Turns per-stage CUDA-event timing on or off (off by default: it serialises). */
int splat_trainer_set_timing(splat_trainer *trainer, int32_t enabled);
/* Trainer::parameters (trainer.hpp:137): the device address of a parameter
 * group (0 positions, 1 scales, 2 rotations, 3 opacities, 4 SH DC planes,
 * 5 SH rest rows), valid until the Gaussians change in number. The DC is
 * stored in 3 FP32 planes, one per channel, each the Gaussian count rounded
 * up to a multiple of 128 elements long; the higher coefficients in one row
 * per Gaussian (coefficient-major, channel-minor, in the sh_storage type),
 * padded to a multiple of 16 bytes, as many rows as a plane is long. */
int splat_trainer_device_parameters(splat_trainer *trainer, int32_t group, uint64_t *device_address, uint64_t *bytes);

/* Debug access to the device buffers of the last step, for parity tests:
 * which: 0 splats (12 floats per Gaussian), 1 reach (1 float), 2 depth keys
 * (u32, in Gaussian order), 3 entry tile keys (u32 or u64 by sort form, sorted),
 * 4 entry values (u32, sorted), 5 tile ranges (2 u32 per tile), 6 image
 * (4 floats per pixel), 7 stops (u32 per pixel), 8 adjoint (4 floats per
 * pixel), 9 raw sums (16 words per Gaussian: int32 fixed point or float),
 * 10 counters (visible, total entries, used entries, 0), 11 loss partials
 * (2 floats per tile), 12 error word, 13 blended splats per pixel (u32; with
 * blend_lists only, else empty), 14-18 the Adam state of parameter groups 0-4
 * (positions, scales, rotations, opacities, SH; u32 words: BF16 pairs, or FP32
 * m values then v values; SH state in rows of 3 (degree + 1)^2 words per
 * Gaussian rounded up to a multiple of 4, the row count rounded up to 128), 19 the two-pixel backward's
 * tile schedule (u32 per tile: the entries each tile's backward walks, as the two-pixel compositing
 * recorded them, then the order the backward took the tiles in). Copies min(bytes, size) bytes; *size
 * gets the buffer's size in bytes. */
int splat_trainer_debug_download(splat_trainer *trainer, int32_t which, void *out, size_t bytes, size_t *size);

/* 3DGS .ply files (src/splat/gaussian_cloud.hpp:60-67, load_ply and
 * save_ply), host memory only. splat_cloud_load_ply reads a binary
 * little-endian or ASCII file (properties a cloud has no use for, such as
 * normals, are skipped; the SH degree follows from the number of f_rest_*
 * properties: 0, 9, 24 or 45). With every array null it reads only the header
 * and sets *count and *sh_degree; then call it again with arrays of 3, 3, 4, 1
 * and 3 (degree + 1)^2 floats per Gaussian. A file that cannot be read or is
 * not a splat file returns SPLAT_ERR_INVALID with the reason, as the
 * reference's std::runtime_error. splat_cloud_save_ply writes the standard
 * binary little-endian layout (x y z, zero normals, f_dc, f_rest channel-major,
 * opacity, scales, rotations). */
int splat_cloud_load_ply(const char *path, int32_t *count, int32_t *sh_degree, float *positions, float *scales,
                         float *rotations, float *opacities, float *sh);
int splat_cloud_save_ply(const char *path, const splat_cloud *cloud);

/* CGC files (src/splat/cgc.hpp:15-50, save_cgc and load_cgc): the lossy
 * layered format for viewing over the network. A file holds three importance
 * layers (opacity times cross-section percentiles), each with its own
 * precision: positions on a symlog grid around the scene's median, stored as
 * gaps along a Morton curve; canonical axes; YCoCg colour; opacity; the higher
 * SH bands as labels into a per-layer k-means codebook; every byte column its
 * own LZMA stream. splat_cloud_save_cgc needs a CUDA device (the per-splat
 * work, the order statistics, the Morton sort and the codebook run on it) and
 * writes nothing when it fails; a cloud with a NaN or infinite value is refused
 * with SPLAT_ERR_INVALID, as the reference throws. splat_cloud_load_cgc reads
 * versions 1 and 2 on the host, with splat_cloud_load_ply's two-call protocol;
 * splats come back layer by layer, each layer in Morton order, with their axes
 * possibly permuted and flipped (the same ellipsoids). */
enum { SPLAT_CGC_BALANCED = 0, SPLAT_CGC_SMALL = 1 };
typedef struct splat_cgc_options {
  int32_t preset; /* SPLAT_CGC_BALANCED (about 28x smaller than .ply) or SPLAT_CGC_SMALL (about 31x) */
  int32_t fast;   /* much quicker and a little larger (training checkpoints) */
} splat_cgc_options;
typedef struct splat_cgc_stats {
  uint64_t bytes;           /* size of the written file */
  uint64_t layer_counts[3]; /* splats per layer, most important first */
} splat_cgc_stats;
/* options may be null (balanced, not fast); stats may be null. */
int splat_cloud_save_cgc(const char *path, const splat_cloud *cloud, const splat_cgc_options *options, splat_cgc_stats *stats);
int splat_cloud_load_cgc(const char *path, int32_t *count, int32_t *sh_degree, float *positions, float *scales,
                         float *rotations, float *opacities, float *sh);
/* The CGC pieces the reference exposes for its unit tests
 * (cgc_detail::morton_code, canonicalize_axes, src/splat/cgc.hpp:50-58): the
 * low 21 bits of x, y, z interleaved (x into bit 0); log scales sorted
 * descending with the quaternion (w, x, y, z) rewritten so that w is its
 * largest component and not negative (a zero quaternion is the identity). */
uint64_t splat_cgc_morton_code(uint32_t x, uint32_t y, uint32_t z);
int splat_cgc_canonicalize_axes(float *log_scales, float *wxyz);
/* The reference's LZMA helpers (src/splat/lzma.hpp:10-17): an "alone" (.lzma)
 * stream from preset `level` (0-9, extreme flag) with lc, lp, pb; *written
 * gets its size, and min(capacity, size) bytes are copied when out is not
 * null. splat_lzma_decompress fails (SPLAT_ERR_INVALID) on corrupt or
 * truncated data and on any size but `expected`. liblzma.so.5 is loaded at
 * the first call. */
int splat_lzma_compress(const uint8_t *data, size_t size, int32_t level, int32_t extreme, int32_t lc, int32_t lp, int32_t pb,
                        uint8_t *out, size_t capacity, size_t *written);
int splat_lzma_decompress(const uint8_t *stream, size_t size, uint8_t *out, size_t expected);

/* Stage-level entry points on device memory, for the reference's operator
 * tests (tests/test_radix_sort.cpp) and for callers with their own buffers. */

/* RadixSorter::record (src/core/radix_sort.hpp, radix_sort.cpp:70-97): stable
 * ascending sort of count (u32 key, u32 value) pairs over the low key_bits
 * bits. keys, values, tmp_keys, tmp_values are device pointers of count
 * elements, each 16-byte aligned (cudaMalloc's are; others are refused with
 * SPLAT_ERR_INVALID); the result is in keys/values. Allocates its scratch.
 * stream may be 0. */
int splat_radix_sort_u32(uint32_t *keys, uint32_t *values, uint32_t *tmp_keys, uint32_t *tmp_values, uint32_t count,
                         int32_t key_bits, int32_t digit_bits, void *stream);
/* The same for 64-bit keys over key_bits bits (the (tile << 32 | depth) keys). */
int splat_radix_sort_u64(uint64_t *keys, uint32_t *values, uint64_t *tmp_keys, uint32_t *tmp_values, uint32_t count,
                         int32_t key_bits, int32_t digit_bits, void *stream);

/* splat_radix_sort_u32 for callers that cannot allocate device memory: an
 * application that owns a fixed device-memory budget and may not let a helper
 * take more, or a latency-critical loop in which cudaMalloc/cudaFree would
 * synchronise the device. This entry point has no counterpart in the
 * reference. It allocates nothing: its scratch is one file-scope __device__
 * array of about 4 MiB that every GPU loading this library holds until the
 * process exits. Limit: count <= 4194304 keys (key_bits 1..32, digit_bits
 * 6..8); larger counts return SPLAT_ERR_INVALID with a message saying so.
 * Every call looks up the array's device address with the caller's device
 * current. Every call shares the one array (it clears what must start at
 * zero), so calls that overlap on the GPU, from any stream or thread, race and
 * must be ordered by the caller. Device pointers and the result as for
 * splat_radix_sort_u32. The call reads its error word back and synchronises
 * its stream before it returns, so it cannot be used inside stream capture. */
int splat_radix_sort_u32_noalloc(uint32_t *keys, uint32_t *values, uint32_t *tmp_keys, uint32_t *tmp_values,
                                 uint32_t count, int32_t key_bits, int32_t digit_bits, void *stream);

/* Throughput the SM pipes reach on the current GPU, measured by
 * microbenchmarks that keep one pipe busy on every SM (a few milliseconds in
 * all): FP32 fused multiply-adds in FLOP/s (two per FMA), the SFU's ex2 in
 * results/s, conflict-free 16-byte shared-memory loads in bytes/s, and the
 * warp instructions the FMA benchmark issues per second. These, not HBM, bound
 * the compositing and backward kernels; the bench reports their issue rates
 * against them. This entry point has no counterpart in the reference. */
typedef struct splat_sm_peaks {
  double fp32_flops;
  double sfu_ops;
  double shared_bytes;
  double warp_instructions;
} splat_sm_peaks;
int splat_measure_sm_peaks(splat_sm_peaks *out);

/* Sets how many times a radix sort pass polls a predecessor's look-back word
 * before it gives up (the default, 2^20, when polls is negative). A pass that
 * gives up sets the look-back timeout bit: the call returns SPLAT_ERR_DEVICE
 * and its output is not sorted, but no write leaves the arrays. For the tests
 * of that failure path; applies to sorts launched after the call (a captured
 * step keeps the limit it was captured with). This entry point has no
 * counterpart in the reference. */
int splat_debug_set_wait_limit(int32_t polls);

/* Evaluates the deterministic exp and log of splat_detmath.h on the device, for
 * the check that they agree bit for bit with the host. Device pointers. */
int splat_debug_detmath(const float *in, float *out_exp, float *out_log, uint32_t count);

#ifdef __cplusplus
}
#endif

#endif /* SPLAT_B200_H */
