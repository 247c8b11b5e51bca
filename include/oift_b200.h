/*
 * oift_b200.h -- C ABI of the B200 (sm_100a) OIFT + relaxation library.
 *
 * Drop-in boundary for the GPU path of jung0221/roift:
 *   oift_fmax_gpu_run  replaces  gpu/oift_fmax_gpu.cu:139-149 (same signature and
 *                      meaning; it additionally returns a negative status on error
 *                      instead of running on unchecked allocations);
 *   oift_gpu_run       replaces  gpu/oift_gpu.cu:149-158 (cost_mode 0 = f_max; the
 *                      additive mode is not provided and returns OIFT_E_UNSUPPORTED).
 * The extended entry points add what the CPU calls gft::ift::OIFT_Multi /
 * OIFT_Multi_PerClass (gft/include/gft_ift.h:108-122) and ORelax_1_Multi /
 * ORelax_1_Multi_PerClass (gft/include/gft_ift.h:451-465) compute, on one GPU:
 * arc-weight building, oriented f_max OIFT with exported cost, relaxation sweeps,
 * argmax labels and a mask.
 *
 * Conventions (the reference's, gft/include/gft_scene32.h:20-179):
 *   voxel address p = x + y*xsize + z*xsize*ysize; 2D images are zsize == 1;
 *   labels: NIL = -1 (unlabelled), 0 = background, >= 1 objects (< 32768);
 *   polarity values are x100 (pol in [-1,1] -> per in [-100,100]).
 * All pointers are plain host or device pointers; sizes are element counts; no
 * function keeps a pointer after it returns.  Every function returns OIFT_OK (0) or
 * a negative oift_status, except the two reference-compatible entry points which
 * return the number of levels processed (>= 0) or -1.
 */
#ifndef OIFT_B200_H
#define OIFT_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define OIFT_API __attribute__((visibility("default")))
#else
#define OIFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    OIFT_OK = 0,
    OIFT_E_BAD_ARG = -1,        /* null pointer, bad size, bad adjacency, |per| > 100 ... */
    OIFT_E_NO_SEEDS = -2,       /* empty seed list */
    OIFT_E_OOM = -3,            /* device allocation failed */
    OIFT_E_NOT_CONVERGED = -4,  /* a bounded wait inside a kernel ran out */
    OIFT_E_QUEUE_OVERFLOW = -5, /* device work queue capacity exceeded */
    OIFT_E_CUDA = -6,           /* other CUDA runtime error */
    OIFT_E_RANGE = -7,          /* weight or intensity outside the supported range */
    OIFT_E_UNSUPPORTED = -8,    /* option not provided (e.g. additive path cost) */
    OIFT_E_SEED_RANGE = -9      /* a seed address is outside the volume */
} oift_status;

/* Arc-weight builders (row a1-a3): base weight of the undirected edge {p,q}. */
typedef enum {
    OIFT_W_GRAD = 0,    /* |I_p - I_q| exactly: up to 16383 on 32-bit keys, up to 2^30 - 1 on
                           64-bit keys (single-volume entries), else OIFT_E_RANGE */
    OIFT_W_GRAD_Q = 1,  /* min(|I_p - I_q|, wq); clamp events counted */
    OIFT_W_RBF_Q = 2,   /* floor(wq*(1 - exp(-d^2/(2 sigma^2))) + 0.5), host LUT */
    OIFT_W_BLEND_Q = 3, /* float a|dI| + (1-a)(g_p+g_q)/2, g = Sobel map scaled to max I
                           (experiments/exp_gradient_weight.cpp:244-254, 596-608); 6 / 4
                           adjacency, global polarity, image in 0..65535 */
    OIFT_W_IMAGEGRAPH = 4  /* 2D image graph (gft_imagegraph.cpp:13-47, 981-1016): |dI| + 1
                              oriented as MAX(ROUND(w (1 +/- per/100)), 1) with per/100 held
                              in a float; relaxation = ORelax_1(sImageGraph) (gft_ift.cpp:
                              7683-7847): one membership channel from label / max label,
                              binary labels.  zsize == 1, adjacency 4 or 8, global polarity */
} oift_weight_mode;

typedef struct oift_b200_ctx oift_b200_ctx;

/* Parameters of one OIFT + relaxation job. */
typedef struct {
    int xsize, ysize, zsize;
    int adjacency;        /* 4 or 8 (zsize == 1), 6 or 26 */
    int weight_mode;      /* oift_weight_mode */
    int wq;               /* quantisation ceiling for the _Q modes (e.g. 4095) */
    float rbf_sigma;      /* OIFT_W_RBF_Q */
    float blend_a;        /* OIFT_W_BLEND_Q */
    float per;            /* global polarity x100 (label 0 uses -per), if per_class NULL */
    const float *per_class; /* host array [max_label+1] of per-label polarity x100, or NULL */
    int max_label;
    int relax_sweeps;     /* K >= 0 */
} oift_b200_params;

/* Device-resident results of the extended entry points (device pointers, may be NULL). */
typedef struct {
    int32_t *cost;        /* [N] f_max cost (INT32_MAX if unreached) */
    int32_t *oift_label;  /* [N] OIFT label before relaxation */
    int32_t *label;       /* [N] final label (argmax of the relaxed membership) */
    uint8_t *mask;        /* [N] 1 where the final label != 0 */
    float *membership;    /* [nclasses][N] relaxed membership (planar) */
} oift_b200_outputs;

/* Per-run statistics. */
typedef struct {
    int levels;           /* (cost,label) levels processed by the OIFT */
    long long tile_steps; /* tile activations */
    long long clamped;    /* edges clamped by a _Q builder */
    int nclasses;         /* relaxation classes */
    float ms_weights, ms_oift, ms_relax, ms_total; /* CUDA-event stage times */
    int kernels;          /* kernel launches issued by the call */
    float ms_oift_kernel; /* persistent OIFT kernel alone (CUDA events around the launch) */
    float ms_sweeps;      /* the K relaxation sweep launches alone */
    long long oift_cycles[24]; /* OIFT SM cycles summed over warps: level switch, owner
                                  phase, queued tiles, drain; key staging, sparse tiles,
                                  dense tiles; counts of stale, sparse, dense tiles; dense
                                  tiles: masks, flood, flood iterations, expansion, faces,
                                  pending; sparse tiles: worklist, flood rounds, face
                                  pushes, publication, pending, counts of rounds, voxels,
                                  publications */
    long long relax_active_voxel_sweeps; /* voxels computed over all sweeps (tiles outside
                                            the reference's growing mask are skipped) */
} oift_b200_stats;

/* Context: owns the device scratch for one device and one stream. */
OIFT_API int oift_b200_create(oift_b200_ctx **out, int device);
OIFT_API int oift_b200_destroy(oift_b200_ctx *ctx);
/* Number of bytes of device scratch currently held. */
OIFT_API size_t oift_b200_scratch_bytes(const oift_b200_ctx *ctx);
/* Stream used by subsequent calls (cudaStream_t as void*; NULL = legacy default). */
OIFT_API int oift_b200_set_stream(oift_b200_ctx *ctx, void *stream);
OIFT_API const char *oift_b200_status_string(int status);

/* Full pipeline on DEVICE pointers: image int16 [N]; seeds int32 [nseeds] addresses;
 * seed_labels int32 [nseeds].  Outputs as requested in `out`.  Runs on the context's
 * stream; synchronises before returning. */
OIFT_API int oift_b200_run_device_i16(oift_b200_ctx *ctx, const oift_b200_params *prm,
                             const int16_t *image, const int32_t *seeds,
                             const int32_t *seed_labels, int nseeds,
                             const oift_b200_outputs *out, oift_b200_stats *stats);

/* Full pipeline on HOST pointers (int32 image as in the reference, already shifted
 * and blurred by the caller).  label: in = NIL except seeds, out = final labels.
 * cost (may be NULL) receives the f_max cost, membership (may be NULL) the relaxed
 * membership [nclasses][N], mask (may be NULL) the uint8 mask. */
OIFT_API int oift_b200_run_host(oift_b200_ctx *ctx, const oift_b200_params *prm,
                       const int32_t *image, int32_t *label, const int32_t *seeds, int nseeds,
                       int32_t *cost, float *membership, int membership_cap_classes,
                       uint8_t *mask, oift_b200_stats *stats);

/* The relaxation alone on HOST pointers, as gft::ift::ORelax_1_Multi /
 * ORelax_1_Multi_PerClass (gft/include/gft_ift.h:451-465, gft/src/gft_ift.cpp:8655-9187)
 * relaxes the labels it is given: label in = the labels to relax (e.g. the OIFT's), out =
 * the relaxed labels; classes = 0 and the labels found at the seeds; prm->relax_sweeps
 * sweeps of the prm->adjacency neighbourhood with prm->per / per_class.  membership
 * ([nclasses][N], may be NULL, at most membership_cap_classes planes) and mask (may be
 * NULL) as in oift_b200_run_host. */
OIFT_API int oift_b200_relax_host(oift_b200_ctx *ctx, const oift_b200_params *prm,
                                  const int32_t *image, int32_t *label, const int32_t *seeds,
                                  int nseeds, float *membership, int membership_cap_classes,
                                  uint8_t *mask);

/* One job of the batched driver: a volume and one seed set (device pointers). */
typedef struct {
    const int16_t *image;
    int xsize, ysize, zsize;
    const int32_t *seeds, *seed_labels;
    int nseeds;
    float per;          /* polarity x100 of this job (global mode) */
    int32_t *cost;      /* device outputs, each may be NULL */
    int32_t *label;     /* final (relaxed) labels */
    uint8_t *mask;
    int status;         /* out: oift_status of this job */
} oift_b200_job;

typedef struct {
    int teams;          /* OIFT teams of the timed part */
    int jobs;
    int tuning;         /* 1 when this call measured a team count for the autotuner */
    float ms_wall;      /* host wall time of the jobs after tuning */
    float ms_oift;      /* device time of weights + batched OIFT */
    float ms_relax;     /* host wall time of the relaxation phase */
    int tile_ty;        /* 3D warp tile of the OIFT teams: 8 = 32x8x4, 4 = 32x4x8 */
} oift_b200_batch_stats;

/* Batched driver for many volumes of uneven sizes with several seed sets per volume.  Runs
 * the pipeline of `common` (adjacency 6 or 4, weights, sweeps; the job gives extents and
 * polarity) for every job.  Edge codes are built once per distinct image; the OIFT of all
 * jobs runs in one persistent launch over all SMs split into `teams` teams, each team
 * taking the next job (largest first) from a device counter; relaxation then runs on
 * several streams.  teams = 0 selects the context's autotuner: its first calls try
 * sms/2, sms/4, sms and sms/8 teams, one per call, and later calls use the fastest.  Writes
 * each job's status; returns the first failing one, OIFT_OK otherwise. */
OIFT_API int oift_b200_run_batch(oift_b200_ctx *ctx, const oift_b200_params *common,
                                 oift_b200_job *jobs, int njobs, int teams,
                                 oift_b200_batch_stats *stats);
/* The same batch recorded once into a CUDA graph and replayed.  Creation plans the batch
 * on the host (job checks, intensity ranges, each job's class set; statuses of failing jobs
 * are written and the first one returned), then captures the weight builds, the team
 * launches and every job's relaxation sweeps from a private context.  A replay is one graph
 * launch followed by a read of the job statuses; it stays valid while the jobs' buffers
 * keep their addresses, the images their intensity range and the seeds their label set.
 * teams = 0 takes the context's autotuned team count (sms/2 before it has one).  `ms`
 * (may be NULL) receives the device time of the replay. */
typedef struct oift_b200_batch_graph oift_b200_batch_graph;
OIFT_API int oift_b200_batch_graph_create(oift_b200_ctx *ctx, const oift_b200_params *common,
                                          oift_b200_job *jobs, int njobs, int teams,
                                          oift_b200_batch_graph **graph);
OIFT_API int oift_b200_batch_graph_launch(oift_b200_batch_graph *graph, oift_b200_job *jobs,
                                          float *ms);
OIFT_API int oift_b200_batch_graph_destroy(oift_b200_batch_graph *graph);
/* 3D warp tile of the batched OIFT for explicit team counts (teams > 0): 8 = 32x8x4 (the
 * default) or 4 = 32x4x8.  With teams = 0 the autotuner chooses the tile with the team count. */
OIFT_API int oift_b200_set_batch_tile(oift_b200_ctx *ctx, int tile_ty);
/* CTAs of the persistent OIFT grid of this context (0 = one per SM, the default). */
OIFT_API int oift_b200_set_oift_grid(oift_b200_ctx *ctx, int ctas);
/* Bounds of the OIFT kernels' device-side waits for later calls of this context:
 * spin_limit = polls (~64 ns each) of one wait (grid or team barrier, end of a level)
 * before it gives up, max_levels = (cost, label) levels before the run counts as runaway.
 * Reaching either ends the launch cleanly (every warp leaves, the context stays usable)
 * and the call returns OIFT_E_NOT_CONVERGED; in the batched driver the team that hit it
 * reports OIFT_E_NOT_CONVERGED for its job, stops, and no team takes a further job.
 * Values <= 0 restore the defaults (2e7 polls, 4e6 levels).  The same guard as the
 * reference's iteration cap (gpu/oift_fmax_gpu.cu:197,240-242), exposed for testing. */
OIFT_API int oift_b200_set_limits(oift_b200_ctx *ctx, long long spin_limit, int max_levels);

/* Steps around the path in the reference CLI (oiftrelax.cpp main). */
/* `passes` Gaussian blurs (Scene32::GaussianBlur, gft_filtering3.cpp:385-397) of a device
 * int32 volume; in == out allowed. */
OIFT_API int oift_b200_gaussian_blur_i32(oift_b200_ctx *ctx, const int32_t *in, int32_t *out,
                                         int xsize, int ysize, int zsize, int passes);
/* Conditional dilation (oiftrelax.cpp:87-169) of a device label map: label-0 voxels within
 * Spheric(radius) of a label-1 voxel whose `image` value ranks within the percentile become
 * 1.  *added (may be NULL) receives the count. */
OIFT_API int oift_b200_conditional_dilation(oift_b200_ctx *ctx, const int32_t *image,
                                            int32_t *label, int xsize, int ysize, int zsize,
                                            float radius, float percentile, long long *added);
/* Boundary seeds (oiftrelax.cpp:175-224) on host arrays: face voxels on the stride grid
 * whose label is NIL (-1) become background (0) and are appended to seeds_out.  Returns the
 * number of seeds (with seeds_out == NULL: counts only, changes nothing), OIFT_E_RANGE if
 * cap is too small. */
OIFT_API int oift_b200_inject_boundary_seeds(int32_t *label, int xsize, int ysize, int zsize,
                                             int stride, int32_t *seeds_out, int cap);
/* The CLI's text inputs (host-only).  Seeds file (oiftrelax.cpp:322-352): a count, then
 * "x y z id label" per seed; negative labels become 0, seeds outside the volume are
 * dropped, label[p] takes the seed's label.  Returns the number of in-volume seeds written
 * to seeds_out (with seeds_out == NULL: counted only, nothing changed), OIFT_E_RANGE when
 * cap is too small, OIFT_E_BAD_ARG when the file cannot be read. */
OIFT_API int oift_b200_read_seeds(const char *path, int xsize, int ysize, int zsize,
                                  int32_t *label, int32_t *seeds_out, int cap);
/* Per-class polarity file (oiftrelax.cpp:280-300): a count n, then n values in [-1, 1],
 * stored x100 in per_class (may be NULL to count).  Returns n. */
OIFT_API int oift_b200_read_polarity(const char *path, float *per_class, int cap);

/* Volume files of the CLI (gft::Scene32::Read / Write, gft/src/gft_scene32.cpp:334-420,
 * 525-580, 600-660, 748-800), host only.  Formats by extension: .scn (8/16/32-bit samples);
 * NIfTI-1 .nii, .nii.gz, .hdr/.img pairs (either byte order).  Reading widens uint8, int8,
 * int16, uint16 and int32 samples and scales float32 by 10000 / max with rounding, as
 * ReadNifti1 does; other sample types and dim[0] outside 3..4 give OIFT_E_UNSUPPORTED.
 * dims = (xsize, ysize, zsize), spacing = (dx, dy, dz).  With data == NULL only dims and
 * spacing are filled; a cap below the voxel count gives OIFT_E_RANGE.  Writing follows
 * Scene32::Write: .scn with the narrowest of 8/16/32 bits that holds the maximum, NIfTI as
 * int32 samples.  OIFT_E_BAD_ARG when a file cannot be opened, read or written. */
OIFT_API int oift_b200_read_volume(const char *path, int32_t *data, size_t cap_voxels,
                                   int dims[3], float spacing[3]);
OIFT_API int oift_b200_write_volume(const char *path, const int32_t *data, const int dims[3],
                                    const float spacing[3]);
/* The CLI's processing chain on host buffers: shift the unshifted int32 `image` to >= 0,
 * `blur_passes` Gaussian blurs (the CLI uses 2), OIFT + relax_sweeps sweeps as run_host,
 * then, if percentile >= 0 and the result is binary, the conditional dilation with
 * Spheric(1).  `label` holds the seed labels on entry and the result on return. */
OIFT_API int oift_b200_run_cli_host(oift_b200_ctx *ctx, const oift_b200_params *prm,
                                    const int32_t *image, int32_t *label, const int32_t *seeds,
                                    int nseeds, int blur_passes, float percentile,
                                    oift_b200_stats *stats);

/* Two-level coarse-to-fine cascade (experiments/exp_coarse_to_fine.cpp:327-414): shift,
 * `blur_passes` blurs, Subsampling to odd half extents, seeds at (x/2, y/2, z/2) (first
 * seed wins), coarse OIFT + relaxation, nearest ScaleLabel, labels that touch another value
 * become NIL, the caller's labels kept, every labelled voxel a seed of the fine OIFT +
 * relaxation, conditional dilation (percentile >= 0) of a binary result.  Host flavour:
 * `label` holds the seed labels on entry (NIL = -1 elsewhere) and the result on return. */
OIFT_API int oift_b200_run_pyramid_host(oift_b200_ctx *ctx, const oift_b200_params *prm,
                                        const int32_t *image, int32_t *label,
                                        const int32_t *seeds, int nseeds, int blur_passes,
                                        float percentile, oift_b200_stats *stats);
/* Device flavour: int16 image, label_in (seed labels, NIL elsewhere), seeds and label_out
 * are device arrays. */
OIFT_API int oift_b200_run_pyramid_device_i16(oift_b200_ctx *ctx, const oift_b200_params *prm,
                                              const int16_t *image, const int32_t *label_in,
                                              const int32_t *seeds, int nseeds, int blur_passes,
                                              float percentile, int32_t *label_out,
                                              oift_b200_stats *stats);

/* Gradient of a soft-Dice loss through K relaxation sweeps (config-5 style training).
 * Forward model per updated voxel p and neighbour q:
 *   d = beta |I_p - I_q| + (1 - beta)(g_p + g_q)/2,  w = d (1 + sign(I_p - I_q) alpha (2 m_bg(q) - 1)),
 *   W = exp(-w^2/sigma^2)/Dpq (OIFT_ADJ_RBF) or max(0, max(I)(1 + |alpha|) - w)^8/Dpq (OIFT_ADJ_POW8),
 *   m'(p) = sum W m(q) / sum W on the mask that grows one ring per sweep from the boundary of
 *   the OIFT labels; seeds stay one-hot.  Loss 1 - (2 sum p t + eps)/(sum p + sum t + eps)
 *   with p = 1 - m_bg.  The OIFT labels are held fixed; states are checkpointed every
 *   `checkpoint` sweeps (0 = ceil(sqrt(K))) and recomputed on the way back. */
typedef enum { OIFT_ADJ_RBF = 0, OIFT_ADJ_POW8 = 1 } oift_adjoint_kernel;

typedef struct {
    int xsize, ysize, zsize;
    int adjacency;        /* 4, 6, 8 or 26 */
    int sweeps;           /* K >= 1 */
    int checkpoint;       /* 0 = ceil(sqrt(K)) */
    int kernel;           /* oift_adjoint_kernel */
    float sigma, alpha, beta, eps;
} oift_b200_adjoint_params;

/* Device inputs: int16 image (shifted to >= 0 for POW8), optional float gradient map,
 * OIFT labels, seeds with their labels, uint8 truth; membership_out [classes][N] may be
 * NULL.  loss receives L; grad (may be NULL: forward only) receives dL/d(sigma, alpha, beta). */
OIFT_API int oift_b200_adjoint(oift_b200_ctx *ctx, const oift_b200_adjoint_params *ap,
                               const int16_t *image, const float *grad_map,
                               const int32_t *labels0, const int32_t *seeds,
                               const int32_t *seed_labels, int nseeds, const uint8_t *truth,
                               float *membership_out, double *loss, double *grad);

/* Arc-weight-map part of the adjoint, on the forest of an integer OIFT result held fixed.
 * oift_b200_bottleneck_arcs reads the forest from that result (DEVICE int16 image, cost
 * and label maps [N] as the OIFT returned them for `prm`, GRAD or GRAD_Q weights, global
 * polarity, and its seeds) and writes, per voxel, the arc that carries its f_max cost:
 * arcs[p] = tail * 32 + d (the arc tail -> tail + offset d of the gft Spheric order,
 * gft/src/gft_adjrel3.cpp:47-85), -2 at seeds, -3 at unreached voxels.  In each (cost, label)
 * level the entry voxels take the arc of weight exactly `cost` from a voxel of their label
 * conquered earlier; the others inherit, round by round, from a same-level neighbour that
 * reaches them through an open arc (gft/src/gft_ift.cpp:965-981 with f_max).  Call it once
 * per OIFT result.  oift_b200_cost_adjoint evaluates, for the weight parameters of `ap`
 * (sigma, alpha, beta, eps), the continuous RBF cost of every voxel's bottleneck arc
 * w = 1 - exp(-c^2 / (2 sigma^2)), c = (beta |dI| + (1 - beta)(g_t + g_h) / 2) (1 + s alpha_l)
 * with alpha_l = -alpha for a background tail, the object confidence u = 1 - w/2 (object
 * label) or w/2 (background, 0 / 1 at seeds), the soft-Dice loss of u against `truth`, and
 * (grad may be NULL) its gradient with respect to (sigma, alpha, beta): the f_max
 * bottleneck-arc subgradient through the fixed forest.  grad_map may be NULL (g = 0). */
OIFT_API int oift_b200_bottleneck_arcs(oift_b200_ctx *ctx, const oift_b200_params *prm,
                                       const int16_t *image, const int32_t *cost,
                                       const int32_t *label, const int32_t *seeds, int nseeds,
                                       int64_t *arcs);
OIFT_API int oift_b200_cost_adjoint(oift_b200_ctx *ctx, const oift_b200_adjoint_params *ap,
                                    const int16_t *image, const float *grad_map,
                                    const int32_t *label, const int64_t *arcs,
                                    const uint8_t *truth, double *loss, double *grad);

/* Stage entry points on device pointers (used by the batched driver and tests). */
OIFT_API int oift_b200_build_weights_i16(oift_b200_ctx *ctx, const oift_b200_params *prm,
                                const int16_t *image, uint16_t *weights /* [planes][N] */,
                                long long *clamped);
OIFT_API int oift_b200_weight_planes(int adjacency);
/* Per-level profile of the last OIFT run: pairs (SM cycles, tile activations) for the
 * first `cap` levels.  Returns the number of pairs written or a negative status. */
OIFT_API int oift_b200_level_profile(oift_b200_ctx *ctx, unsigned int *cycles_steps, int cap);

/* Device self-test of the FP32 division by 100 used inside the relaxation sweeps:
 * counts, over all 2^32 FP32 bit patterns (NaN/Inf skipped, signed zeros equal), the
 * inputs whose quotient differs from the IEEE division; first_bad = smallest such
 * pattern (0xFFFFFFFF if none).  Uses device 0 of the calling thread's context. */
OIFT_API int oift_b200_selftest_div100(unsigned long long *mismatches, unsigned int *first_bad);

/* OIFT without device allocation (no counterpart in the reference): for callers that
 * cannot let a library call cudaMalloc while they run -- an application whose own memory
 * pool already holds the GPU's memory, a pipeline that must not allocate (and so
 * synchronise the device) after start-up, a host that forbids plug-ins to allocate.
 * Builds the 6-/4-adjacency arc weights (OIFT_W_GRAD or OIFT_W_GRAD_Q) from the int16
 * DEVICE image and runs the f_max OIFT, with every intermediate buffer inside one static
 * device array of oift_b200_noalloc_scratch_bytes() bytes (about 10.3 MB, held by each GPU
 * that loads the library until the process exits).  Inputs and outputs are device
 * pointers owned by the caller: seeds / seed_labels [nseeds], cost and/or label [N]
 * (either may be NULL).  per / per_class / max_label as in oift_b200_params.
 * Limits: at most OIFT_NOALLOC_MAX_VOXELS voxels and 65536 warp tiles; larger volumes
 * return OIFT_E_RANGE before any device work.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) -- make it before any stream capture.  The
 * address is kept for the process: do not call this entry on a device after a
 * cudaDeviceReset of it (the reset reloads the library's device code elsewhere).
 * All calls share the array: calls that overlap on the GPU race and corrupt each other.
 * Runs on `stream` (cudaStream_t as void*) and synchronises it before returning. */
#define OIFT_NOALLOC_MAX_VOXELS (1u << 20)
OIFT_API int oift_b200_oift_noalloc(const int16_t *image, int xsize, int ysize, int zsize,
                                    int adjacency, int weight_mode, int wq, float per,
                                    const float *per_class, int max_label,
                                    const int32_t *seeds, const int32_t *seed_labels,
                                    int nseeds, int32_t *cost, int32_t *label, void *stream);
OIFT_API size_t oift_b200_noalloc_scratch_bytes(void);

/* Reference-compatible drop-in (gpu/oift_fmax_gpu.cu:139-149).  Host pointers.
 * h_labels: in = labels (seed voxels carry their label, NIL elsewhere), out = OIFT
 * labels.  h_per_class [max_label+1] polarity x100.  Returns the number of levels
 * processed, or -1 on error (oift_b200_last_status() gives the reason). */
OIFT_API int oift_fmax_gpu_run(const int *h_image, int *h_labels, int n, int xsize, int ysize,
                      int zsize, const float *h_per_class, int max_label,
                      const int *h_seeds, int n_seeds);
/* gpu/oift_gpu.cu:149-158: cost_mode 0 (f_max) only. */
OIFT_API int oift_gpu_run(int cost_mode, const int *h_image, int *h_labels, int n, int xsize,
                 int ysize, int zsize, const float *h_per_class, int max_label,
                 const int *h_seeds, int n_seeds);
/* Status of the last reference-compatible call on this host thread. */
OIFT_API int oift_b200_last_status(void);

#ifdef __cplusplus
}
#endif
#endif
