/*
 * ssim2b200.h -- C ABI of the B200-native SSIMULACRA2 engine.
 *
 * The engine is a drop-in for the `Ssimulacra2` type of the turbo-metrics
 * crate `ssimulacra2-cuda` (crates/ssimulacra2-cuda/src/lib.rs) and, sharing
 * its input conversion and pyramid, for the `Dssim` type of `dssim-cuda`
 * (crates/dssim-cuda/src/lib.rs).  Every entry point below names the
 * reference interface it replaces.  Signatures use
 * plain pointers and sizes only; `stream` arguments are `cudaStream_t` values
 * passed as `void *` (NULL = the legacy default stream).
 *
 * Images:
 *   linear f32   packed interleaved RGB, 3 floats per pixel, rows `pitch`
 *                bytes apart (the NPP C3 layout the reference binds)
 *   sRGB8        packed interleaved RGB, 3 bytes per pixel, gamma-2.4 sRGB
 *   NV12         8-bit 4:2:0, Y plane then interleaved CbCr plane (w/2 pairs
 *                per row, h/2 rows), both with the same `pitch`; BT.709 or
 *                BT.601-525/625 matrix, limited or full range
 *   P016         the same layout with 16-bit samples (P010/P012 left-aligned)
 *   RGB16        packed RGB uint16 code values of `bits` bits (10 or 12),
 *                BT.2020 primaries, BT.709/BT.2020 transfer
 * Device pointers must stay valid until the stream work completes.
 *
 * Results: the score and the 108 pooled statistics, in the order of the
 * reference weight table: index = c*36 + scale*6 + norm*3 + map, c in
 * {X, Y, B}, norm 0 = mean (L1), 1 = (mean d^4)^(1/4) (L4), map 0 = SSIM
 * error, 1 = artifact, 2 = detail loss.  Unscored scales hold 0.
 *
 * Thread safety: one context per thread, or external synchronisation.  No
 * process-global state except the no-allocation entry point's scratch and
 * the tile-height autotuner's per-class choices (mutex-protected).
 */
#ifndef SSIM2B200_H
#define SSIM2B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define S2_ABI_VERSION 1
#define S2_NUM_STATS 108
#define S2_NUM_SCALES 6

typedef enum {
    S2_OK = 0,
    S2_ERR_OOM = 1,            /* device allocation failed or over the HBM budget */
    S2_ERR_INVALID_SIZE = 2,   /* width or height below 8 (or above the limit) */
    S2_ERR_DIM_MISMATCH = 3,   /* image does not match the context's size */
    S2_ERR_NO_REFERENCE = 4,   /* compute_with_reference without a cached reference */
    S2_ERR_CUDA = 5,           /* a CUDA runtime call failed (see s2_last_error) */
    S2_ERR_TIMEOUT = 6,        /* a bounded wait ran out */
    S2_ERR_BUSY = 7,           /* server queue full / admission refused */
    S2_ERR_INVALID_ARG = 8,    /* NULL pointer, bad enum, bad pitch */
    S2_ERR_NOT_READY = 9,      /* result not computed yet */
    S2_ERR_CANCELLED = 10      /* job cancelled by the caller */
} s2_status;

/* Blur arithmetic. */
enum {
    /* Default.  Separable 9-tap FIR (the exact closed form of the reference's
     * recursive Gaussian), fused with the error maps in one pass per scale,
     * f32 arithmetic on block-shifted moments, the SSIM error formed from
     * the blurred difference of the two images.  Scores within ~3e-5 of
     * the FP64 oracle. */
    S2_BLUR_FIR = 0,
    /* The reference's own f32 recursive walk (ssimulacra2-kernel blur.rs:95-136),
     * vertical then horizontal, reproduced operation for operation, so that
     * the 108 statistics match ssimulacra2-cuda's arithmetic. */
    S2_BLUR_IIR_REF = 1
};

/* Storage type of the intermediate pyramid levels and reference caches.
 * Only S2_STORAGE_F32 is accepted; the 16-bit values are kept for ABI
 * stability and make s2_config-taking constructors return
 * S2_ERR_INVALID_ARG (both passes are compute-bound, so 16-bit planes buy no
 * time, and they cost up to 0.2 (F16) and 4 (BF16) in score). */
enum { S2_STORAGE_F32 = 0, S2_STORAGE_F16 = 1, S2_STORAGE_BF16 = 2 };

/* Which pyramid scales are scored. */
enum {
    S2_SCALES_CPU = 0,  /* CPU crate ssimulacra2 0.5.1 (examples/cpu.rs:359-361) */
    S2_SCALES_MIN8 = 1, /* ssim2-gpu (pipeline.rs:194-206): scales >= 8x8 only */
    S2_SCALES_ALL6 = 2  /* ssimulacra2-cuda (lib.rs:138-143): always 6 */
};

/* 4:2:0 YUV matrix / range selectors (cuda-colorspace/src/lib.rs:9-20 ColorMatrix;
 * cuda-colorspace-kernel/src/lib.rs:46-140 Full / Limited).  The reference
 * implements limited range only (full range is todo!()); full range here
 * follows its Full definition (0 .. 2^N - 1, chroma neutral 2^(N-1)). */
enum { S2_MATRIX_BT709 = 0, S2_MATRIX_BT601_525 = 1, S2_MATRIX_BT601_625 = 2 };
enum { S2_RANGE_LIMITED = 0, S2_RANGE_FULL = 1 };

typedef struct {
    uint32_t struct_size;  /* sizeof(s2_config) */
    int32_t device;        /* CUDA device ordinal */
    int32_t blur;          /* S2_BLUR_* */
    int32_t storage;       /* S2_STORAGE_* */
    int32_t scale_rule;    /* S2_SCALES_* */
    int32_t strip_rows;    /* rows per fused tile: 16/32/64, or 0 = autotuned: the first
                              submission of a workload class (work items in half-octave
                              buckets) times the tile pass at each height and the
                              fastest is kept for the class (process-wide) */
    uint64_t hbm_budget;   /* bytes this context may allocate; 0 = no limit */
} s2_config;

typedef struct {
    double score;
    double stats[S2_NUM_STATS];
    double sums[S2_NUM_STATS]; /* raw pooled sums: sum d (L1 slots), sum d^4 (L4 slots) */
    int32_t n_scales;
    int32_t status;            /* s2_status of this pair */
    /* DSSIM (the sibling metric of crates/dssim-cuda, scored from the same
     * pyramid when S2_METRIC_DSSIM is on): the value and the five per-scale
     * scores 1 - mean |mean^(0.5^s) - ssim|.  NaN when DSSIM was not scored. */
    double dssim;
    double dssim_scale[5];
} s2_result;

typedef struct s2_ctx s2_ctx;

/* ---- library ---------------------------------------------------------- */
const char *s2_version(void);
const char *s2_status_string(s2_status st);
/* Message of the last failing CUDA call on this thread (empty if none). */
const char *s2_last_error(void);
void s2_config_default(s2_config *cfg);
/* Number of scales scored for a w x h pair under a rule (0 if too small). */
int s2_num_scales(uint32_t w, uint32_t h, int32_t scale_rule);
/* The 4:2:0 YUV conversion coefficients the engine uses for a matrix
 * (S2_MATRIX_*), range (S2_RANGE_*) and sample depth (8 for NV12, 16 for
 * P016): y_coeff, r_coeff, b_coeff, g_coeff1, g_coeff2 as
 * MatrixCoefficients::coefficients computes them (cuda-colorspace-kernel/
 * src/lib.rs:188-203, Kr / Kb from constants_from_primaries :205-221, in
 * f32), the luma minimum and the chroma neutral value (lib.rs:46-140).
 * Introspection for parity checks; S2_ERR_INVALID_ARG on a bad selector. */
s2_status s2_yuv_coefficients(int32_t matrix, int32_t range, int32_t bits, float coeffs[5],
                              int32_t *luma_min, int32_t *chroma_neutral);

/* ---- single pair (the drop-in) ----------------------------------------- */

/* Replaces Ssimulacra2::new (ssimulacra2-cuda/src/lib.rs:80-197).  Allocates
 * every intermediate for a w x h pair.  Unlike the reference, the context is
 * not bound to input pointers: they are passed per call.  Errors instead of
 * panics: S2_ERR_INVALID_SIZE (< 8 under the CPU/MIN8 rules), S2_ERR_OOM
 * (pre-flight estimate over the free memory or the budget, or a failed
 * allocation), S2_ERR_CUDA. */
s2_status s2_create(const s2_config *cfg, uint32_t width, uint32_t height, s2_ctx **out);
/* Replaces Drop for Ssimulacra2 (lib.rs:1195-1202); synchronises only this
 * context's own work, then frees. */
void s2_destroy(s2_ctx *ctx);
/* Replaces Ssimulacra2::mem_usage (lib.rs:207-235): device bytes owned. */
s2_status s2_mem_usage(const s2_ctx *ctx, size_t *bytes);
s2_status s2_dimensions(const s2_ctx *ctx, uint32_t *width, uint32_t *height);

/* Replaces Ssimulacra2::compute (lib.rs:421-424): enqueue the whole pair
 * pipeline on `stream`, asynchronously.  Inputs are linear RGB on the device. */
s2_status s2_compute_linear_f32(s2_ctx *ctx, const float *ref, size_t ref_pitch,
                                const float *dis, size_t dis_pitch, void *stream);
/* Replaces compute_srgb_sync / compute_from_cpu_srgb_sync (lib.rs:329-345,
 * 391-404) without the sync: sRGB8 inputs on the device (on_host = 0) or in
 * host memory (on_host = 1; copied through the context's staging buffers). */
s2_status s2_compute_srgb8(s2_ctx *ctx, const uint8_t *ref, size_t ref_pitch,
                           const uint8_t *dis, size_t dis_pitch, int32_t on_host,
                           void *stream);
/* NV12 pair (cuda-colorspace biplanaryuv420_to_linearrgb_8_{l}_{bt709,
 * bt601_525,bt601_625} followed by Ssimulacra2::compute; cuda-colorspace/src/
 * lib.rs:33-82), conversion fused.  matrix S2_MATRIX_*, range S2_RANGE_*. */
s2_status s2_compute_nv12(s2_ctx *ctx, const uint8_t *ref_y, const uint8_t *ref_uv,
                          size_t ref_pitch, const uint8_t *dis_y, const uint8_t *dis_uv,
                          size_t dis_pitch, int32_t matrix, int32_t range, int32_t on_host,
                          void *stream);
/* P016 pair: 16-bit samples in both planes (P010 / P012 data, left-aligned,
 * is read the same way), as biplanaryuv420_to_linearrgb_16_* (cuda-colorspace/
 * src/lib.rs:84-131).  Pitch in bytes. */
s2_status s2_compute_p016(s2_ctx *ctx, const uint16_t *ref_y, const uint16_t *ref_uv,
                          size_t ref_pitch, const uint16_t *dis_y, const uint16_t *dis_uv,
                          size_t dis_pitch, int32_t matrix, int32_t range, int32_t on_host,
                          void *stream);
/* 10/12-bit BT.2020 RGB pair (no reference counterpart: the reference has no
 * BT.2020 path; cuda-colorspace/src/lib.rs:46-68 are todo!()). */
s2_status s2_compute_rgb16(s2_ctx *ctx, const uint16_t *ref, size_t ref_pitch,
                           const uint16_t *dis, size_t dis_pitch, int32_t bits,
                           int32_t on_host, void *stream);

/* Replaces Ssimulacra2::get_score (lib.rs:427-429, post_process_scores
 * :1018-1192).  Waits for the last enqueued compute of this context and
 * returns its result.  Idempotent (the reference re-weights its buffer in
 * place on every call).  `stats` / `sums` may be NULL. */
s2_status s2_get_result(s2_ctx *ctx, double *score, double stats[S2_NUM_STATS],
                        double sums[S2_NUM_STATS]);
/* Replaces Ssimulacra2::compute_sync (lib.rs:409-416). */
s2_status s2_compute_sync_linear_f32(s2_ctx *ctx, const float *ref, size_t ref_pitch,
                                     const float *dis, size_t dis_pitch, void *stream,
                                     double *score);

/* ---- cached reference -------------------------------------------------- */
/* Replaces set_reference_linear (lib.rs:440-546): keeps the reference's
 * XYB pyramid resident on the device; compute_with_reference then converts
 * only the distorted image, and its scores equal the direct path's bit for
 * bit (the same tile pass over the same planes).  The reference also keeps
 * the blurred mu1 / sigma11; here they would save no work (the tile pass
 * blurs its planes in f32x2 pairs), so they are not kept. */
s2_status s2_set_reference_linear_f32(s2_ctx *ctx, const float *ref, size_t pitch, void *stream);
s2_status s2_set_reference_srgb8(s2_ctx *ctx, const uint8_t *ref, size_t pitch,
                                 int32_t on_host, void *stream);
/* Replaces compute_with_reference_linear (lib.rs:556-590); returns
 * S2_ERR_NO_REFERENCE where the reference panics.  Asynchronous: read the
 * result with s2_get_result. */
s2_status s2_compute_with_reference_linear_f32(s2_ctx *ctx, const float *dis, size_t pitch,
                                               void *stream);
s2_status s2_compute_with_reference_srgb8(s2_ctx *ctx, const uint8_t *dis, size_t pitch,
                                          int32_t on_host, void *stream);
/* Replaces clear_reference / has_reference (lib.rs:595-602). */
s2_status s2_clear_reference(s2_ctx *ctx);
int32_t s2_has_reference(const s2_ctx *ctx);

/* Error-map export (the reference materialises the maps per scale,
 * ssimulacra2-cuda/src/lib.rs:965-970; the fused pass here pools them
 * without storing): writes the last compute's SSIM error, artifact and
 * detail-loss maps of `scale` to the device buffer `maps` as 9 float planes
 * [channel X, Y, B][ssim, artifact, detail], each h_s rows of `pitch` bytes
 * (w_s = ceil(w / 2^scale), h_s likewise).  Enqueued on `stream` after that
 * compute (its planes must not have been overwritten by another compute);
 * returns when the maps are written.  FIR blur only (S2_ERR_INVALID_ARG for
 * S2_BLUR_IIR_REF); S2_ERR_NOT_READY before a scored compute. */
s2_status s2_error_maps(s2_ctx *ctx, int32_t scale, float *maps, size_t pitch, void *stream);

/* ---- batches of pairs of uneven sizes ---------------------------------- */
/* Semantics from ssim2-gpu Ssim2Batch (pipeline_batch.rs:120-382), widened to
 * mixed sizes: all pairs of a submission run as one pyramid launch, one
 * persistent tile launch over every (pair, scale, strip) and one finalize
 * launch.  Pairs are any of the image formats above, mixed freely. */
typedef enum {
    S2_FMT_LINEAR_F32 = 0,
    S2_FMT_SRGB8 = 1,
    S2_FMT_NV12 = 2,  /* 4:2:0 biplanar, 8-bit samples */
    S2_FMT_RGB16 = 3,
    S2_FMT_P016 = 4   /* 4:2:0 biplanar, 16-bit samples */
} s2_format;

typedef struct {
    uint32_t width, height;
    int32_t format;          /* s2_format */
    int32_t bits;            /* RGB16 only */
    const void *ref, *dis;   /* packed image, or NV12 / P016 Y plane */
    const void *ref_uv, *dis_uv; /* NV12 / P016 CbCr planes */
    size_t ref_pitch, dis_pitch;
    int32_t matrix, range;   /* NV12 / P016: S2_MATRIX_*, S2_RANGE_* (0, 0 = BT.709 limited) */
} s2_pair_desc;

typedef struct s2_batch s2_batch;

/* max_pairs: most pairs per submission; max_pixels: most scale-0 pixels of
 * all pairs of one submission together. */
s2_status s2_batch_create(const s2_config *cfg, uint32_t max_pairs, uint64_t max_pixels,
                          s2_batch **out);
void s2_batch_destroy(s2_batch *b);
/* Enqueue n pairs on `stream` (asynchronous).  A pair below 8x8 gets
 * S2_ERR_INVALID_SIZE in its result; the others run. */
s2_status s2_batch_submit(s2_batch *b, const s2_pair_desc *pairs, uint32_t n, void *stream);
/* The same submission with every plane in HOST memory (the decoder's output
 * buffers): the batch uploads the planes into its own device staging in up
 * to 16 groups of about equal pixel count on an internal copy stream, and
 * each group's launches on `stream` wait only for that group's planes, so the
 * uploads of later groups overlap the compute of earlier ones (ssim2-gpu's
 * batch takes device images only, pipeline_batch.rs:247-382; its callers
 * upload first, then compute).  Page-locked host memory gives asynchronous
 * uploads; pageable memory works, with each copy finishing before the call
 * goes on.  The host planes must stay unchanged until s2_batch_results
 * returns.  S2_ERR_DIM_MISMATCH if a pitch is below the row's bytes. */
s2_status s2_batch_submit_host(s2_batch *b, const s2_pair_desc *pairs, uint32_t n, void *stream);
/* Wait for the oldest submission whose results were not read yet (else the
 * last one again) and copy its n results.  A batch has two submission
 * slots: device-input submissions use the first; a host-input submission
 * takes a slot without pending results, so submission k+1 may be enqueued
 * before submission k's results are read (its uploads and preps overlap k's
 * tile pass).  With both slots pending, a new host submission drops the
 * older one's results. */
/* Replaces Ssim2Batch::set_reference (ssim2-gpu/src/pipeline_batch.rs:206-208):
 * converts `ref` (its ref / ref_uv planes, on the device; any format) and keeps
 * its XYB pyramid in the batch.  Returns after the device
 * work is done.  S2_ERR_INVALID_SIZE below 8x8 or above max_pixels. */
s2_status s2_batch_set_reference(s2_batch *b, const s2_pair_desc *ref, void *stream);
/* Replaces Ssim2Batch::compute_batch (pipeline_batch.rs:247-330): enqueue n
 * distorted images (the dis / dis_uv planes of each descriptor, on the
 * device, any format) against the cached reference, as one submission; read
 * the results with s2_batch_results.  S2_ERR_NO_REFERENCE without
 * s2_batch_set_reference, S2_ERR_DIM_MISMATCH for a size other than the
 * reference's, S2_ERR_INVALID_ARG beyond max_pairs / max_pixels (the
 * reference's InvalidBatchSize).  SSIMULACRA2 only. */
s2_status s2_batch_submit_with_reference(s2_batch *b, const s2_pair_desc *dis, uint32_t n, void *stream);
/* Replaces clear_reference / has_cached_reference (pipeline_batch.rs:210-216). */
s2_status s2_batch_clear_reference(s2_batch *b);
int32_t s2_batch_has_reference(const s2_batch *b);
s2_status s2_batch_results(s2_batch *b, s2_result *out, uint32_t n);
s2_status s2_batch_mem_usage(const s2_batch *b, size_t *bytes);
/* CUDA graphs (1 = on, the default): the operations of a device-input
 * submission (descriptor upload, counter reset, prep, tile pass, finalize,
 * result download) are recorded once per plan shape (pair count and block,
 * tile and segment counts) and replayed for later submissions of that shape,
 * like the reference's graph per bound pair (ssimulacra2-cuda/src/lib.rs:
 * 409-424); pointers and sizes of the pairs travel in the uploaded
 * descriptors, so one graph serves any pairs of the shape.  Host-input
 * submissions and profiled submissions launch directly. */
s2_status s2_batch_set_graphs(s2_batch *b, int32_t enable);
/* The same switch for a single-pair context (default on). */
s2_status s2_set_graphs(s2_ctx *ctx, int32_t enable);

/* ---- DSSIM, the sibling metric sharing the pyramid ----------------------
 * DSSIM as crates/dssim-cuda computes it (five scales of dssim-core's scaled
 * Lab, two-pass 3x3 blurs, a channel-averaged SSIM map, per-scale
 * 1 - mean |mean^(0.5^s) - ssim|, weighted, 1/ssim - 1), scored from the
 * same prep pass as SSIMULACRA2: the pass reads each input once, builds one
 * linear-RGB pyramid and writes the XYB planes of one metric and the Lab
 * planes of the other side by side.  Any input format of this library
 * (the reference's DSSIM takes sRGB8 only).  Scores are in s2_result's
 * dssim fields (s2_get_dssim for a context). */
enum { S2_METRIC_SSIMULACRA2 = 1, S2_METRIC_DSSIM = 2 };
/* Metrics scored by later submissions of a context or batch: a non-empty
 * set of S2_METRIC_* bits (default S2_METRIC_SSIMULACRA2).  With DSSIM alone
 * the SSIMULACRA2 fields of a result hold NaN / 0.  Cached-reference
 * submissions (s2_set_reference_* / s2_compute_with_reference_*) score
 * SSIMULACRA2 only (S2_ERR_INVALID_ARG on a context scoring DSSIM alone). */
s2_status s2_set_metrics(s2_ctx *ctx, int32_t metrics);
s2_status s2_batch_set_metrics(s2_batch *b, int32_t metrics);
/* The last submission's DSSIM and its five per-scale scores (waits for the
 * stream work).  S2_ERR_NOT_READY when that submission did not score DSSIM. */
s2_status s2_get_dssim(s2_ctx *ctx, double *dssim, double scale_scores[5]);

/* The drop-in for dssim-cuda's `Dssim` (crates/dssim-cuda/src/lib.rs:170-467):
 * a context of one size that scores DSSIM only. */
typedef struct s2_dssim s2_dssim;
/* Dssim::new (lib.rs:184-222).  S2_ERR_INVALID_SIZE below 8x8. */
s2_status s2_dssim_create(int32_t device, uint32_t width, uint32_t height, s2_dssim **out);
void s2_dssim_destroy(s2_dssim *d);
/* Dssim::compute_sync (lib.rs:225-232): sRGB8 images, device memory or,
 * with on_host, host memory; waits for the result. */
s2_status s2_dssim_compute_srgb8(s2_dssim *d, const uint8_t *ref, size_t ref_pitch, const uint8_t *dis,
                                 size_t dis_pitch, int32_t on_host, void *stream, double *dssim);
/* Dssim::compute_sync_dis_only (lib.rs:245-251): scores `dis` against the
 * reference of this context's last compute, whose Lab planes stay on the
 * device; only the distorted image is converted.  S2_ERR_NO_REFERENCE before
 * a first compute. */
s2_status s2_dssim_compute_dis_only_srgb8(s2_dssim *d, const uint8_t *dis, size_t dis_pitch, int32_t on_host,
                                          void *stream, double *dssim);
/* Dssim::mem_usage (lib.rs:438-451): device bytes held. */
s2_status s2_dssim_mem_usage(const s2_dssim *d, size_t *bytes);

/* ---- serving: continuous batching of jobs (reference + k candidates) -----
 * No single counterpart in the reference: it combines the cached-reference
 * path (ssimulacra2-cuda/src/lib.rs:440-860) with ssim2-gpu's batch
 * (pipeline_batch.rs:247-382) behind a worker thread.  Jobs of any size arrive
 * at any time; they are admitted in arrival order while their device bytes
 * fit the HBM budget, their images are uploaded on a copy stream, and every
 * round scores the pending work of all admitted jobs in one submission.  A
 * job's reference pyramid is built once and shared by its
 * candidates (scored as s2_compute_with_reference_* scores them).  A job
 * scores bit-identically alone and mixed with others.  Host images must stay
 * valid until s2_server_wait returns for the job. */
typedef struct {
    uint32_t struct_size;      /* sizeof(s2_server_config) */
    int32_t device;
    uint32_t max_batch_pairs;  /* candidates + reference builds per round */
    uint64_t max_batch_pixels; /* scale-0 pixels per round */
    uint64_t hbm_budget;       /* device bytes for admitted jobs + workspaces; 0 = no limit */
    uint32_t max_queued_jobs;  /* unfinished jobs (waiting or admitted); submit returns
                                  S2_ERR_BUSY beyond this (default 128: an overloaded
                                  server sheds work instead of growing its latency) */
} s2_server_config;

typedef struct {
    uint32_t width, height;
    int32_t format;                  /* S2_FMT_SRGB8 */
    const void *ref;                 /* host image */
    size_t ref_pitch;
    uint32_t n_candidates;
    const void *const *candidates;   /* host images */
    size_t cand_pitch;
} s2_job_desc;

typedef struct {
    uint64_t jobs_done, pairs_done, rounds, queued_jobs, hbm_in_use;
    double p50_ms, p99_ms, max_ms;   /* arrival -> completion of finished jobs */
    double uptime_s;
    double gpu_busy_s;               /* device time of the rounds' kernels */
    double worker_wait_s;            /* worker time blocked on finished rounds */
    double worker_upload_s;          /* worker time issuing uploads */
    double worker_submit_s;          /* worker time planning and enqueueing rounds */
    double copy_busy_s;              /* copy-stream time of finished jobs' uploads (CUDA events) */
    uint64_t bytes_uploaded;         /* host -> device bytes of finished jobs */
} s2_server_report;

typedef struct s2_server s2_server;

void s2_server_config_default(s2_server_config *cfg);
s2_status s2_server_create(const s2_server_config *cfg, s2_server **out);
/* Stops accepting work, finishes admitted jobs, frees everything. */
void s2_server_destroy(s2_server *sv);
/* S2_ERR_OOM if the job alone exceeds the budget, S2_ERR_BUSY if the queue is full. */
s2_status s2_server_submit(s2_server *sv, const s2_job_desc *job, uint64_t *job_id);
/* Waits up to timeout_ms for the job; S2_ERR_TIMEOUT if it is not done.  On
 * completion copies the n scores and per-candidate statuses and releases the
 * job; returns S2_ERR_CANCELLED for a cancelled job. */
s2_status s2_server_wait(s2_server *sv, uint64_t job_id, uint32_t timeout_ms, double *scores,
                         int32_t *statuses, double *latency_ms);
/* Candidates not yet on the GPU are dropped; in-flight ones finish. */
s2_status s2_server_cancel(s2_server *sv, uint64_t job_id);
s2_status s2_server_stats(s2_server *sv, s2_server_report *out);
s2_status s2_server_reset_stats(s2_server *sv);

/* ---- scoring one pair without allocating device memory --------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (a host framework that owns all device memory through its own pool, a
 * plug-in that must not grow the process's footprint after start-up, code
 * that must not block on the allocator): every intermediate lives in one
 * 16 MiB array inside the library, held on every GPU that loads the
 * library's device code.  The driver reserves it when it loads that code:
 * at library load with eager module loading, or -- under lazy module
 * loading, CUDA's default since 12.2 -- during the first call on each
 * device, which may then synchronise: make that first call at start-up.
 * sRGB8 pair on the device, default configuration (FIR blur, f32,
 * CPU-crate scale rule); the result is written to `out_device`, a device
 * buffer of one s2_result that the caller owns (read it after the stream
 * completes).  A pair whose layout does not fit the array returns
 * S2_ERR_INVALID_SIZE: any pair whose width and height are both at most 512
 * fits, larger ones are checked exactly.  All calls share the array, so calls
 * whose GPU work overlaps race: serialise them.  The first call on a device
 * sets the array up with that device current (a synchronous copy of the sRGB
 * table into it); make it before any stream capture.  Each call hands its
 * pair descriptor to the GPU as kernel arguments, so nothing reads the
 * caller's host memory after the call returns.  Allocates nothing. */
s2_status s2_compute_srgb8_noalloc(const uint8_t *ref, size_t ref_pitch, const uint8_t *dis,
                                   size_t dis_pitch, uint32_t width, uint32_t height,
                                   s2_result *out_device, void *stream);
/* (The no-allocation entry point scores SSIMULACRA2 only and leaves the
 * dssim fields of *out_device unwritten.) */

/* ---- zensim features (crates/zensim-cuda) ------------------------------ *
 * The feature side of zensim's GPU port: positive XYB at the SIMD-padded
 * width, 4 box-pyramid scales, radius-5 box blurs and, per scale and
 * channel, 13 pooled features + 6 peak features: 228 in all, in the order of
 * Zensim::compute_features (zensim-cuda/src/lib.rs:686-819; scales that the
 * image is too small for are 0).  The score itself needs the trained table
 * WEIGHTS_PREVIEW_V0_2 of the zensim crate, which is not part of the
 * reference tree, so no score is offered.  Sums are reduced in a fixed order
 * (the reference adds columns with float atomics). */
#define S2_ZENSIM_FEATURES 228
typedef struct s2_zensim s2_zensim;
/* Replaces Zensim::new (lib.rs:198-287): S2_ERR_INVALID_SIZE below 8x8. */
s2_status s2_zensim_create(int32_t device, uint32_t width, uint32_t height, s2_zensim **out);
void s2_zensim_destroy(s2_zensim *z);
/* Replaces Zensim::set_reference (lib.rs:340-376): packed sRGB8 rows of
 * `pitch` bytes, on the device or (on_host) in host memory; the reference's
 * pyramid stays resident.  Returns after the device work is done. */
s2_status s2_zensim_set_reference_srgb8(s2_zensim *z, const uint8_t *ref, size_t pitch, int32_t on_host,
                                        void *stream);
/* Replaces Zensim::compute_with_reference (lib.rs:388-395): the 228 features
 * of `dis` against the cached reference; *n_scales = scales computed.
 * S2_ERR_NO_REFERENCE without a reference.  Synchronous. */
s2_status s2_zensim_compute_with_reference_srgb8(s2_zensim *z, const uint8_t *dis, size_t pitch, int32_t on_host,
                                                 void *stream, double *features, int32_t *n_scales);
/* Replaces Zensim::compute_features (lib.rs:322-329): set_reference + compute. */
s2_status s2_zensim_compute_features_srgb8(s2_zensim *z, const uint8_t *ref, size_t ref_pitch, const uint8_t *dis,
                                           size_t dis_pitch, int32_t on_host, void *stream, double *features,
                                           int32_t *n_scales);
int32_t s2_zensim_has_reference(const s2_zensim *z);
s2_status s2_zensim_clear_reference(s2_zensim *z);
/* Replaces Zensim::debug_compute_raw (lib.rs:303-310): the last compute's
 * 17 sums per [scale][channel] (acc: 4 * 3 * 17 doubles) and 3 maxima per
 * [scale][channel] as f32 bits (peaks: 4 * 3 * 3). */
s2_status s2_zensim_raw(const s2_zensim *z, double *acc, uint32_t *peaks);
s2_status s2_zensim_mem_usage(const s2_zensim *z, size_t *bytes);

/* ---- kernel timing (no reference counterpart; the reference has commented-
 * out cuProfilerStart/Stop calls, ssimulacra2-cuda/src/lib.rs:311,963) ----
 * When enabled, CUDA events bracket the three launches of every submission;
 * `ms` receives the device time of the pyramid, fused and finalize kernels of
 * the last one. */
s2_status s2_profile_enable(s2_ctx *ctx, int32_t enable);
s2_status s2_profile_last(s2_ctx *ctx, float ms[3]);
s2_status s2_batch_set_profiling(s2_batch *b, int32_t enable);
s2_status s2_batch_last_timings(s2_batch *b, float ms[3]);
/* Device time of the DSSIM passes (clamp, tile, mean, MAD, final) of the
 * last profiled submission that scored DSSIM. */
s2_status s2_batch_last_dssim_ms(s2_batch *b, float *ms);
/* Failure-detection hook of the tile pass.  Every wait of the tile pass on
 * its bulk row copies is bounded (wait_cycles SM clock cycles; 0 restores
 * the default, about one second); a wait that runs out makes the submission
 * report S2_ERR_TIMEOUT instead of hanging.  drop_item >= 0 makes the pass
 * withhold the row copies of that work item, so that its waits run out: the
 * way the tests exercise that path without any fault.  -1 (the default)
 * withholds nothing.  Process-wide; read when a submission is enqueued (a
 * CUDA graph keeps the values it was captured with). */
s2_status s2_debug_tile_timeout(int32_t drop_item, int64_t wait_cycles);
/* Resident blocks per SM of the fused kernel for a storage type (0 on error). */
int32_t s2_fused_blocks_per_sm(int32_t storage);

#ifdef __cplusplus
}
#endif
#endif
