/*
 * artefact_b200 -- C ABI of the B200 (sm_100a) JPEG restoration solver.
 *
 * Drop-in replacement for the solver entry point of Delnegend/artefact's
 * artefact-lib. Citations (file:line) refer to that project's
 * backend/artefact-lib/ and backend/zune-jpeg/ trees.
 *
 * Conventions: every function returns ART_OK (0) or a negative ART_ERR_* code;
 * on error, art_last_error() returns a message for the calling thread. All
 * entry points are thread-safe and re-entrant: concurrent calls from different
 * host threads (the reference calls compute() from rayon workers in
 * separate-components mode, lib.rs:133-153) each use their own CUDA stream.
 * Pointers are plain host pointers unless a name says _device.
 */
#ifndef ARTEFACT_B200_H
#define ARTEFACT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ART_OK 0
#define ART_ERR_INVALID_ARGUMENT (-1) /* bad sizes, sampling factors, null pointers */
#define ART_ERR_INVALID_DATA (-2)     /* non-integral / out-of-range coefficients, quant entries <= 0 */
#define ART_ERR_CUDA (-3)             /* CUDA runtime failure (no device, out of memory, launch error) */
#define ART_ERR_DECODE (-4)           /* JPEG stream could not be decoded */
#define ART_ERR_UNSUPPORTED (-5)      /* valid input outside what this build handles */

#define ART_COEF_F32 0 /* dct_coefs points to float values (integral), as jpeg/zune.rs:33-37 makes them */
#define ART_COEF_I16 1 /* dct_coefs points to int16 values, as the decoder produces them */

#define ART_INIT_DECODED 0       /* x0 = block IDCT of c*q, unboxed once (pipeline_simd_adaptive/coef.rs:69-95) */
#define ART_INIT_SCALAR_COMPAT 1 /* x0 as pipeline_scalar/coef.rs:29-50 builds it (per-block whole-plane unboxing) */
#define ART_INIT_LEARNED 2       /* x0 = projection of the warm-start network's prediction (art_context_set_warm_start);
                                    no reference counterpart: only the starting point changes, the iteration is the
                                    reference's */

typedef struct ArtNet ArtNet; /* warm-start network, declared with its functions at the end of this file */

/*
 * One JPEG component as the solver receives it.
 * Replaces: struct Coefficient, backend/artefact-lib/jpeg/mod.rs:8-27.
 */
typedef struct ArtChannel {
    uint32_t rounded_px_w; /* component plane width, multiple of 8 */
    uint32_t rounded_px_h; /* component plane height, multiple of 8 */
    uint32_t block_w;      /* rounded_px_w / 8 */
    uint32_t block_h;      /* rounded_px_h / 8 */
    uint32_t samp_h;       /* horizontal sampling factor relative to the max: 1 or 2 */
    uint32_t samp_v;       /* vertical sampling factor relative to the max: 1 or 2 */
    uint32_t coef_type;    /* ART_COEF_F32 or ART_COEF_I16 */
    uint32_t reserved;
    const void *dct_coefs;    /* block_w*block_h*64 values: blocks in raster order, natural (v*8+u) order inside */
    const float *quant_table; /* 64 quantisation steps, natural order */
} ArtChannel;

typedef struct ArtOptions {
    uint32_t init_mode;       /* ART_INIT_DECODED (default), ART_INIT_SCALAR_COMPAT or ART_INIT_LEARNED */
    int32_t device;           /* CUDA device ordinal, -1 = current device */
    uint32_t step_iterations; /* 0: step size radius / sqrt(1 + iterations) as mod.rs:71 forms it; otherwise
                                 radius / sqrt(1 + step_iterations), the step of a run of that many iterations
                                 (a refinement after a learned start can take a long run's step) */
    uint32_t tail_iterations; /* 0: one phase (the reference). Otherwise the last tail_iterations of the
                                 `iterations` form a second phase: FISTA restarted and steps of
                                 radius / sqrt(1 + tail_step_iterations) -- large steps first to remove a warm
                                 start's error, then small ones to settle. No reference counterpart. */
    uint32_t tail_step_iterations;
    float step_decay;         /* 0: constant steps in the first phase (the reference). In (0, 1]: step k of the
                                 first phase is step_decay^k times the solve's step, so a warm start's
                                 refinement can shrink its steps geometrically. No reference counterpart. */
    uint32_t reserved[2];
} ArtOptions;

typedef struct ArtContext ArtContext;

/* Message describing the last error on the calling thread ("" if none). */
const char *art_last_error(void);

/* Library version string. */
const char *art_version(void);

/*
 * Run the solver on one image.
 * Replaces: pipeline_scalar::compute, backend/artefact-lib/pipeline_scalar/mod.rs:17-78
 * (same signature in pipeline_simd_8/mod.rs:22-31 and pipeline_simd_adaptive/mod.rs:19-28):
 *   compute(nchannel, coefs, weight, pweight, iterations, max_rounded_px_w,
 *           max_rounded_px_h, max_rounded_px_count) -> Vec<Vec<f32>>
 * out_planes[c] receives max_rounded_px_count floats (row stride max_rounded_px_w),
 * level-shifted like the reference's return value (no +128 on luma).
 * nchannel is 1..3; channel c uses pweight[c] (compute_step.rs:19-26).
 * opts may be NULL (decoded init, current device).
 */
int32_t art_compute(uint32_t nchannel, const ArtChannel *coefs, float weight, const float pweight[3],
                    uint32_t iterations, uint32_t max_rounded_px_w, uint32_t max_rounded_px_h,
                    uint64_t max_rounded_px_count, float *const *out_planes, const ArtOptions *opts);

/* Explicit contexts: device buffers, CUDA graphs and a stream reused across calls.
 * A context must not be used by two threads at once. */
int32_t art_context_create(int32_t device, ArtContext **out);
void art_context_destroy(ArtContext *ctx);

/* art_compute on an explicit context. */
int32_t art_context_compute(ArtContext *ctx, uint32_t nchannel, const ArtChannel *coefs, float weight,
                            const float pweight[3], uint32_t iterations, uint32_t max_rounded_px_w,
                            uint32_t max_rounded_px_h, float *const *out_planes, const ArtOptions *opts);

/*
 * Device-resident variant: ArtChannel.dct_coefs points to device memory (the
 * 64-entry quant_table stays a host pointer), out_planes_device[c] to device buffers of max_rounded_px_h rows of
 * out_pitch floats. The work runs on the context's stream, ordered after the
 * work already queued on `stream` (a cudaStream_t; NULL is the legacy default
 * stream) and before anything queued on `stream` afterwards; the call returns
 * without synchronising.
 * Replaces the same reference entry point as art_compute.
 */
int32_t art_context_compute_device(ArtContext *ctx, uint32_t nchannel, const ArtChannel *coefs, float weight,
                                   const float pweight[3], uint32_t iterations, uint32_t max_rounded_px_w,
                                   uint32_t max_rounded_px_h, float *const *out_planes_device, uint32_t out_pitch,
                                   const ArtOptions *opts, void *stream);

/*
 * Solver dispatch and output stage of Artefact::process (lib.rs:105-212) on
 * decoded coefficients: with nchannel == 3 and separate == 0 one joint solve
 * with weight[0], pweight and iterations[0] (lib.rs:122-132); otherwise each
 * component alone with weight[c], pweight (so pweight[0] for every component,
 * as compute(1, ...) reads it) and iterations[c] (lib.rs:133-153). Then luma
 * + 128, YCbCr -> RGB with truncating u8 casts and crop to real_w x real_h
 * (lib.rs:159-211), fused on the GPU. rgb_out receives real_h*real_w*3 bytes;
 * NULL skips the output stage (benchmark mode, lib.rs:155-157).
 * Replaces: Artefact::process after Jpeg::from, backend/artefact-lib/lib.rs:108-211.
 */
int32_t art_context_process(ArtContext *ctx, uint32_t nchannel, const ArtChannel *coefs, const float weight[3],
                            const float pweight[3], const uint32_t iterations[3], int32_t separate, uint32_t real_w,
                            uint32_t real_h, uint8_t *rgb_out, const ArtOptions *opts);

/*
 * A batch of images solved together: every gradient sweep and projection of an
 * iteration covers all images in one launch (per channel count and sampling
 * mode), and the fixed-count iteration loop is one captured CUDA graph.
 * Each image has its own size, channels, sampling, weight and pweight; all run
 * `iterations` steps. Per image the result equals art_compute's.
 * No reference counterpart (the reference solves one image per call); it
 * batches what artefact-lib's callers would do in a loop over
 * compute(), pipeline_scalar/mod.rs:17-78.
 */
typedef struct ArtImage {
    uint32_t nchannel;
    uint32_t max_rounded_px_w, max_rounded_px_h;
    uint32_t out_pitch;            /* device variant: floats per output row (>= width); host variant ignores it */
    const ArtChannel *channels;    /* nchannel components */
    float weight;
    float pweight[3];
    float *const *out_planes;      /* nchannel planes */
} ArtImage;

/* Host coefficients in, host planes (row stride = width) out. */
int32_t art_context_compute_batch(ArtContext *ctx, uint32_t nimages, const ArtImage *images, uint32_t iterations,
                                  const ArtOptions *opts);
/* Device coefficients in, device planes out; ordered after `stream`, returns without synchronising. */
int32_t art_context_compute_batch_device(ArtContext *ctx, uint32_t nimages, const ArtImage *images,
                                         uint32_t iterations, const ArtOptions *opts, void *stream);

/*
 * art_context_process for many decoded images at once: each image's solves
 * (one joint solve of a 3-component image unless `separate`, else one per
 * component reading pweight[0], lib.rs:122-153) all run in one batched solve
 * of `iterations` steps, then the fused output stage (lib.rs:159-211) writes
 * each image's real_h*real_w*3 RGB bytes to its host rgb_out (NULL skips it).
 * Per image the RGB equals art_context_process's with iterations[c] =
 * `iterations`. Host coefficients; returns when done.
 * Replaces: a loop of Artefact::process calls after Jpeg::from,
 * backend/artefact-lib/lib.rs:105-212.
 */
typedef struct ArtProcessImage {
    uint32_t nchannel;          /* 1..4 components */
    uint32_t real_w, real_h;    /* real image size (crop of the rounded planes) */
    uint32_t reserved;
    const ArtChannel *channels; /* host coefficients */
    float weight[3];            /* joint solve: weight[0]; separate: weight[c] (weight[2] for a 4th) */
    float pweight[3];
    uint8_t *rgb_out;
} ArtProcessImage;
int32_t art_context_process_batch(ArtContext *ctx, uint32_t nimages, const ArtProcessImage *images,
                                  uint32_t iterations, int32_t separate, const ArtOptions *opts);

/*
 * Autotuner (no reference counterpart). It picks the launch shapes of the two
 * kernels of an iteration: the gradient sweep's variant (0 = narrow, one
 * column per lane; 1 = wide, two columns per lane on packed FP32x2
 * arithmetic; 2 = quad, four columns per lane, float4 loads and stores and
 * packed FP32x2 arithmetic) and strip height (16, 32, 64 or 128 rows), then the
 * projection's warps per block (2, 4 or 8; blocks per SM follow from it and
 * the shared memory a warp stages). Candidates are timed on the GPU
 * (`iterations` steps, 0 = 10; each captured and warmed once, then timed 5
 * times, median), sweep first with the projection at 4 warps, then the
 * projection with the chosen sweep. The size heuristic's choice is tried
 * first and the first candidate within 2 % of the fastest wins, so the
 * choice changes only for a clear gain and repeats from run to run. The
 * variants sum the same terms in different orders (results agree to fp32
 * rounding), and each is deterministic.
 *
 * art_context_autotune tunes one geometry on a deterministic synthetic image
 * and caches the choice for its bucket (channel count, sampling, width and
 * height rounded up to powers of two); later solves of images in that bucket
 * use it. art_context_autotune_batch tunes on the given batch itself (host
 * coefficients, as art_context_compute_batch takes them) and caches the
 * choice for batches of its bucket (image count and total pixels rounded up to
 * powers of two), which takes precedence over the per-image buckets in batched
 * solves. art_context_last_tune returns the last run's choice and timings,
 * art_context_tune_candidates the timing of every candidate it tried.
 * art_context_tune_cache saves (save != 0) or loads the cache as a text file
 * of "<bucket> <variant> <rows> <projection warps>" lines (three-field lines
 * keep 4 projection warps). Output pointers may be NULL.
 */
typedef struct ArtTuneResult {
    uint32_t variant, strip_rows, proj_warps; /* the choice */
    uint32_t candidates;                      /* candidates timed */
    float best_ms;                            /* the choice's median time for `iterations` steps */
    float heuristic_ms;                       /* the size heuristic's shape (4 projection warps), same measure */
    uint32_t heuristic_variant, heuristic_strip_rows;
} ArtTuneResult;
int32_t art_context_autotune(ArtContext *ctx, uint32_t nchannel, const uint32_t *samp_h, const uint32_t *samp_v,
                             uint32_t max_rounded_px_w, uint32_t max_rounded_px_h, uint32_t iterations,
                             uint32_t *variant_out, uint32_t *strip_rows_out);
int32_t art_context_autotune_batch(ArtContext *ctx, uint32_t nimages, const ArtImage *images, uint32_t iterations,
                                   ArtTuneResult *out);
int32_t art_context_last_tune(ArtContext *ctx, ArtTuneResult *out);
/* Every candidate the last autotune run timed, in the order it timed them:
 * up to `capacity` entries into out; *count receives the number timed. */
typedef struct ArtTuneCandidate {
    uint32_t variant, strip_rows, proj_warps;
    float ms; /* median time for the run's `iterations` steps */
} ArtTuneCandidate;
int32_t art_context_tune_candidates(ArtContext *ctx, ArtTuneCandidate *out, uint32_t capacity, uint32_t *count);
int32_t art_context_tune_cache(ArtContext *ctx, const char *path, int32_t save);

/*
 * Attach the warm-start network used by ART_INIT_LEARNED solves on this
 * context (NULL detaches). The network must live on the context's device and
 * outlive its use; it is not owned by the context. With a learned start, each
 * component's prediction (art_net_predict at the component's resolution) is
 * upsampled to full resolution along each subsampled axis by linear
 * interpolation between cell centres (sample 2 i + d of cell i = 3/4 of cell i
 * + 1/4 of cell i - 1 for d = 0, of cell i + 1 for d = 1, clamped at the
 * edges; horizontal first, every product and sum rounded to float), projected
 * onto the quantisation box, and the solve's `iterations` plain iterations
 * refine it with the FISTA sequence restarted. No reference counterpart.
 * The predictions of one solve run on the context's two streams, each with
 * one of the network's two sets of activation buffers; so learned solves on
 * different contexts that share one network must not overlap in time. The
 * second learned solve of one geometry on a context records the prediction
 * launches as a CUDA graph, which later solves of that geometry replay.
 */
int32_t art_context_set_warm_start(ArtContext *ctx, ArtNet *net);
/*
 * Attach a joint 4:2:0 warm-start network (art_net_predict_joint; NULL
 * detaches). ART_INIT_LEARNED solves of 4:2:0 images (three components, luma
 * H x W and both chroma H/2 x W/2, H and W multiples of 16) then predict all
 * three components at full resolution in one pass of it; other images use the
 * network of art_context_set_warm_start. Same lifetime and sharing rules.
 */
int32_t art_context_set_joint_warm_start(ArtContext *ctx, ArtNet *net);

/*
 * Objective and feasibility of image `image`'s result of the context's last
 * solve, in fp64 on the GPU (waits for the solve). out[0] = objective E,
 * out[1..3] = its TV, TGV and DCT-distance terms, out[4] = the largest
 * distance (coefficient units) by which a DCT coefficient of a result block
 * (cell-averaged for subsampled components) lies outside its quantisation
 * interval, 0 when all are inside. E is the function whose gradient the
 * reference follows (compute_step_tv.rs:63-71, compute_step_tv2.rs:76-90,
 * compute_step_prob.rs:24-55); the reference itself never evaluates it
 * (compute_step.rs:39-48 discards the TV value).
 */
int32_t art_context_evaluate(ArtContext *ctx, uint32_t image, double out[5]);

/* Wait for the context's queued work; returns the first error it met. */
int32_t art_context_synchronize(ArtContext *ctx);

/*
 * Kernel timing of the last device-resident solve on this context, measured
 * with CUDA events around the iteration loop: total milliseconds and, per
 * kernel kind, summed milliseconds over all launches (gradient, update).
 * Only filled when the context was created with timing enabled.
 */
int32_t art_context_set_timing(ArtContext *ctx, int32_t enabled);
int32_t art_context_last_timing(ArtContext *ctx, float *loop_ms, float *gradient_ms, float *update_ms,
                                uint32_t *launches);

/*
 * Allocation-free solve. No counterpart in the reference: artefact-lib runs
 * on the CPU and owns its buffers. For callers that must not allocate device
 * memory -- their GPU memory belongs to another allocator (a framework's
 * caching allocator, a server that partitions each GPU up front), or they
 * cannot afford the device-wide synchronisation cudaMalloc/cudaFree may
 * imply. It runs the iteration of a default-options solve (decoded start, the
 * reference's step size and one FISTA phase) with the narrow gradient sweep
 * and 32-row strips whatever the image size, so its result equals
 * art_context_compute_device's within the parity tolerance (the sweep
 * variant and strip height change the summation order), not bit for bit.
 * Every scratch buffer comes from one fixed 64 MiB array in device memory that the
 * library holds on every GPU it is loaded on until the process exits; images
 * that need more (about 1 megapixel per channel) are rejected with
 * ART_ERR_INVALID_ARGUMENT. dct_coefs and out_planes_device are device
 * pointers, quant_table a host pointer; work runs on `stream` (NULL = legacy
 * default stream) and the call returns when it is done. The first call on a
 * device resolves the array's address there (cudaGetSymbolAddress), so make
 * that first call before any CUDA stream capture. All calls share the array, so
 * calls whose GPU work overlaps race; each call clears what must start at zero.
 * A call that fails after queueing work waits for that work before returning.
 */
int32_t art_solve_noalloc(uint32_t nchannel, const ArtChannel *coefs, float weight, const float pweight[3],
                          uint32_t iterations, uint32_t max_rounded_px_w, uint32_t max_rounded_px_h,
                          float *const *out_planes_device, uint32_t out_pitch, void *stream);

/* ---- host JPEG front end (stand-in for jpeg/zune.rs:5-55 on the host) ---- */

typedef struct ArtJpeg ArtJpeg;

/* Decode the entropy-coded coefficients of a baseline JPEG held in memory.
 * Replaces: Jpeg::from, backend/artefact-lib/jpeg/zune.rs:5-55. */
int32_t art_jpeg_decode(const uint8_t *data, size_t len, ArtJpeg **out);
void art_jpeg_free(ArtJpeg *jpeg);
/* real_px_w/h and component count (jpeg/mod.rs:30-36). */
int32_t art_jpeg_info(const ArtJpeg *jpeg, uint32_t *nchannel, uint32_t *real_px_w, uint32_t *real_px_h);
/* Fill `out` with component c; pointers stay valid until art_jpeg_free. coef_type is ART_COEF_I16. */
int32_t art_jpeg_channel(const ArtJpeg *jpeg, uint32_t c, ArtChannel *out);


/* ------------------------------------------------------------------------
 * Warm-start network kernels (no counterpart in the reference: the network
 * only chooses the solver's starting point). All pointers are device
 * pointers; tensors are NHWC bf16 ([B][H][W][C], channels innermost) unless
 * stated; `stream` is a cudaStream_t (NULL = legacy default stream). `err`
 * is a device int that a kernel sets to 1 if one of its bounded waits gave up.
 * ------------------------------------------------------------------------ */

/* 3x3 convolution, stride 1, zero padding 1, BF16 x BF16 -> FP32 on the
 * tensor cores: out[p][n] = sum_{tap, c} x[p + d(tap)][c] * W[n][tap][c]
 * (+ bias, ReLU, zeroed where mask <= 0, + the previous output when
 * accumulate), stored as bf16 into channels [out_coff, out_coff + n_store) of
 * a tensor with out_cstride channels and/or as fp32 with f32_cstride.
 * wpack holds the weights as art_cnn_pack_weights lays them out for this ck
 * and n. cin is a multiple of ck (16 or 32); n, n_store multiples of 16,
 * n <= 128. */
typedef struct ArtCnnConv {
    int32_t B, H, W;
    int32_t cin, ck, n, n_store;
    const void *x;
    const void *wpack;
    const float *bias;
    void *out;
    int32_t out_cstride, out_coff;
    float *out_f32;
    int32_t f32_cstride;
    const void *mask;
    int32_t mask_cstride;
    int32_t relu, accumulate;
    int32_t *err;
    void *pool_out; /* optional: also the 2x2 average of the bf16 output (after bias / ReLU / mask),
                       [B][H/2][W/2][n_store]; H and W even */
    int32_t up2;    /* nonzero: `out` is 2H x 2W and each output pixel is stored to its 2x2 cell
                       (nearest upsampling fused into the store; not with accumulate) */
    int32_t tile_rows; /* output rows per 128-pixel tile: 1, 2, 4 or 8 with tile_rows x n <= 256
                          (a pooled output needs an even count); 0 picks by layer shape */
    int32_t f32_channels; /* channels 0 .. f32_channels-1 go to out_f32: a multiple of 4 up to n_store;
                             0 = n_store */
} ArtCnnConv;
int32_t art_cnn_conv3x3(const ArtCnnConv *desc, void *stream);

/* Weight gradient of a 3x3 convolution: dw[n][tap][c] (+)= sum_p dy[p][n] *
 * x[p + d(tap)][c], fp32 [cout][9][cin]. cout a multiple of 8 up to 128, cin
 * a multiple of 16. `workspace` holds per-band partial sums (reduced in a
 * fixed order, so results are deterministic); a few MB suffice. */
typedef struct ArtCnnWgrad {
    int32_t B, H, W, cout, cin;
    const void *dy;
    const void *x;
    float *dw;
    int32_t accumulate;
    void *workspace;
    int64_t workspace_bytes;
    int32_t *err;
} ArtCnnWgrad;
int32_t art_cnn_wgrad3x3(const ArtCnnWgrad *desc, void *stream);

/* Pack fp32 weights w[cout][9][cin] into the bf16 stage layout of
 * art_cnn_conv3x3: [cin/ck][tap column tx][ck/8][tap row ty][n][8] (tap =
 * 3 ty + tx), so that the three tap rows of one tap column form one operand
 * of 3n rows. transpose != 0 packs the
 * backward-data weights of input channels [ci0, ci0 + n) (taps mirrored,
 * reduction over cout). */
int32_t art_cnn_pack_weights(const float *w, int32_t cout, int32_t cin, int32_t transpose, int32_t ci0, int32_t n,
                             int32_t ck, void *out, void *stream);
/* 2x2 average pooling of channels [in_coff, in_coff + C) of [B][H][W][in_cstride] -> [B][H/2][W/2][C]. */
int32_t art_cnn_pool2(const void *in, int32_t B, int32_t H, int32_t W, int32_t C, int32_t in_cstride,
                      int32_t in_coff, void *out, void *stream);
/* Nearest 2x upsampling of [B][H/2][W/2][C] into channels [out_coff, +C) of [B][H][W][out_cstride]. */
int32_t art_cnn_upsample2(const void *in, int32_t B, int32_t H, int32_t W, int32_t C, void *out, int32_t out_cstride,
                          int32_t out_coff, void *stream);
/* out[B][H/2][W/2][C] = (2x2 sums of g[B][H][W][C]) * (act > 0). */
int32_t art_cnn_downsum2_mask(const void *g, int32_t B, int32_t H, int32_t W, int32_t C, const void *act, void *out,
                              void *stream);
/* In place: g = (g + gp[upsampled] / 4) * (act > 0); gp ([B][H/2][W/2][C]) may be NULL; act is channels
 * [act_coff, act_coff + C) of a tensor with act_cstride channels. */
int32_t art_cnn_unpool_add_mask(void *g, const void *gp, int32_t B, int32_t H, int32_t W, int32_t C, const void *act,
                                int32_t act_cstride, int32_t act_coff, void *stream);
/* out[c] (+)= sum over npix pixels of g[p][c] (bf16), fixed reduction order. */
int32_t art_cnn_bias_grad(const void *g, int64_t npix, int32_t C, float *workspace, int64_t workspace_bytes,
                          float *out, int32_t accumulate, void *stream);
/* Network input from B int16 coefficient images (rows of cpitch, images
 * img_stride elements apart, coefficient (v,u) of block (bx,by) at
 * (8by+v, 8bx+u)) and B quantisation tables q[B][64]: dec = IDCT(c q) per
 * block (fp32 [B][H][W]) and feat[B][H0][W0][16] on the network's first
 * level, H0 = ceil(H / 16) * 8, W0 = ceil(W / 16) * 8 (space to depth):
 * level-0 pixel (y, x) holds samples (2y + dy, 2x + dx) as channels
 * 2 dy + dx = dec / 128 and 4 + 2 dy + dx = q / 64 (zero outside the image;
 * channels 8-15 zero). feat may be NULL (decode only). coef, dec and feat
 * 16-byte aligned; cpitch and img_stride multiples of 8. */
int32_t art_cnn_features(const int16_t *coef, int32_t cpitch, int64_t img_stride, const float *q, int32_t B,
                         int32_t H, int32_t W, float *dec, void *feat, void *stream);
/* Prediction pred[B][H][W] = dec + 16 r, r the depth-to-space of channels
 * 0-3 of the level-0 head output r[B][H0][W0][rstride] (inverse of the
 * features' layout); with a target [B][H][W], the gradient of the mean
 * squared error over the B H W samples into grad[B][H0][W0][16] (channels
 * 0-3) and loss_blocks partial sums of the squared error in units of 16 levels. */
int32_t art_cnn_residual(const float *r, int32_t rstride, const float *dec, const float *target, int32_t B,
                         int32_t H, int32_t W, float *pred, void *grad, float *loss_partial, int32_t loss_blocks,
                         void *stream);
/* Self-test of the bounded waits of the tensor-core pipelines: one thread
 * waits on an mbarrier phase that nothing completes, gives up after
 * limit_cycles clock cycles (1 .. 8e9) and writes 1 to the device int *err;
 * the kernel then returns normally. The pipelines' own waits give up after
 * about 4e9 cycles and report through their err flag the same way. */
int32_t art_cnn_wait_selftest(int32_t *err, int64_t limit_cycles, void *stream);
/* One Adam step on n fp32 parameters (step counts from 1). */
int32_t art_cnn_adam(float *w, const float *g, float *m, float *v, int64_t n, float lr, float beta1, float beta2,
                     float eps, int32_t step, void *stream);


/* The warm-start network as a whole (4-level encoder-decoder, 3x3 convs,
 * 32/64/96/128 channels, BF16 weights and activations, FP32 accumulation and
 * master weights). Its first level is the component at half resolution, each
 * pixel carrying a 2x2 cell of samples (art_cnn_features), so the levels are
 * 1/2, 1/4, 1/8 and 1/16 of the component's size. Parameters are one fp32 array of art_net_num_params()
 * values: per layer (e1, e2, e3, e4, d3, d2, d1, head) the weights
 * [cout][9][cin] then the bias [cout]. Inputs are B int16 coefficient images
 * of H x W (multiples of 8; rows of cpitch elements, images img_stride
 * elements apart) with their quantisation tables q[B][64], all on the device. */
int64_t art_net_num_params(void);
int32_t art_net_create(int32_t device, const float *params_host, int64_t nparams, ArtNet **out);
void art_net_destroy(ArtNet *net);
/* Copy the current parameters / the last step's gradients to the host. */
int32_t art_net_params(ArtNet *net, float *host, int64_t n);
int32_t art_net_gradients(ArtNet *net, float *host, int64_t n);
/* Warm start: pred[B][H][W] (fp32, level-shifted samples) = decoded + 16 * residual. */
int32_t art_net_predict(ArtNet *net, const int16_t *coef, int32_t cpitch, int64_t img_stride, const float *q,
                        int32_t B, int32_t H, int32_t W, float *pred, void *stream);
/* Joint 4:2:0 warm start: one pass per image over the luma's level-0 grid
 * (H/2 x W/2), whose pixels each carry a 2x2 luma cell and one sample of each
 * chroma component (feature channels 8-11: decoded Cb / 128, its step / 64,
 * the same for Cr). The head's outputs 4 c + 2 dy + dx are residuals of the
 * full-resolution sample (2 y + dy, 2 x + dx) of component c, over the decoded
 * luma and over the decoded chroma upsampled smoothly (as the learned start
 * upsamples). Luma coefficient images coef_y[B] (H x W, rows of cpitch_y,
 * stride_y apart), chroma coef_c[B][2] (H/2 x W/2, rows of cpitch_c; image b's
 * Cb at coef_c + 2 b stride_c, its Cr stride_c after that), tables q_y[B][64]
 * and q_c[B][2][64], all on the device; H, W multiples of 16.
 * pred[3][B][H][W]: all luma planes, then all Cb, then all Cr. */
int32_t art_net_predict_joint(ArtNet *net, const int16_t *coef_y, int32_t cpitch_y, int64_t stride_y,
                              const int16_t *coef_c, int32_t cpitch_c, int64_t stride_c, const float *q_y,
                              const float *q_c, int32_t B, int32_t H, int32_t W, float *pred, void *stream);
/* One joint training step on the mean squared error (units of 16 levels) of
 * all 3 B H W samples against target[3][B][H][W] (layout of pred above), the
 * luma's weighted (art_net_set_joint_loss). The smoothness and objective terms
 * are not used here. */
int32_t art_net_train_step_joint(ArtNet *net, const int16_t *coef_y, int32_t cpitch_y, int64_t stride_y,
                                 const int16_t *coef_c, int32_t cpitch_c, int64_t stride_c, const float *q_y,
                                 const float *q_c, const float *target, int32_t B, int32_t H, int32_t W, float lr,
                                 float *loss, void *stream);
/* Weight of the luma's squared errors in the joint training loss (default 1;
 * the chroma's weigh 1): loss = (luma_weight sum e_Y^2 + sum e_C^2) / (3 B H W). */
int32_t art_net_set_joint_loss(ArtNet *net, float luma_weight);
/* Training loss: mean squared error (in units of 16 levels) plus
 * smooth_weight times the mean over samples of the squared differences of the
 * error between horizontally and vertically adjacent samples (0, the default,
 * is plain MSE). The smoothness term penalises prediction errors that vary
 * from sample to sample, which the TV/TGV objective penalises most. */
int32_t art_net_set_loss(ArtNet *net, float smooth_weight);
/* Objective term of the training loss: adds lambda / (B H W) times the
 * solver's objective of each sample's prediction after projection onto its
 * quantisation box (per 8x8 block: DCT, clamp to [(c - 1/2) q, (c + 1/2) q],
 * IDCT), with the term weights the solver uses for an nch-channel image with
 * these weight and pweight options: TV 1/sqrt(nch), second-order TGV
 * weight/sqrt(nch), DCT distance pweight * 2 * 255 * sqrt(2)
 * (pipeline_scalar/compute_step.rs:8-72). The gradient is the objective's,
 * taken through the projection. lambda = 0 (the default) turns it off; while
 * it is on, the smoothness term is not used. */
int32_t art_net_set_objective(ArtNet *net, float lambda, float weight, float pweight, int32_t nch);
/* One training step on the mean squared error against target[B][H][W]
 * (in units of 16 levels): forward, backward, then Adam with learning rate
 * lr (lr <= 0: gradients only). *loss (may be NULL) receives the mean loss. */
int32_t art_net_train_step(ArtNet *net, const int16_t *coef, int32_t cpitch, int64_t img_stride, const float *q,
                           const float *target, int32_t B, int32_t H, int32_t W, float lr, float *loss, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* ARTEFACT_B200_H */
