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
    uint32_t init_mode; /* ART_INIT_DECODED (default) or ART_INIT_SCALAR_COMPAT */
    int32_t device;     /* CUDA device ordinal, -1 = current device */
    uint32_t reserved[6];
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
 * Autotuner. Times both gradient-sweep variants (0 = narrow, one column per
 * lane; 1 = wide, two columns per lane on packed FP32x2 arithmetic) at each
 * strip height (16, 32, 64, 128 rows) on a deterministic synthetic image of
 * the given geometry (`iterations` steps, 0 = 10) and caches the fastest pair
 * for the geometry's bucket (channel count, sampling, width and height rounded
 * up to powers of two); later solves of images in that bucket use it. The two
 * variants sum the same terms in a different order (results agree to fp32
 * rounding), and each is deterministic. art_context_tune_cache saves
 * (save != 0) or loads the cache as a text file of
 * "<bucket> <variant> <rows>" lines. Either output pointer may be NULL.
 */
int32_t art_context_autotune(ArtContext *ctx, uint32_t nchannel, const uint32_t *samp_h, const uint32_t *samp_v,
                             uint32_t max_rounded_px_w, uint32_t max_rounded_px_h, uint32_t iterations,
                             uint32_t *variant_out, uint32_t *strip_rows_out);
int32_t art_context_tune_cache(ArtContext *ctx, const char *path, int32_t save);

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
 * imply. Same kernels and results as art_context_compute_device, but every
 * scratch buffer comes from one fixed 64 MiB array in device memory that the
 * library holds on every GPU it is loaded on until the process exits; images
 * that need more (about 1 megapixel per channel) are rejected with
 * ART_ERR_INVALID_ARGUMENT. dct_coefs and out_planes_device are device
 * pointers, quant_table a host pointer; work runs on `stream` (NULL = legacy
 * default stream) and the call returns when it is done. The first call on a
 * device resolves the array's address there. All calls share the array, so
 * calls whose GPU work overlaps race; each call clears what must start at zero.
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

#ifdef __cplusplus
}
#endif

#endif /* ARTEFACT_B200_H */
