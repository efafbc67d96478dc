/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the artefact restoration solver.
 *
 * Only tests, the smoke check and the CPU-baseline leg of the benchmark load
 * this library, and only as the checker. The product never links it.
 *
 * Parity status: UNPINNED against the reference's own outputs. The reference
 * (Delnegend/artefact, backend/artefact-lib, Rust) has no solver tests, no golden
 * vectors and cannot be compiled here (no Rust toolchain). This file restates
 * backend/artefact-lib/pipeline_scalar/ operation by operation; it is pinned by
 * DCT known-answer tests, a finite-difference check of the gradient against the
 * objective below, and agreement between its fp32 and fp64 twins.
 *
 * Build: oracle/Makefile (gcc -O3 -ffp-contract=off, single-threaded).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* One JPEG component as the solver receives it: jpeg/mod.rs:8-27 (Coefficient). */
typedef struct {
    uint32_t rounded_px_w, rounded_px_h; /* component plane, multiples of 8 */
    uint32_t block_w, block_h;           /* rounded / 8 */
    uint32_t samp_h, samp_v;             /* max sampling / component sampling: 1 or 2 */
    const float *dct_coefs;              /* block_w*block_h*64, block raster, natural order */
    const float *quant_table;            /* 64, natural order */
} oracle_channel;

#define R float
#define PFX(n) oracle_f32_##n
#define SQRT sqrtf
#define KLIT(v) v##f
#include "oracle_body.inc"
#undef R
#undef PFX
#undef SQRT
#undef KLIT

#define R double
#define PFX(n) oracle_f64_##n
#define SQRT sqrt
#define KLIT(v) v
#include "oracle_body.inc"
#undef R
#undef PFX
#undef SQRT
#undef KLIT

/*
 * Objective of the solver, evaluated in fp64 on final float planes.
 * The reference never evaluates it (compute_step.rs:39-48 drops the values of
 * compute_step_tv.rs:9-26 and compute_step_tv2.rs:4-29), so it is defined here
 * as the function whose gradient the reference's step follows:
 *   E = sum_p a1 * n1(p) + sum_p a2 * n2(p)
 *     + sum_c (alpha_c * sh * sv / 2) * sum_blocks sum_j ((X_j - c_j q_j) / q_j)^2
 * with a1 = 1/sqrt(nch), a2 = (weight/sqrt(2))/sqrt(nch), alpha_c =
 * pweight_c * 2 * 255 * sqrt(2), n1/n2 the channel-coupled TV and TGV norms of
 * compute_step_tv.rs:45-69 and compute_step_tv2.rs:46-86, and X the DCT of the
 * (mean-pooled, for subsampled components) channel. The factor sh*sv accounts
 * for the prob gradient being replicated to every full-resolution pixel of a
 * subsampled cell without a 1/(sh*sv) factor (compute_step_prob.rs:43-55).
 * terms[0..2] receive the TV, TGV and prob parts (may be NULL).
 */
static void pool_plane(const double *plane, uint32_t W, const oracle_channel *c, double *out)
{
    uint32_t rw = c->rounded_px_w, rh = c->rounded_px_h, sh = c->samp_h, sv = c->samp_v;
    for (uint32_t cy = 0; cy < rh; cy++)
        for (uint32_t cx = 0; cx < rw; cx++) {
            double m = 0;
            for (uint32_t sy = 0; sy < sv; sy++)
                for (uint32_t sx = 0; sx < sh; sx++) m += plane[(size_t)(cy * sv + sy) * W + cx * sh + sx];
            out[(size_t)cy * rw + cx] = m / (double)(sh * sv);
        }
}

double oracle_objective_f64(uint32_t nch, const oracle_channel *chs, float weight, const float *pweight,
                            uint32_t W, uint32_t H, const double *const *planes, double *terms)
{
    double a1 = 1.0 / sqrt((double)nch);
    double a2 = ((double)weight / sqrt(2.0)) / sqrt((double)nch);
    double tv = 0, tv2 = 0, prob = 0;
    for (uint32_t y = 0; y < H; y++)
        for (uint32_t x = 0; x < W; x++) {
            double n1 = 0, n2 = 0;
            size_t p = (size_t)y * W + x;
            for (uint32_t c = 0; c < nch; c++) {
                const double *f = planes[c];
#define DX(xx, yy) ((xx) < W - 1 ? (double)f[(size_t)(yy) * W + (xx) + 1] - (double)f[(size_t)(yy) * W + (xx)] : 0.0)
#define DY(xx, yy) ((yy) < H - 1 ? (double)f[(size_t)((yy) + 1) * W + (xx)] - (double)f[(size_t)(yy) * W + (xx)] : 0.0)
                double dx = DX(x, y), dy = DY(x, y);
                n1 += dx * dx + dy * dy;
                double gxx = 0, gyx = 0, gyy = 0, gxy = 0;
                if (x > 0) { gxx = dx - DX(x - 1, y); gyx = dy - DY(x - 1, y); }
                if (y > 0) { gyy = dy - DY(x, y - 1); gxy = dx - DX(x, y - 1); }
                double s = 0.5 * (gxy + gyx);
                n2 += gyy * gyy + 2.0 * s * s + gxx * gxx;
#undef DX
#undef DY
            }
            (void)p;
            tv += a1 * sqrt(n1);
            tv2 += a2 * sqrt(n2);
        }
    for (uint32_t c = 0; c < nch; c++) {
        const oracle_channel *ch = &chs[c];
        if (pweight[c] == 0.0f) continue;
        double alpha = (double)pweight[c] * 2.0 * 255.0 * sqrt(2.0) * (double)(ch->samp_h * ch->samp_v);
        size_t nc = (size_t)ch->rounded_px_w * ch->rounded_px_h;
        double *pool = (double *)malloc(nc * sizeof(double));
        pool_plane(planes[c], W, ch, pool);
        double acc = 0, blk[64];
        for (uint32_t by = 0; by < ch->block_h; by++)
            for (uint32_t bx = 0; bx < ch->block_w; bx++) {
                for (int j = 0; j < 64; j++)
                    blk[j] = pool[(size_t)(by * 8 + j / 8) * ch->rounded_px_w + bx * 8 + j % 8];
                oracle_f64_dct8x8(blk);
                size_t bi = (size_t)by * ch->block_w + bx;
                for (int j = 0; j < 64; j++) {
                    double q = ch->quant_table[j];
                    double d = (blk[j] - (double)ch->dct_coefs[bi * 64 + j] * q) / q;
                    acc += d * d;
                }
            }
        free(pool);
        prob += 0.5 * alpha * acc;
    }
    if (terms) { terms[0] = tv; terms[1] = tv2; terms[2] = prob; }
    return tv + tv2 + prob;
}

static double **widen(uint32_t nch, size_t n, const float *const *planes)
{
    double **p = (double **)calloc(nch, sizeof(double *));
    for (uint32_t c = 0; c < nch; c++) {
        p[c] = (double *)malloc(n * sizeof(double));
        for (size_t i = 0; i < n; i++) p[c][i] = planes[c][i];
    }
    return p;
}

static void free_widened(uint32_t nch, double **p)
{
    for (uint32_t c = 0; c < nch; c++) free(p[c]);
    free(p);
}

double oracle_objective(uint32_t nch, const oracle_channel *chs, float weight, const float *pweight, uint32_t W,
                        uint32_t H, const float *const *planes, double *terms)
{
    double **p = widen(nch, (size_t)W * H, planes);
    double e = oracle_objective_f64(nch, chs, weight, pweight, W, H, (const double *const *)p, terms);
    free_widened(nch, p);
    return e;
}

/*
 * Feasibility of final planes: the largest distance (in coefficient units) by
 * which an fp64 DCT coefficient of an output block (mean-pooled for subsampled
 * components) lies outside [(c - 1/2) q, (c + 1/2) q], the box of
 * compute_projection.rs:72-79. Returns 0 when every coefficient is inside.
 */
double oracle_feasibility(uint32_t nch, const oracle_channel *chs, uint32_t W, uint32_t H,
                          const float *const *planes)
{
    double worst = 0;
    double **wide = widen(nch, (size_t)W * H, planes);
    for (uint32_t c = 0; c < nch; c++) {
        const oracle_channel *ch = &chs[c];
        size_t nc = (size_t)ch->rounded_px_w * ch->rounded_px_h;
        double *pool = (double *)malloc(nc * sizeof(double));
        pool_plane(wide[c], W, ch, pool);
        double blk[64];
        for (uint32_t by = 0; by < ch->block_h; by++)
            for (uint32_t bx = 0; bx < ch->block_w; bx++) {
                for (int j = 0; j < 64; j++)
                    blk[j] = pool[(size_t)(by * 8 + j / 8) * ch->rounded_px_w + bx * 8 + j % 8];
                oracle_f64_dct8x8(blk);
                size_t bi = (size_t)by * ch->block_w + bx;
                for (int j = 0; j < 64; j++) {
                    double q = ch->quant_table[j], cc = ch->dct_coefs[bi * 64 + j];
                    double lo = (cc - 0.5) * q, hi = (cc + 0.5) * q, v = blk[j];
                    double viol = v < lo ? lo - v : (v > hi ? v - hi : 0.0);
                    if (viol > worst) worst = viol;
                }
            }
        free(pool);
    }
    free_widened(nch, wide);
    return worst;
}

/* Rust `f32 as u8` after clamp(0, 255): truncation toward zero, NaN -> 0. */
static uint8_t to_u8(float v)
{
    if (v != v) return 0;
    if (v < 0.0f) v = 0.0f;
    if (v > 255.0f) v = 255.0f;
    return (uint8_t)v;
}

/*
 * Output stage of Artefact::process, lib.rs:159-211: luma + 128, YCbCr -> RGB
 * with unfused multiply-adds and truncating u8 casts, crop to the real size
 * from row stride W; a single channel is replicated to RGB.
 * rgb receives real_h * real_w * 3 bytes.
 */
void oracle_rgb(uint32_t nch, uint32_t W, uint32_t real_w, uint32_t real_h, const float *const *planes,
                uint8_t *rgb)
{
    for (uint32_t i = 0; i < real_h; i++)
        for (uint32_t j = 0; j < real_w; j++) {
            size_t idx = (size_t)i * W + j, o = ((size_t)i * real_w + j) * 3;
            float yi = planes[0][idx] + 128.0f;
            if (nch == 3) {
                float cb = planes[1][idx], cr = planes[2][idx];
                rgb[o + 0] = to_u8(1.402f * cr + yi);
                rgb[o + 1] = to_u8(0.71414f * -cr + (0.34414f * -cb + yi));
                rgb[o + 2] = to_u8(1.772f * cb + yi);
            } else {
                uint8_t g = to_u8(yi);
                rgb[o + 0] = g;
                rgb[o + 1] = g;
                rgb[o + 2] = g;
            }
        }
}
