// Device code of the B200 restoration solver.
//
// One solver iteration of backend/artefact-lib/pipeline_scalar (mod.rs:49-75,
// compute_step.rs:8-72) runs as two kernels over 32 x TH pixel tiles of every
// channel at once:
//   k_gradient  FISTA extrapolation y = x_k + f (x_k - x_{k-1}) on the tile and a
//               2-pixel halo; the channel-coupled TV (compute_step_tv.rs:29-93)
//               and TGV (compute_step_tv2.rs:32-136) gradients, written as a
//               gather of the reference's scatter; the DCT-distance gradient
//               (compute_step_prob.rs:5-60) with the lagged coefficients
//               recomputed as the clamped DCT of x_k; writes g and the tile's
//               sum of g^2 per channel; the last tile of an image reduces those
//               sums in a fixed order and stores sigma_c = step / ||g_c||.
//   k_update    y again, x' = y - sigma_c g (compute_step.rs:52-66), then the
//               projection onto the quantisation box per 8x8 coefficient block
//               (compute_projection.rs:8-122): mean-pool for subsampled
//               components, DCT, clamp to [(c-1/2)q, (c+1/2)q], IDCT, add the
//               residual back; writes x_{k+1} over x_{k-1}.
// The 8x8 transforms are Ooura's separable butterflies (utils/dct.rs:30-169).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace art {

constexpr int TILE_W = 32;

struct ChanDev {
    int cw, chh;   // component plane size (rounded_px_w/h)
    int sh, sv;    // sampling factors relative to the max (1 or 2)
    int cpitch;    // int16 elements per row of the coefficient image
    int pad0;
    const int16_t *coef;  // coefficient image: coef(8by+v, 8bx+u) = block (bx,by), index v*8+u
    float alpha_p;        // pweight * 2 * 255 * sqrt(2); 0 disables the DCT-distance term
    float pad1;
};

struct ImgDev {
    int nch, W, H, pitch;  // full-resolution plane size; pitch in floats
    int tiles_x, tiles_y, ntiles, th;
    long long cstride;     // floats between channel planes
    float *x[2];           // state buffers; channel c at x[b] + c * cstride
    float *g;              // gradient planes
    float alpha_tv, alpha_tgv, step, pad;
    float *sigma;          // [4] per channel step / ||g||
    float *partial;        // [ntiles * 4] per-tile sums of g^2
    unsigned int *counter; // tiles done in the current iteration
    ChanDev ch[3];
    float q[3][64];
    float invq2[3][64];
};

// ---------------------------------------------------------------- transforms
#define ART_C1R 0.49039264020161522456f
#define ART_C1I 0.09754516100806413392f
#define ART_C2R 0.46193976625564337806f
#define ART_C2I 0.19134171618254488586f
#define ART_C3R 0.41573480615127261854f
#define ART_C3I 0.27778511650980111237f
#define ART_C4R 0.35355339059327376220f
#define ART_W4R 0.70710678118654752440f

__device__ __forceinline__ void idct8(float *a)
{
    float x0r, x0i, x1r, x1i, x2r, x2i, x3r, x3i, xr, xi;
    x1r = ART_C1R * a[1] + ART_C1I * a[7];
    x1i = ART_C1R * a[7] - ART_C1I * a[1];
    x3r = ART_C3R * a[3] + ART_C3I * a[5];
    x3i = ART_C3R * a[5] - ART_C3I * a[3];
    xr = x1r - x3r;
    xi = x1i + x3i;
    x1r += x3r;
    x3i -= x1i;
    x1i = ART_W4R * (xr + xi);
    x3r = ART_W4R * (xr - xi);
    xr = ART_C2R * a[2] + ART_C2I * a[6];
    xi = ART_C2R * a[6] - ART_C2I * a[2];
    x0r = ART_C4R * (a[0] + a[4]);
    x0i = ART_C4R * (a[0] - a[4]);
    x2r = x0r - xr;
    x2i = x0i - xi;
    x0r += xr;
    x0i += xi;
    a[0] = x0r + x1r;
    a[7] = x0r - x1r;
    a[2] = x0i + x1i;
    a[5] = x0i - x1i;
    a[4] = x2r - x3i;
    a[3] = x2r + x3i;
    a[6] = x2i - x3r;
    a[1] = x2i + x3r;
}

__device__ __forceinline__ void dct8(float *a)
{
    float x0r, x0i, x1r, x1i, x2r, x2i, x3r, x3i, xr, xi;
    x0r = a[0] + a[7];
    x1r = a[0] - a[7];
    x0i = a[2] + a[5];
    x1i = a[2] - a[5];
    x2r = a[4] + a[3];
    x3r = a[4] - a[3];
    x2i = a[6] + a[1];
    x3i = a[6] - a[1];
    xr = x0r + x2r;
    xi = x0i + x2i;
    a[0] = ART_C4R * (xr + xi);
    a[4] = ART_C4R * (xr - xi);
    xr = x0r - x2r;
    xi = x0i - x2i;
    a[2] = ART_C2R * xr - ART_C2I * xi;
    a[6] = ART_C2R * xi + ART_C2I * xr;
    xr = ART_W4R * (x1i - x3i);
    x1i = ART_W4R * (x1i + x3i);
    x3i = x1i - x3r;
    x1i += x3r;
    x3r = x1r - xr;
    x1r += xr;
    a[1] = ART_C1R * x1r - ART_C1I * x1i;
    a[7] = ART_C1R * x1i + ART_C1I * x1r;
    a[3] = ART_C3R * x3r - ART_C3I * x3i;
    a[5] = ART_C3R * x3i + ART_C3I * x3r;
}

// Clamp one row of 8 DCT coefficients (v = row) to their quantisation
// intervals; returns the clamped values in a[] (compute_projection.rs:72-79).
__device__ __forceinline__ void load_coef_row(const int16_t *row, float *c)
{
    const uint4 raw = *reinterpret_cast<const uint4 *>(row);
    const uint32_t w[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        c[2 * i] = (float)(int16_t)(w[i] & 0xffffu);
        c[2 * i + 1] = (float)(int16_t)(w[i] >> 16);
    }
}

// Cell tasks: one 8x8 coefficient block of one channel, covering an
// (8 sh) x (8 sv) full-resolution cell, handled by 8 consecutive lanes.
struct CellTask {
    int c, cx0, cy0;  // channel, cell origin inside the tile (full resolution)
};

template <int TH>
__device__ __forceinline__ int count_tasks(const ImgDev &im)
{
    int n = 0;
    for (int c = 0; c < im.nch; c++) n += (TILE_W / (8 * im.ch[c].sh)) * (TH / (8 * im.ch[c].sv));
    return n;
}

template <int TH>
__device__ __forceinline__ CellTask get_task(const ImgDev &im, int t)
{
    CellTask r{0, 0, 0};
    for (int c = 0; c < im.nch; c++) {
        int sh = im.ch[c].sh, sv = im.ch[c].sv;
        int ncx = TILE_W / (8 * sh), n = ncx * (TH / (8 * sv));
        if (t < n) {
            r.c = c;
            r.cx0 = (t % ncx) * 8 * sh;
            r.cy0 = (t / ncx) * 8 * sv;
            return r;
        }
        t -= n;
    }
    r.c = -1;
    return r;
}

}  // namespace art
