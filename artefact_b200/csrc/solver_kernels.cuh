// Device code of the B200 restoration solver.
//
// One solver iteration of backend/artefact-lib/pipeline_scalar (mod.rs:49-75,
// compute_step.rs:8-72) runs as two kernels:
//   k_grad_sweep  one warp walks down a 28-column strip of all channels (32
//                 lanes with a 2-column halo) of the FISTA point y_k, keeping a
//                 rolling window in registers: channel-coupled TV (compute_step_tv.rs:29-93)
//                 and TGV (compute_step_tv2.rs:32-136) gradients written as a
//                 gather of the reference's scatter (horizontal neighbours by
//                 warp shuffles), plus the DCT-distance gradient plane the last
//                 projection left (compute_step_prob.rs:5-60); writes g and
//                 sums g^2 per channel; the last block of an image reduces the
//                 sums in a fixed order and stores sigma_c = step / ||g_c||.
//   k_project     eight lanes per 8x8 coefficient block (lane = block row; a
//                 16x16 / 16x8 cell of full-resolution pixels for subsampled
//                 components), transposes through shared memory:
//                 x' = y_k - sigma_c g (compute_step.rs:60-66), mean pooling,
//                 DCT, clamp to [(c-1/2)q, (c+1/2)q], IDCT, residual
//                 (compute_projection.rs:8-122); writes x_{k+1} over x_k and the
//                 next FISTA point y_{k+1} = x_{k+1} + f_{k+1} (x_{k+1} - x_k)
//                 (mod.rs:50-59) over y_k, and, from the clamped coefficients it
//                 keeps (the reference's cos, compute_projection.rs:82), the next
//                 DCT-distance gradient alpha_p * IDCT((cos - c q) / q^2).
// The 8x8 transforms are Ooura's separable butterflies (utils/dct.rs:30-169).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace art {

struct ChanDev {
    int cw, chh;   // component plane size (rounded_px_w/h)
    int sh, sv;    // sampling factors relative to the max (1 or 2)
    int cpitch;    // int16 elements per row of the coefficient image
    int ppitch;    // floats per row of the DCT-distance gradient plane
    const int16_t *coef;  // coefficient image: coef(8by+v, 8bx+u) = block (bx,by), index v*8+u
    float *P;             // alpha_p * IDCT((cos - c q) / q^2) at component resolution
    float alpha_p;        // pweight * 2 * 255 * sqrt(2); 0 disables the DCT-distance term
    float pad1;
};

struct ImgDev {
    int nch, W, H, pitch;  // full-resolution plane size; pitch in floats
    int strips_x, strips_y, nstrips, strip_rows;  // gradient sweep strips (28 or 60 columns x strip_rows)
    int ncta;              // gradient-sweep blocks of this image
    int sweep_kind;        // 0 = narrow sweep (one column per lane), 1 = wide (two, packed FP32x2), 2 = quad (four)
    long long cstride;     // floats between channel planes
    float *x;              // iterate x_k; channel c at x + c * cstride
    float *y;              // FISTA point y_k = x_k + f_k (x_k - x_{k-1})
    float *g;              // gradient planes
    float alpha_tv, alpha_tgv, step, pad;
    float *sigma;          // [4] per channel step / ||g||
    float *partial;        // [ncta * 4] per-block sums of g^2
    unsigned int *counter; // sweep blocks done in the current iteration
    ChanDev ch[3];
    float q[3][64];
    float invq2[3][64];
};

// Resident blocks per SM the sweeps' register counts must allow (wide: 3 x 4
// warps at <= 168 registers; narrow: 2 x 8 warps). Tighter caps spill and
// measured slower on 1080p and 24 MP.
constexpr int SWEEP_MIN_BLOCKS = 3;
constexpr int SWEEP_MIN_BLOCKS_N = 2;
constexpr int SWEEP_PF = 4;       // wide sweep: y rows loaded ahead of use
constexpr int SWEEP_PPF = 3;      // wide sweep: DCT-distance rows loaded ahead of use
constexpr int SWEEP_OUT = 60;     // wide sweep: output columns per warp strip (32 lanes x 2 columns, 2 of halo each side)
constexpr int SWEEP_WARPS = 4;    // wide sweep: warps (strips) per block
constexpr int SWEEP_PF_N = 3;     // narrow sweep: y rows loaded ahead of use
constexpr int SWEEP_PPF_N = 2;    // narrow sweep: DCT-distance rows loaded ahead of use
constexpr int SWEEP_OUT_N = 28;   // narrow sweep: 32 lanes x 1 column, 2 of halo each side
constexpr int SWEEP_WARPS_N = 8;  // narrow sweep: warps per block
constexpr int SWEEP_OUT_Q = 120;  // quad sweep: output columns per warp strip (32 lanes x 4 columns, 4 of halo each side)
constexpr int SWEEP_WARPS_Q = 4;  // quad sweep: warps per block
constexpr int SWEEP_MIN_BLOCKS_Q = 2;
constexpr int SWEEP_PF_Q = 2;     // quad sweep: y rows loaded ahead of use
constexpr int SWEEP_PPF_Q = 1;    // quad sweep: DCT-distance rows loaded ahead of use
constexpr int PROJ_WARPS = 4;   // warps per projection block (4 coefficient blocks per warp)

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

// The 8 quantised coefficients of one block row (int16) as floats.
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

// 2-D transforms of a register-resident 8x8 block, columns first then rows,
// as dct8x8s / idct8x8s do (utils/dct.rs:30-169).
__device__ __forceinline__ void dct8x8_regs(float *a)
{
#pragma unroll
    for (int j = 0; j < 8; j++) {
        float v[8];
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = a[k * 8 + j];
        dct8(v);
#pragma unroll
        for (int k = 0; k < 8; k++) a[k * 8 + j] = v[k];
    }
#pragma unroll
    for (int j = 0; j < 8; j++) dct8(a + j * 8);
}

__device__ __forceinline__ void idct8x8_regs(float *a)
{
#pragma unroll
    for (int j = 0; j < 8; j++) {
        float v[8];
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = a[k * 8 + j];
        idct8(v);
#pragma unroll
        for (int k = 0; k < 8; k++) a[k * 8 + j] = v[k];
    }
#pragma unroll
    for (int j = 0; j < 8; j++) idct8(a + j * 8);
}

// Packed FP32x2 arithmetic (one instruction for two lanes' worth of work).
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b)
{
    unsigned long long ua, ub, r;
    ua = (unsigned long long)__float_as_uint(a.x) | ((unsigned long long)__float_as_uint(a.y) << 32);
    ub = (unsigned long long)__float_as_uint(b.x) | ((unsigned long long)__float_as_uint(b.y) << 32);
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(ua), "l"(ub));
    return make_float2(__uint_as_float((unsigned)r), __uint_as_float((unsigned)(r >> 32)));
}

// 8x8 transpose among the 8 lanes (r = lane & 7) of a lane group through a
// 8x9 shared scratch: a lane holding row r leaves holding column r, and back.
__device__ __forceinline__ void transpose8(float (*T)[9], int r, float *v)
{
    __syncwarp();
#pragma unroll
    for (int u = 0; u < 8; u++) T[r][u] = v[u];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = T[k][r];
}

// Asynchronous global -> shared copies of 16 bytes (L2 only), and their fence.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

}  // namespace art
