// B200 (sm_100a) restoration solver: kernels and host orchestration behind the
// C ABI declared in include/artefact_b200.h.
//
// Reference: Delnegend/artefact backend/artefact-lib/pipeline_scalar/ (the
// default CLI build). Citations are file:line inside backend/artefact-lib/.
//
// HBM layout (per image):
//   x[2]  two state buffers of nch full-resolution fp32 planes (pitch = W
//         rounded up to 32 floats, 128 B rows); they hold x_k and x_{k-1} and
//         trade roles every iteration (x_{k+1} overwrites x_{k-1} in place).
//   g     nch fp32 gradient planes, same geometry.
//   coef  per channel an int16 "coefficient image": coefficient (v,u) of block
//         (bx,by) sits at row 8by+v, column 8bx+u, so a pixel tile and its
//         coefficient tile coincide (rows padded to 64 elements).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/artefact_b200.h"
#include "art_internal.h"
#include "solver_kernels.cuh"

namespace art {

// ============================================================== kernels ====

template <int TH>
struct GradLayout {
    static constexpr int NT = TILE_W * TH / 4;
    static constexpr int YW = TILE_W + 4, YH = TH + 4;  // y with a 2-pixel halo
    static constexpr int EW = TILE_W + 2, EH = TH + 2;  // per-pixel terms with a 1-pixel ring
    static constexpr int YS = 3 * YH * YW;
    static constexpr int PS = 3 * TH * TILE_W;
    static constexpr int ES = 3 * EH * EW;
    static constexpr int FLOATS = YS + PS + 5 * ES;
    static constexpr size_t BYTES = FLOATS * sizeof(float);
    static_assert(3 * TH * TILE_W <= ES, "x_k tile must fit in the aliased term array");
};

// Gradient of the objective at the FISTA point y (compute_step.rs:8-48), with
// the per-channel sum of squares reduced to sigma_c = step / ||g_c||
// (compute_step.rs:52-58).
template <int TH>
__global__ void __launch_bounds__(TILE_W *TH / 4) k_gradient(const ImgDev *__restrict__ imgs,
                                                            const int2 *__restrict__ tilemap, int parity, float f)
{
    using L = GradLayout<TH>;
    constexpr int NT = L::NT, YW = L::YW, YH = L::YH, EW = L::EW, EH = L::EH;
    extern __shared__ float4 smem4[];
    float *Ys = reinterpret_cast<float *>(smem4);
    float *P = Ys + L::YS;
    float *AU = P + L::PS;
    float *U = AU + L::ES;
    float *BV = U + L::ES;
    float *V = BV + L::ES;
    float *Wt = V + L::ES;
    float *Xc = Wt;  // x_k of the tile; dead before Wt is written
    __shared__ float s_q[3][64], s_iq[3][64];
    __shared__ float s_red[NT / 32][3];
    __shared__ double s_dred[NT / 32][3];
    __shared__ int s_last;

    const int tid = threadIdx.x;
    const int2 tm = tilemap[blockIdx.x];
    const ImgDev &im = imgs[tm.x];
    const int nch = im.nch, W = im.W, H = im.H, pitch = im.pitch;
    const int tx = tm.y % im.tiles_x, ty = tm.y / im.tiles_x;
    const int x0 = tx * TILE_W, y0 = ty * TH;
    const long long cs = im.cstride;
    const float *cur = im.x[parity];
    const float *prev = im.x[parity ^ 1];

    for (int i = tid; i < nch * 64; i += NT) {
        s_q[i >> 6][i & 63] = im.q[i >> 6][i & 63];
        s_iq[i >> 6][i & 63] = im.invq2[i >> 6][i & 63];
    }

    // Phase 0: y = x_k + f (x_k - x_{k-1}) (mod.rs:54-57) on the tile plus a
    // 2-pixel halo, coordinates clamped into the image (replicated edges make
    // the forward differences vanish on the last row/column as the reference's
    // edge tests do, compute_step_tv.rs:105-120).
    for (int i = tid; i < YH * YW; i += NT) {
        const int ey = i / YW, ex = i - ey * YW;
        const int gy = min(max(y0 - 2 + ey, 0), H - 1), gx = min(max(x0 - 2 + ex, 0), W - 1);
        const long long o = (long long)gy * pitch + gx;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (c < nch) {
                const float a = __ldg(cur + c * cs + o), b = __ldg(prev + c * cs + o);
                Ys[c * YH * YW + i] = fmaf(f, a - b, a);
            }
        }
    }
    {
        const int r = tid >> 3, c4 = (tid & 7) * 4;
        const int gy = y0 + r, gx = x0 + c4;
        if (gy < H && gx < W) {
#pragma unroll
            for (int c = 0; c < 3; c++)
                if (c < nch)
                    *reinterpret_cast<float4 *>(&Xc[c * TH * TILE_W + r * TILE_W + c4]) =
                        __ldg(reinterpret_cast<const float4 *>(cur + c * cs + (long long)gy * pitch + gx));
        }
    }
    __syncthreads();

    // DCT-distance gradient (compute_step_prob.rs:5-60): per coefficient block
    // d = (cos - c q) / q^2, IDCT, times alpha_p, replicated to the sh x sv
    // pixels of each component sample. cos is the clamped DCT of the (pooled)
    // x_k, which equals the reference's stored copy (compute_projection.rs:82)
    // up to rounding.
    {
        const int ntask = count_tasks<TH>(im);
        const int lane8 = tid & 7, grp = tid >> 3;
        for (int base = 0; base < ntask; base += NT / 8) {
            const CellTask t = get_task<TH>(im, base + grp);
            const bool act = t.c >= 0 && (x0 + t.cx0) < W && (y0 + t.cy0) < H;
            const int cc = act ? t.c : 0;
            const int sh = im.ch[cc].sh, sv = im.ch[cc].sv;
            const float ap = act ? im.ch[cc].alpha_p : 0.f;
            const bool doprob = act && ap != 0.f;
            float *X = Xc + cc * TH * TILE_W;
            float v[8];
            if (doprob) {
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    float s = 0.f;
                    for (int sy = 0; sy < sv; sy++)
                        for (int sx = 0; sx < sh; sx++)
                            s += X[(t.cy0 + k * sv + sy) * TILE_W + t.cx0 + lane8 * sh + sx];
                    v[k] = s / (float)(sh * sv);
                }
                dct8(v);
#pragma unroll
                for (int k = 0; k < 8; k++) X[(t.cy0 + k * sv) * TILE_W + t.cx0 + lane8 * sh] = v[k];
            }
            __syncwarp();
            if (doprob) {
                float *row = X + (t.cy0 + lane8 * sv) * TILE_W + t.cx0;
#pragma unroll
                for (int u = 0; u < 8; u++) v[u] = row[u * sh];
                dct8(v);
                const ChanDev &cd = im.ch[cc];
                const int bx = (x0 + t.cx0) / (8 * sh), by = (y0 + t.cy0) / (8 * sv);
                float co[8];
                load_coef_row(cd.coef + (long long)(by * 8 + lane8) * cd.cpitch + bx * 8, co);
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const float q = s_q[cc][lane8 * 8 + u];
                    const float lo = (co[u] - 0.5f) * q, hi = (co[u] + 0.5f) * q;
                    const float cl = fminf(fmaxf(v[u], lo), hi);
                    v[u] = (cl - co[u] * q) * s_iq[cc][lane8 * 8 + u];
                }
                idct8(v);
#pragma unroll
                for (int u = 0; u < 8; u++) row[u * sh] = v[u];
            }
            __syncwarp();
            if (act) {
                float *Pc = P + cc * TH * TILE_W;
                if (doprob) {
#pragma unroll
                    for (int k = 0; k < 8; k++) v[k] = X[(t.cy0 + k * sv) * TILE_W + t.cx0 + lane8 * sh];
                    idct8(v);
                } else {
#pragma unroll
                    for (int k = 0; k < 8; k++) v[k] = 0.f;
                }
#pragma unroll
                for (int k = 0; k < 8; k++)
                    for (int sy = 0; sy < sv; sy++)
                        for (int sx = 0; sx < sh; sx++)
                            Pc[(t.cy0 + k * sv + sy) * TILE_W + t.cx0 + lane8 * sh + sx] = ap * v[k];
            }
            __syncwarp();
        }
    }
    __syncthreads();

    // Phase 1: for every pixel q of the tile and a 1-pixel ring, the TV terms
    // (compute_step_tv.rs:98-146) and the TGV terms (compute_step_tv2.rs:42-135),
    // both normalised by the norms coupled over channels. Terms of pixels
    // outside the image are zero, which reproduces the reference's guards.
    {
        const float at = im.alpha_tv, ag = im.alpha_tgv;
        for (int i = tid; i < EH * EW; i += NT) {
            const int ey = i / EW, ex = i - ey * EW;
            const int gxq = x0 - 1 + ex, gyq = y0 - 1 + ey;
            const bool inside = gxq >= 0 && gxq < W && gyq >= 0 && gyq < H;
            float dx[3], dy[3], gxx[3], gyy[3], gs[3];
            float n1 = 0.f, n2 = 0.f;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                dx[c] = dy[c] = gxx[c] = gyy[c] = gs[c] = 0.f;
                if (c < nch) {
                    const float *Y = Ys + c * YH * YW + (ey + 1) * YW + (ex + 1);
                    const float yc = Y[0], yr = Y[1], yl = Y[-1], yd = Y[YW], yu = Y[-YW];
                    const float ydl = Y[YW - 1], yur = Y[-YW + 1];
                    const float ddx = yr - yc, ddy = yd - yc;
                    const float dxl = yc - yl, dyl = ydl - yl, dxu = yur - yu, dyu = yc - yu;
                    const float axx = gxq > 0 ? ddx - dxl : 0.f;
                    const float ayx = gxq > 0 ? ddy - dyl : 0.f;
                    const float ayy = gyq > 0 ? ddy - dyu : 0.f;
                    const float axy = gyq > 0 ? ddx - dxu : 0.f;
                    const float s = 0.5f * (axy + ayx);
                    n1 += ddx * ddx;
                    n1 += ddy * ddy;
                    n2 += ayy * ayy + (2.f * (s * s) + axx * axx);
                    dx[c] = ddx;
                    dy[c] = ddy;
                    gxx[c] = axx;
                    gyy[c] = ayy;
                    gs[c] = s;
                }
            }
            const float inv1 = (inside && n1 > 0.f) ? rsqrtf(n1) : 0.f;
            const float inv2 = (inside && n2 > 0.f) ? rsqrtf(n2) : 0.f;
            const bool intile = ex >= 1 && ex <= TILE_W && ey >= 1 && ey <= TH;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                if (c < nch) {
                    const float a = at * dx[c] * inv1, b = at * dy[c] * inv1;
                    const float u = ag * (gs[c] + gxx[c]) * inv2;
                    const float vv = ag * (gyy[c] + gs[c]) * inv2;
                    const float w = ag * gs[c] * inv2;
                    const int e = c * EH * EW + i;
                    AU[e] = a + u;
                    U[e] = u;
                    BV[e] = b + vv;
                    V[e] = vv;
                    Wt[e] = w;
                    if (intile) P[c * TH * TILE_W + (ey - 1) * TILE_W + (ex - 1)] += -(a + b) - 2.f * (u + vv - w);
                }
            }
        }
    }
    __syncthreads();

    // Phase 2: gather the neighbours' scattered terms, write g, sum g^2.
    float ss[3] = {0.f, 0.f, 0.f};
    {
        const int r = tid >> 3, c4 = (tid & 7) * 4;
        const int gy = y0 + r, gx = x0 + c4;
        const bool valid = gy < H && gx < W;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (c < nch) {
                float go[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int col = c4 + j;
                    const int ep = c * EH * EW + (r + 1) * EW + (col + 1);
                    const float gv = P[c * TH * TILE_W + r * TILE_W + col] + AU[ep - 1] + U[ep + 1] + BV[ep - EW] +
                                     V[ep + EW] - Wt[ep + EW - 1] - Wt[ep - EW + 1];
                    go[j] = gv;
                    ss[c] = fmaf(gv, gv, ss[c]);
                }
                if (valid)
                    *reinterpret_cast<float4 *>(im.g + c * cs + (long long)gy * pitch + gx) =
                        make_float4(go[0], go[1], go[2], go[3]);
                else
                    ss[c] = 0.f;
            }
        }
    }
    // Deterministic block reduction of the three sums.
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float s = ss[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((tid & 31) == 0) s_red[tid >> 5][c] = s;
    }
    __syncthreads();
    if (tid == 0) {
        for (int c = 0; c < 3; c++) {
            float s = 0.f;
            for (int w = 0; w < NT / 32; w++) s += s_red[w][c];
            im.partial[tm.y * 4 + c] = s;
        }
        __threadfence();
        const unsigned prevc = atomicAdd(im.counter, 1u);
        s_last = prevc == (unsigned)(im.ntiles - 1);
    }
    __syncthreads();
    if (s_last) {
        // Last tile of the image: fixed-order fp64 sum of all tile sums.
        __threadfence();
        double acc[3] = {0.0, 0.0, 0.0};
        for (int t = tid; t < im.ntiles; t += NT) {
#pragma unroll
            for (int c = 0; c < 3; c++) acc[c] += (double)__ldcg(im.partial + t * 4 + c);
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double s = acc[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if ((tid & 31) == 0) s_dred[tid >> 5][c] = s;
        }
        __syncthreads();
        if (tid == 0) {
            for (int c = 0; c < 3; c++) {
                double s = 0.0;
                for (int w = 0; w < NT / 32; w++) s += s_dred[w][c];
                const double nrm = sqrt(s);
                im.sigma[c] = nrm > 0.0 ? (float)((double)im.step / nrm) : 0.f;
            }
            atomicExch(im.counter, 0u);
        }
    }
}

template <int TH>
struct UpdLayout {
    static constexpr int NT = TILE_W * TH / 4;
    static constexpr int XS = 3 * TH * TILE_W;
    static constexpr int SCS = 72;  // scratch floats per 8-lane group (64 + bank padding)
    static constexpr int FLOATS = XS + (NT / 8) * SCS;
    static constexpr size_t BYTES = FLOATS * sizeof(float);
};

// Descent step and projection onto the quantisation box
// (compute_step.rs:60-71, compute_projection.rs:8-122).
template <int TH>
__global__ void __launch_bounds__(TILE_W *TH / 4) k_update(const ImgDev *__restrict__ imgs,
                                                          const int2 *__restrict__ tilemap, int ntiles_total,
                                                          int parity, float f, int reverse)
{
    using L = UpdLayout<TH>;
    constexpr int NT = L::NT;
    extern __shared__ float4 smem4[];
    float *Xs = reinterpret_cast<float *>(smem4);
    float *Sc = Xs + L::XS;
    __shared__ float s_q[3][64];

    const int tid = threadIdx.x;
    const int bid = reverse ? ntiles_total - 1 - (int)blockIdx.x : (int)blockIdx.x;
    const int2 tm = tilemap[bid];
    const ImgDev &im = imgs[tm.x];
    const int nch = im.nch, W = im.W, H = im.H, pitch = im.pitch;
    const int tx = tm.y % im.tiles_x, ty = tm.y / im.tiles_x;
    const int x0 = tx * TILE_W, y0 = ty * TH;
    const long long cs = im.cstride;
    const float *cur = im.x[parity];
    float *prev = im.x[parity ^ 1];

    for (int i = tid; i < nch * 64; i += NT) s_q[i >> 6][i & 63] = im.q[i >> 6][i & 63];

    const int r = tid >> 3, c4 = (tid & 7) * 4;
    const int gy = y0 + r, gx = x0 + c4;
    const bool valid = gy < H && gx < W;
    const long long o = (long long)gy * pitch + gx;
    if (valid) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (c < nch) {
                const float sg = im.sigma[c];
                const float4 a = __ldg(reinterpret_cast<const float4 *>(cur + c * cs + o));
                const float4 b = *reinterpret_cast<const float4 *>(prev + c * cs + o);
                const float4 g = __ldg(reinterpret_cast<const float4 *>(im.g + c * cs + o));
                float4 xo;
                xo.x = fmaf(-sg, g.x, fmaf(f, a.x - b.x, a.x));
                xo.y = fmaf(-sg, g.y, fmaf(f, a.y - b.y, a.y));
                xo.z = fmaf(-sg, g.z, fmaf(f, a.z - b.z, a.z));
                xo.w = fmaf(-sg, g.w, fmaf(f, a.w - b.w, a.w));
                *reinterpret_cast<float4 *>(&Xs[c * TH * TILE_W + r * TILE_W + c4]) = xo;
            }
        }
    }
    __syncthreads();

    {
        const int ntask = count_tasks<TH>(im);
        const int lane8 = tid & 7, grp = tid >> 3;
        float *S = Sc + grp * L::SCS;
        for (int base = 0; base < ntask; base += NT / 8) {
            const CellTask t = get_task<TH>(im, base + grp);
            const bool act = t.c >= 0 && (x0 + t.cx0) < W && (y0 + t.cy0) < H;
            const int cc = act ? t.c : 0;
            const int sh = im.ch[cc].sh, sv = im.ch[cc].sv;
            float *X = Xs + cc * TH * TILE_W;
            float v[8];
            if (act) {
                if (sh * sv == 1) {
#pragma unroll
                    for (int k = 0; k < 8; k++) v[k] = X[(t.cy0 + k) * TILE_W + t.cx0 + lane8];
                } else {
                    // compute_projection.rs:18-47: mean over the cell, keep the residual.
                    const float inv = 1.f / (float)(sh * sv);
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        float m = 0.f;
                        for (int sy = 0; sy < sv; sy++)
                            for (int sx = 0; sx < sh; sx++) m += X[(t.cy0 + k * sv + sy) * TILE_W + t.cx0 + lane8 * sh + sx];
                        m *= inv;
                        for (int sy = 0; sy < sv; sy++)
                            for (int sx = 0; sx < sh; sx++) X[(t.cy0 + k * sv + sy) * TILE_W + t.cx0 + lane8 * sh + sx] -= m;
                        v[k] = m;
                    }
                }
                dct8(v);
#pragma unroll
                for (int k = 0; k < 8; k++) S[k * 8 + lane8] = v[k];
            }
            __syncwarp();
            if (act) {
#pragma unroll
                for (int u = 0; u < 8; u++) v[u] = S[lane8 * 8 + u];
                dct8(v);
                const ChanDev &cd = im.ch[cc];
                const int bx = (x0 + t.cx0) / (8 * sh), by = (y0 + t.cy0) / (8 * sv);
                float co[8];
                load_coef_row(cd.coef + (long long)(by * 8 + lane8) * cd.cpitch + bx * 8, co);
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const float q = s_q[cc][lane8 * 8 + u];
                    v[u] = fminf(fmaxf(v[u], (co[u] - 0.5f) * q), (co[u] + 0.5f) * q);
                }
                idct8(v);
#pragma unroll
                for (int u = 0; u < 8; u++) S[lane8 * 8 + u] = v[u];
            }
            __syncwarp();
            if (act) {
#pragma unroll
                for (int k = 0; k < 8; k++) v[k] = S[k * 8 + lane8];
                idct8(v);
                if (sh * sv == 1) {
#pragma unroll
                    for (int k = 0; k < 8; k++) X[(t.cy0 + k) * TILE_W + t.cx0 + lane8] = v[k];
                } else {
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        for (int sy = 0; sy < sv; sy++)
                            for (int sx = 0; sx < sh; sx++) X[(t.cy0 + k * sv + sy) * TILE_W + t.cx0 + lane8 * sh + sx] += v[k];
                }
            }
            __syncwarp();
        }
    }
    __syncthreads();

    if (valid) {
#pragma unroll
        for (int c = 0; c < 3; c++)
            if (c < nch)
                *reinterpret_cast<float4 *>(prev + c * cs + o) =
                    *reinterpret_cast<const float4 *>(&Xs[c * TH * TILE_W + r * TILE_W + c4]);
    }
}

// Initial image (coef.rs:24-92 with the single unboxing of
// pipeline_simd_adaptive/coef.rs:69-95): IDCT of c*q per block, nearest
// upsampling to full resolution, written to both state buffers (aux.rs:62-63).
template <int TH>
__global__ void __launch_bounds__(TILE_W *TH / 4) k_init(const ImgDev *__restrict__ imgs,
                                                        const int2 *__restrict__ tilemap)
{
    constexpr int NT = TILE_W * TH / 4;
    __shared__ float Sc[NT / 8][72];
    const int tid = threadIdx.x;
    const int2 tm = tilemap[blockIdx.x];
    const ImgDev &im = imgs[tm.x];
    const int W = im.W, H = im.H, pitch = im.pitch;
    const int tx = tm.y % im.tiles_x, ty = tm.y / im.tiles_x;
    const int x0 = tx * TILE_W, y0 = ty * TH;
    const int ntask = count_tasks<TH>(im);
    const int lane8 = tid & 7, grp = tid >> 3;
    for (int base = 0; base < ntask; base += NT / 8) {
        const CellTask t = get_task<TH>(im, base + grp);
        const bool act = t.c >= 0 && (x0 + t.cx0) < W && (y0 + t.cy0) < H;
        const int cc = act ? t.c : 0;
        const ChanDev &cd = im.ch[cc];
        const int sh = cd.sh, sv = cd.sv;
        const int bx = (x0 + t.cx0) / (8 * sh), by = (y0 + t.cy0) / (8 * sv);
        float v[8];
        if (act) {
#pragma unroll
            for (int k = 0; k < 8; k++)
                v[k] = (float)cd.coef[(long long)(by * 8 + k) * cd.cpitch + bx * 8 + lane8] * im.q[cc][k * 8 + lane8];
            idct8(v);
#pragma unroll
            for (int k = 0; k < 8; k++) Sc[grp][k * 8 + lane8] = v[k];
        }
        __syncwarp();
        if (act) {
#pragma unroll
            for (int u = 0; u < 8; u++) v[u] = Sc[grp][lane8 * 8 + u];
            idct8(v);
            for (int sy = 0; sy < sv; sy++) {
                const long long rowo = (long long)(y0 + t.cy0 + lane8 * sv + sy) * pitch;
#pragma unroll
                for (int u = 0; u < 8; u++)
                    for (int sx = 0; sx < sh; sx++) {
                        const long long off = cc * im.cstride + rowo + x0 + t.cx0 + u * sh + sx;
                        im.x[0][off] = v[u];
                        im.x[1][off] = v[u];
                    }
            }
        }
        __syncwarp();
    }
}

// Block raster (jpeg/mod.rs:25, zune-jpeg mcu.rs:219-285) -> coefficient
// image, rejecting non-integral or out-of-range float coefficients.
__global__ void k_ingest(const void *__restrict__ src, int type, int bw, long long ncoef, int16_t *__restrict__ dst,
                         int cpitch, unsigned int *err)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncoef) return;
    const long long b = i >> 6;
    const int j = (int)(i & 63);
    const int by = (int)(b / bw), bx = (int)(b % bw);
    int16_t val;
    if (type == ART_COEF_F32) {
        const float x = static_cast<const float *>(src)[i];
        if (!(x == rintf(x)) || x < -32768.f || x > 32767.f) {
            atomicOr(err, 1u);
            val = 0;
        } else {
            val = (int16_t)x;
        }
    } else {
        val = static_cast<const int16_t *>(src)[i];
    }
    dst[(long long)(by * 8 + (j >> 3)) * cpitch + bx * 8 + (j & 7)] = val;
}

// One step of the scalar pipeline's initialisation (coef.rs:29-50): block i
// of the component is dequantised and inverse transformed into linear
// positions [64 i, 64 i + 64) of `a`, then the whole buffer is unboxed into b.
__global__ void k_compat_step(const float *__restrict__ a, float *__restrict__ b, const ImgDev *__restrict__ imgs,
                              int c, int blk, long long nc)
{
    __shared__ float sblk[64];
    const ImgDev &im = imgs[0];
    const ChanDev &cd = im.ch[c];
    const int bw = cd.cw / 8;
    const long long lo = 64LL * blk;
    const long long cta_lo = (long long)blockIdx.x * blockDim.x;
    const bool owner = lo >= cta_lo && lo < cta_lo + blockDim.x;
    if (owner) {
        if (threadIdx.x < 8) {
            const int l = threadIdx.x, bx = blk % bw, by = blk / bw;
            float v[8];
            for (int k = 0; k < 8; k++) v[k] = (float)cd.coef[(long long)(by * 8 + k) * cd.cpitch + bx * 8 + l] * im.q[c][k * 8 + l];
            idct8(v);
            for (int k = 0; k < 8; k++) sblk[k * 8 + l] = v[k];
            __syncwarp(0xffu);
            for (int u = 0; u < 8; u++) v[u] = sblk[l * 8 + u];
            idct8(v);
            __syncwarp(0xffu);
            for (int u = 0; u < 8; u++) sblk[l * 8 + u] = v[u];
        }
        __syncthreads();
    }
    const long long i = cta_lo + threadIdx.x;
    if (i >= nc) return;
    const float val = (i >= lo && i < lo + 64) ? sblk[i - lo] : a[i];
    const long long bb = i >> 6;
    const int k = (int)(i & 63);
    const long long bx = bb % bw, by = bb / bw;
    b[(by * 8 + (k >> 3)) * cd.cw + bx * 8 + (k & 7)] = val;
}

// Nearest upsampling of a component image to both state buffers (coef.rs:69-92).
__global__ void k_upsample(const float *__restrict__ img, const ImgDev *__restrict__ imgs, int c)
{
    const ImgDev &im = imgs[0];
    const ChanDev &cd = im.ch[c];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)im.W * im.H) return;
    const int y = (int)(i / im.W), x = (int)(i % im.W);
    const int cy = min(y / cd.sv, cd.chh - 1), cx = min(x / cd.sh, cd.cw - 1);
    const float v = img[(long long)cy * cd.cw + cx];
    const long long off = c * im.cstride + (long long)y * im.pitch + x;
    im.x[0][off] = v;
    im.x[1][off] = v;
}

// Output stage of Artefact::process (lib.rs:159-211): luma + 128, YCbCr ->
// RGB with unfused multiply-adds, clamp to [0, 255], truncating u8 cast (NaN
// -> 0), crop to the real size. A single channel is replicated to gray RGB.
__device__ __forceinline__ uint8_t to_u8(float v)
{
    if (v != v) return 0;
    v = fminf(fmaxf(v, 0.f), 255.f);
    return (uint8_t)__float2uint_rz(v);
}

__global__ void k_rgb(const float *__restrict__ p0, const float *__restrict__ p1, const float *__restrict__ p2,
                      long long pitch, int nch, int real_w, int real_h, uint8_t *__restrict__ rgb)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)real_w * real_h) return;
    const int y = (int)(i / real_w), x = (int)(i % real_w);
    const long long idx = (long long)y * pitch + x;
    const float yi = __fadd_rn(p0[idx], 128.0f);
    uint8_t r, g, b;
    if (nch == 3) {
        const float cb = p1[idx], cr = p2[idx];
        r = to_u8(__fadd_rn(__fmul_rn(1.402f, cr), yi));
        g = to_u8(__fadd_rn(__fmul_rn(0.71414f, -cr), __fadd_rn(__fmul_rn(0.34414f, -cb), yi)));
        b = to_u8(__fadd_rn(__fmul_rn(1.772f, cb), yi));
    } else {
        r = g = b = to_u8(yi);
    }
    rgb[3 * i + 0] = r;
    rgb[3 * i + 1] = g;
    rgb[3 * i + 2] = b;
}

// ========================================================== host side ======

thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }

namespace {

int fail(int code, const std::string &msg)
{
    set_error(msg);
    return code;
}

#define ART_CUDA(call)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(ART_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
    } while (0)

struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
    int ensure(size_t bytes)
    {
        if (bytes <= n) return ART_OK;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(ART_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        n = bytes;
        return ART_OK;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// FISTA factors of pipeline_scalar/mod.rs:46-61, in fp32 like the reference:
// t' = midpoint(1, sqrt(4 t^2 + 1)), f = (t - 1) / t'.
std::vector<float> fista_factors(uint32_t iterations)
{
    std::vector<float> fs(iterations);
    float term = 1.0f;
    for (uint32_t i = 0; i < iterations; i++) {
        volatile float t2 = term * term;
        volatile float inner = 4.0f * t2 + 1.0f;
        const float next = (float)(((double)1.0f + (double)sqrtf(inner)) / 2.0);
        fs[i] = (term - 1.0f) / next;
        term = next;
    }
    return fs;
}

struct GraphKey {
    int th = 0, ntiles = 0, nimg = 0;
    uint32_t iterations = 0;
    bool timing = false;
    const void *desc = nullptr, *tilemap = nullptr;
    bool operator==(const GraphKey &o) const
    {
        return th == o.th && ntiles == o.ntiles && nimg == o.nimg && iterations == o.iterations &&
               timing == o.timing && desc == o.desc && tilemap == o.tilemap;
    }
};

}  // namespace

}  // namespace art

struct ArtContext {
    int device = 0;
    cudaStream_t stream = nullptr;
    art::DevBuf xbuf, gbuf, coefimg, stage, misc, desc, tilemap, compat, sepplanes, rgb;
    art::ImgDev *h_desc = nullptr;  // pinned host copy of the descriptors
    size_t h_desc_cap = 0;
    std::vector<int2> h_tilemap;
    cudaGraphExec_t exec = nullptr;
    art::GraphKey key;
    bool timing = false;
    std::vector<cudaEvent_t> events;  // [0,1] loop; then 4 per iteration
    uint32_t timed_iterations = 0;
    int last_th = 32;
    int pending_error = 0;
    float *final_planes = nullptr;  // device planes holding the result of the last solve
    int final_pitch = 0;
    long long final_cstride = 0;
};

namespace art {
namespace {

int pick_tile_height(int W, int H)
{
    (void)W;
    (void)H;
    const char *env = getenv("ART_TILE_H");
    if (env && atoi(env) == 16) return 16;
    return 32;
}

// Raises the dynamic shared-memory limit of the tile kernels, once per device.
int configure_kernels(int device)
{
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)done.size() <= device) done.resize(device + 1, 0);
    if (done[device]) return ART_OK;
    int status = ART_OK;
    {
        cudaError_t e = cudaFuncSetAttribute(k_gradient<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)GradLayout<32>::BYTES);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_gradient<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)GradLayout<16>::BYTES);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_update<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)UpdLayout<32>::BYTES);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_update<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)UpdLayout<16>::BYTES);
        if (e != cudaSuccess) {
            set_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
            status = ART_ERR_CUDA;
        }
    }
    if (status == ART_OK) done[device] = 1;
    return status;
}

int validate(uint32_t nch, const ArtChannel *ch, float weight, const float *pweight, uint32_t W, uint32_t H)
{
    if (nch < 1 || nch > 3) return fail(ART_ERR_INVALID_ARGUMENT, "nchannel must be 1, 2 or 3");
    if (!ch || !pweight) return fail(ART_ERR_INVALID_ARGUMENT, "null coefficient or pweight pointer");
    if (W == 0 || H == 0 || W % 8 || H % 8) return fail(ART_ERR_INVALID_ARGUMENT, "max rounded size must be a positive multiple of 8");
    if (W > 65536 || H > 65536) return fail(ART_ERR_INVALID_ARGUMENT, "image larger than 65536 pixels on a side");
    if (!std::isfinite(weight)) return fail(ART_ERR_INVALID_ARGUMENT, "weight is not finite");
    for (uint32_t c = 0; c < nch; c++) {
        const ArtChannel &a = ch[c];
        if (!std::isfinite(pweight[c])) return fail(ART_ERR_INVALID_ARGUMENT, "pweight is not finite");
        if ((a.samp_h != 1 && a.samp_h != 2) || (a.samp_v != 1 && a.samp_v != 2))
            return fail(ART_ERR_INVALID_ARGUMENT, "sampling factors must be 1 or 2");
        if (a.rounded_px_w != a.block_w * 8 || a.rounded_px_h != a.block_h * 8 || a.block_w == 0 || a.block_h == 0)
            return fail(ART_ERR_INVALID_ARGUMENT, "rounded size must equal 8 x block count");
        if (a.rounded_px_w * a.samp_h != W || a.rounded_px_h * a.samp_v != H)
            return fail(ART_ERR_INVALID_ARGUMENT,
                        "component size times sampling factor must equal the max rounded size");
        if (a.coef_type != ART_COEF_F32 && a.coef_type != ART_COEF_I16)
            return fail(ART_ERR_INVALID_ARGUMENT, "unknown coefficient type");
        if (!a.dct_coefs || !a.quant_table) return fail(ART_ERR_INVALID_ARGUMENT, "null coefficient pointer");
        for (int j = 0; j < 64; j++) {
            const float q = a.quant_table[j];
            if (!(q > 0.f) || !(q <= 65535.f))
                return fail(ART_ERR_INVALID_DATA, "quantisation steps must lie in (0, 65535]");
        }
    }
    return ART_OK;
}

}  // namespace

// Lays out buffers for one image, uploads descriptors, ingests coefficients
// and queues the initialisation. `coef_src[c]` is a device pointer.
static int prepare(ArtContext *ctx, uint32_t nch, const ArtChannel *ch, const void *const *coef_src, float weight,
                   const float *pweight, uint32_t iterations, uint32_t W, uint32_t H, int init_mode)
{
    int rc;
    const int th = pick_tile_height((int)W, (int)H);
    const int pitch = (int)align_up(W, 32);
    const size_t rows = align_up(H, 32);
    const long long cstride = (long long)pitch * (long long)rows;
    const int tiles_x = (int)((W + TILE_W - 1) / TILE_W), tiles_y = (int)((H + th - 1) / th);
    const int ntiles = tiles_x * tiles_y;

    if ((rc = ctx->xbuf.ensure(2 * 3 * cstride * sizeof(float)))) return rc;
    if ((rc = ctx->gbuf.ensure(3 * cstride * sizeof(float)))) return rc;
    size_t coef_bytes = 0;
    size_t coef_off[3];
    int cpitch[3];
    for (uint32_t c = 0; c < nch; c++) {
        cpitch[c] = (int)align_up(ch[c].rounded_px_w, 64);
        coef_off[c] = coef_bytes;
        coef_bytes += align_up((size_t)cpitch[c] * ch[c].rounded_px_h * sizeof(int16_t), 256);
    }
    if ((rc = ctx->coefimg.ensure(coef_bytes))) return rc;
    const size_t misc_bytes = align_up(ntiles * 4 * sizeof(float), 256) + 256;
    if ((rc = ctx->misc.ensure(misc_bytes))) return rc;
    if ((rc = ctx->desc.ensure(sizeof(ImgDev)))) return rc;
    if ((rc = ctx->tilemap.ensure(ntiles * sizeof(int2)))) return rc;
    if (!ctx->h_desc) {
        // Pageable on purpose: cudaMemcpyAsync stages it before returning, so
        // the next call may rewrite it while this solve is still queued.
        ctx->h_desc = new ImgDev();
        ctx->h_desc_cap = 1;
    }

    ImgDev &d = *ctx->h_desc;
    memset(&d, 0, sizeof(d));
    d.nch = (int)nch;
    d.W = (int)W;
    d.H = (int)H;
    d.pitch = pitch;
    d.tiles_x = tiles_x;
    d.tiles_y = tiles_y;
    d.ntiles = ntiles;
    d.th = th;
    d.cstride = cstride;
    d.x[0] = static_cast<float *>(ctx->xbuf.p);
    d.x[1] = d.x[0] + 3 * cstride;
    d.g = static_cast<float *>(ctx->gbuf.p);
    // compute_step_tv.rs:130 and compute_step_tv2.rs:88-89, compute_step.rs:47.
    d.alpha_tv = 1.0f / sqrtf((float)nch);
    d.alpha_tgv = (weight / sqrtf(2.0f)) / sqrtf((float)nch);
    // mod.rs:45 and :71.
    const float radius = sqrtf((float)((uint64_t)W * H)) / 2.0f;
    d.step = radius / sqrtf(1.0f + (float)iterations);
    char *misc = static_cast<char *>(ctx->misc.p);
    d.partial = reinterpret_cast<float *>(misc);
    d.sigma = reinterpret_cast<float *>(misc + align_up(ntiles * 4 * sizeof(float), 256));
    d.counter = reinterpret_cast<unsigned *>(d.sigma + 4);
    unsigned *errflag = d.counter + 1;
    for (uint32_t c = 0; c < nch; c++) {
        ChanDev &cd = d.ch[c];
        cd.cw = (int)ch[c].rounded_px_w;
        cd.chh = (int)ch[c].rounded_px_h;
        cd.sh = (int)ch[c].samp_h;
        cd.sv = (int)ch[c].samp_v;
        cd.cpitch = cpitch[c];
        cd.coef = reinterpret_cast<const int16_t *>(static_cast<char *>(ctx->coefimg.p) + coef_off[c]);
        // compute_step.rs:20-31: alpha = pweight * 2 * 255 * sqrt(2).
        cd.alpha_p = pweight[c] * 2.0f * 255.0f * sqrtf(2.0f);
        for (int j = 0; j < 64; j++) {
            const float q = ch[c].quant_table[j];
            d.q[c][j] = q;
            d.invq2[c][j] = 1.0f / (q * q);
        }
    }
    ctx->h_tilemap.resize(ntiles);
    for (int t = 0; t < ntiles; t++) ctx->h_tilemap[t] = make_int2(0, t);

    cudaStream_t s = ctx->stream;
    ART_CUDA(cudaMemcpyAsync(ctx->desc.p, &d, sizeof(ImgDev), cudaMemcpyHostToDevice, s));
    ART_CUDA(cudaMemcpyAsync(ctx->tilemap.p, ctx->h_tilemap.data(), ntiles * sizeof(int2), cudaMemcpyHostToDevice, s));
    ART_CUDA(cudaMemsetAsync(ctx->misc.p, 0, misc_bytes, s));
    const ImgDev *ddesc = static_cast<const ImgDev *>(ctx->desc.p);
    const int2 *dtm = static_cast<const int2 *>(ctx->tilemap.p);
    for (uint32_t c = 0; c < nch; c++) {
        const long long ncoef = (long long)ch[c].block_w * ch[c].block_h * 64;
        const int blocks = (int)((ncoef + 255) / 256);
        k_ingest<<<blocks, 256, 0, s>>>(coef_src[c], (int)ch[c].coef_type, (int)ch[c].block_w, ncoef,
                                        const_cast<int16_t *>(d.ch[c].coef), cpitch[c], errflag);
    }
    if (init_mode == ART_INIT_SCALAR_COMPAT) {
        size_t need = 0;
        for (uint32_t c = 0; c < nch; c++) need = std::max(need, (size_t)ch[c].rounded_px_w * ch[c].rounded_px_h);
        if ((rc = ctx->compat.ensure(2 * need * sizeof(float)))) return rc;
        for (uint32_t c = 0; c < nch; c++) {
            const long long nc = (long long)ch[c].rounded_px_w * ch[c].rounded_px_h;
            float *a = static_cast<float *>(ctx->compat.p), *b = a + need;
            ART_CUDA(cudaMemsetAsync(a, 0, nc * sizeof(float), s));
            const int nb = (int)(ch[c].block_w * ch[c].block_h);
            const int grid = (int)((nc + 255) / 256);
            for (int i = 0; i < nb; i++) {
                k_compat_step<<<grid, 256, 0, s>>>(a, b, ddesc, (int)c, i, nc);
                std::swap(a, b);
            }
            k_upsample<<<(int)(((long long)W * H + 255) / 256), 256, 0, s>>>(a, ddesc, (int)c);
        }
    } else {
        if (th == 16)
            k_init<16><<<ntiles, GradLayout<16>::NT, 0, s>>>(ddesc, dtm);
        else
            k_init<32><<<ntiles, GradLayout<32>::NT, 0, s>>>(ddesc, dtm);
    }
    ART_CUDA(cudaGetLastError());
    ctx->last_th = th;
    ctx->final_planes = d.x[iterations & 1];
    ctx->final_pitch = pitch;
    ctx->final_cstride = cstride;
    return ART_OK;
}

static void launch_iteration(ArtContext *ctx, int th, int ntiles, int it, float f)
{
    const ImgDev *ddesc = static_cast<const ImgDev *>(ctx->desc.p);
    const int2 *dtm = static_cast<const int2 *>(ctx->tilemap.p);
    cudaStream_t s = ctx->stream;
    const int parity = it & 1;
    const bool tm = ctx->timing;
    if (tm) cudaEventRecordWithFlags(ctx->events[2 + 4 * it], s, cudaEventRecordExternal);
    if (th == 16)
        k_gradient<16><<<ntiles, GradLayout<16>::NT, GradLayout<16>::BYTES, s>>>(ddesc, dtm, parity, f);
    else
        k_gradient<32><<<ntiles, GradLayout<32>::NT, GradLayout<32>::BYTES, s>>>(ddesc, dtm, parity, f);
    if (tm) cudaEventRecordWithFlags(ctx->events[3 + 4 * it], s, cudaEventRecordExternal);
    if (tm) cudaEventRecordWithFlags(ctx->events[4 + 4 * it], s, cudaEventRecordExternal);
    if (th == 16)
        k_update<16><<<ntiles, UpdLayout<16>::NT, UpdLayout<16>::BYTES, s>>>(ddesc, dtm, ntiles, parity, f, 1);
    else
        k_update<32><<<ntiles, UpdLayout<32>::NT, UpdLayout<32>::BYTES, s>>>(ddesc, dtm, ntiles, parity, f, 1);
    if (tm) cudaEventRecordWithFlags(ctx->events[5 + 4 * it], s, cudaEventRecordExternal);
}

static int run_iterations(ArtContext *ctx, uint32_t iterations)
{
    const ImgDev &d = *ctx->h_desc;
    const int th = ctx->last_th, ntiles = d.ntiles;
    if (iterations == 0) return ART_OK;
    if (ctx->timing) {
        const size_t need = 2 + 4 * (size_t)iterations;
        while (ctx->events.size() < need) {
            cudaEvent_t e;
            ART_CUDA(cudaEventCreate(&e));
            ctx->events.push_back(e);
        }
    }
    GraphKey key;
    key.th = th;
    key.ntiles = ntiles;
    key.nimg = 1;
    key.iterations = iterations;
    key.timing = ctx->timing;
    key.desc = ctx->desc.p;
    key.tilemap = ctx->tilemap.p;
    cudaStream_t s = ctx->stream;
    if (!ctx->exec || !(ctx->key == key)) {
        if (ctx->exec) {
            cudaGraphExecDestroy(ctx->exec);
            ctx->exec = nullptr;
        }
        const std::vector<float> fs = fista_factors(iterations);
        cudaGraph_t graph;
        ART_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        if (ctx->timing) cudaEventRecordWithFlags(ctx->events[0], s, cudaEventRecordExternal);
        for (uint32_t it = 0; it < iterations; it++) launch_iteration(ctx, th, ntiles, (int)it, fs[it]);
        if (ctx->timing) cudaEventRecordWithFlags(ctx->events[1], s, cudaEventRecordExternal);
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (e != cudaSuccess) return fail(ART_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&ctx->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            ctx->exec = nullptr;
            return fail(ART_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        ctx->key = key;
    }
    ART_CUDA(cudaGraphLaunch(ctx->exec, s));
    ctx->timed_iterations = ctx->timing ? iterations : 0;
    return ART_OK;
}

static int check_errflag(ArtContext *ctx)
{
    unsigned flag = 0;
    const ImgDev &d = *ctx->h_desc;
    ART_CUDA(cudaMemcpy(&flag, d.counter + 1, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (flag) return fail(ART_ERR_INVALID_DATA, "coefficients must be integers in [-32768, 32767]");
    return ART_OK;
}

}  // namespace art

using namespace art;

// ============================================================== C ABI ======

extern "C" {

const char *art_last_error(void) { return art::g_err.c_str(); }

const char *art_version(void) { return "artefact_b200 0.1.0 (sm_100a)"; }

int32_t art_context_create(int32_t device, ArtContext **out)
{
    if (!out) return fail(ART_ERR_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(ART_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (device < 0) ART_CUDA(cudaGetDevice(&device));
    if (device >= ndev) return fail(ART_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    ART_CUDA(cudaSetDevice(device));
    int rc = configure_kernels(device);
    if (rc) return rc;
    std::unique_ptr<ArtContext> ctx(new ArtContext());
    ctx->device = device;
    ART_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    *out = ctx.release();
    return ART_OK;
}

void art_context_destroy(ArtContext *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->exec) cudaGraphExecDestroy(ctx->exec);
    for (auto e : ctx->events) cudaEventDestroy(e);
    ctx->xbuf.release();
    ctx->gbuf.release();
    ctx->coefimg.release();
    ctx->stage.release();
    ctx->misc.release();
    ctx->desc.release();
    ctx->tilemap.release();
    ctx->compat.release();
    ctx->sepplanes.release();
    ctx->rgb.release();
    delete ctx->h_desc;
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int32_t art_context_set_timing(ArtContext *ctx, int32_t enabled)
{
    if (!ctx) return fail(ART_ERR_INVALID_ARGUMENT, "null context");
    ctx->timing = enabled != 0;
    return ART_OK;
}

int32_t art_context_last_timing(ArtContext *ctx, float *loop_ms, float *gradient_ms, float *update_ms,
                                uint32_t *launches)
{
    if (!ctx) return fail(ART_ERR_INVALID_ARGUMENT, "null context");
    if (!ctx->timing || ctx->timed_iterations == 0) return fail(ART_ERR_INVALID_ARGUMENT, "no timed solve recorded");
    ART_CUDA(cudaSetDevice(ctx->device));
    ART_CUDA(cudaStreamSynchronize(ctx->stream));
    float loop = 0, gsum = 0, usum = 0, t;
    ART_CUDA(cudaEventElapsedTime(&loop, ctx->events[0], ctx->events[1]));
    for (uint32_t it = 0; it < ctx->timed_iterations; it++) {
        ART_CUDA(cudaEventElapsedTime(&t, ctx->events[2 + 4 * it], ctx->events[3 + 4 * it]));
        gsum += t;
        ART_CUDA(cudaEventElapsedTime(&t, ctx->events[4 + 4 * it], ctx->events[5 + 4 * it]));
        usum += t;
    }
    if (loop_ms) *loop_ms = loop;
    if (gradient_ms) *gradient_ms = gsum;
    if (update_ms) *update_ms = usum;
    if (launches) *launches = 2 * ctx->timed_iterations;
    return ART_OK;
}

int32_t art_context_compute_device(ArtContext *ctx, uint32_t nchannel, const ArtChannel *coefs, float weight,
                                   const float pweight[3], uint32_t iterations, uint32_t max_w, uint32_t max_h,
                                   float *const *out_planes_device, uint32_t out_pitch, const ArtOptions *opts,
                                   void *stream)
{
    if (!ctx) return fail(ART_ERR_INVALID_ARGUMENT, "null context");
    int rc = validate(nchannel, coefs, weight, pweight, max_w, max_h);
    if (rc) return rc;
    if (!out_planes_device || out_pitch < max_w) return fail(ART_ERR_INVALID_ARGUMENT, "bad output planes");
    for (uint32_t c = 0; c < nchannel; c++)
        if (!out_planes_device[c]) return fail(ART_ERR_INVALID_ARGUMENT, "null output plane");
    const int init_mode = opts ? (int)opts->init_mode : ART_INIT_DECODED;
    if (init_mode != ART_INIT_DECODED && init_mode != ART_INIT_SCALAR_COMPAT)
        return fail(ART_ERR_INVALID_ARGUMENT, "unknown init mode");
    ART_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t user = static_cast<cudaStream_t>(stream);
    cudaEvent_t join = nullptr;
    if (user && user != ctx->stream) {
        // Order the context's stream after the caller's work.
        ART_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
        ART_CUDA(cudaEventRecord(join, user));
        ART_CUDA(cudaStreamWaitEvent(ctx->stream, join, 0));
    }
    const void *src[3];
    for (uint32_t c = 0; c < nchannel; c++) src[c] = coefs[c].dct_coefs;
    rc = prepare(ctx, nchannel, coefs, src, weight, pweight, iterations, max_w, max_h, init_mode);
    if (!rc) rc = run_iterations(ctx, iterations);
    if (!rc) {
        for (uint32_t c = 0; c < nchannel; c++) {
            cudaError_t e = cudaMemcpy2DAsync(out_planes_device[c], (size_t)out_pitch * sizeof(float),
                                              ctx->final_planes + c * ctx->final_cstride,
                                              (size_t)ctx->final_pitch * sizeof(float), (size_t)max_w * sizeof(float),
                                              max_h, cudaMemcpyDeviceToDevice, ctx->stream);
            if (e != cudaSuccess) rc = fail(ART_ERR_CUDA, std::string("output copy: ") + cudaGetErrorString(e));
        }
    }
    if (join) {
        if (!rc) {
            cudaEventRecord(join, ctx->stream);
            cudaStreamWaitEvent(user, join, 0);
        }
        cudaEventDestroy(join);
    }
    return rc;
}

int32_t art_context_synchronize(ArtContext *ctx)
{
    if (!ctx) return fail(ART_ERR_INVALID_ARGUMENT, "null context");
    ART_CUDA(cudaSetDevice(ctx->device));
    ART_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->h_desc) return check_errflag(ctx);
    return ART_OK;
}

static int solve_host(ArtContext *ctx, uint32_t nchannel, const ArtChannel *coefs, float weight,
                      const float pweight[3], uint32_t iterations, uint32_t max_w, uint32_t max_h, int init_mode)
{
    int rc = validate(nchannel, coefs, weight, pweight, max_w, max_h);
    if (rc) return rc;
    if (init_mode != ART_INIT_DECODED && init_mode != ART_INIT_SCALAR_COMPAT)
        return fail(ART_ERR_INVALID_ARGUMENT, "unknown init mode");
    // Host coefficients go through a device staging buffer.
    size_t off[3], total = 0;
    for (uint32_t c = 0; c < nchannel; c++) {
        off[c] = total;
        const size_t es = coefs[c].coef_type == ART_COEF_I16 ? 2 : 4;
        total += align_up((size_t)coefs[c].block_w * coefs[c].block_h * 64 * es, 256);
    }
    if ((rc = ctx->stage.ensure(total))) return rc;
    const void *src[3];
    for (uint32_t c = 0; c < nchannel; c++) {
        const size_t es = coefs[c].coef_type == ART_COEF_I16 ? 2 : 4;
        char *dst = static_cast<char *>(ctx->stage.p) + off[c];
        ART_CUDA(cudaMemcpyAsync(dst, coefs[c].dct_coefs, (size_t)coefs[c].block_w * coefs[c].block_h * 64 * es,
                                 cudaMemcpyHostToDevice, ctx->stream));
        src[c] = dst;
    }
    rc = prepare(ctx, nchannel, coefs, src, weight, pweight, iterations, max_w, max_h, init_mode);
    if (!rc) rc = run_iterations(ctx, iterations);
    return rc;
}

int32_t art_context_compute(ArtContext *ctx, uint32_t nchannel, const ArtChannel *coefs, float weight,
                            const float pweight[3], uint32_t iterations, uint32_t max_w, uint32_t max_h,
                            float *const *out_planes, const ArtOptions *opts)
{
    if (!ctx) return fail(ART_ERR_INVALID_ARGUMENT, "null context");
    if (!out_planes) return fail(ART_ERR_INVALID_ARGUMENT, "null output planes");
    for (uint32_t c = 0; c < nchannel && c < 3; c++)
        if (!out_planes[c]) return fail(ART_ERR_INVALID_ARGUMENT, "null output plane");
    ART_CUDA(cudaSetDevice(ctx->device));
    const int init_mode = opts ? (int)opts->init_mode : ART_INIT_DECODED;
    int rc = solve_host(ctx, nchannel, coefs, weight, pweight, iterations, max_w, max_h, init_mode);
    if (rc) {
        cudaStreamSynchronize(ctx->stream);
        return rc;
    }
    for (uint32_t c = 0; c < nchannel; c++)
        ART_CUDA(cudaMemcpy2DAsync(out_planes[c], (size_t)max_w * sizeof(float),
                                   ctx->final_planes + c * ctx->final_cstride, (size_t)ctx->final_pitch * sizeof(float),
                                   (size_t)max_w * sizeof(float), max_h, cudaMemcpyDeviceToHost, ctx->stream));
    ART_CUDA(cudaStreamSynchronize(ctx->stream));
    return check_errflag(ctx);
}

int32_t art_context_process(ArtContext *ctx, uint32_t nchannel, const ArtChannel *coefs, const float weight[3],
                            const float pweight[3], const uint32_t iterations[3], int32_t separate, uint32_t real_w,
                            uint32_t real_h, uint8_t *rgb_out, const ArtOptions *opts)
{
    if (!ctx) return fail(ART_ERR_INVALID_ARGUMENT, "null context");
    if (!coefs || !weight || !pweight || !iterations) return fail(ART_ERR_INVALID_ARGUMENT, "null argument");
    if (nchannel < 1 || nchannel > 4) return fail(ART_ERR_INVALID_ARGUMENT, "nchannel must be 1 to 4");
    ART_CUDA(cudaSetDevice(ctx->device));
    const int init_mode = opts ? (int)opts->init_mode : ART_INIT_DECODED;
    // lib.rs:108-116: max rounded size over components.
    uint32_t W = 0, H = 0;
    for (uint32_t c = 0; c < nchannel; c++) {
        W = std::max(W, coefs[c].rounded_px_w);
        H = std::max(H, coefs[c].rounded_px_h);
    }
    if (real_w == 0 || real_h == 0 || real_w > W || real_h > H)
        return fail(ART_ERR_INVALID_ARGUMENT, "real size must be positive and within the rounded size");
    const uint32_t nout = nchannel == 3 ? 3 : 1;
    const float *planes[3] = {nullptr, nullptr, nullptr};
    long long pitch = 0;
    int rc;
    if (nchannel == 3 && !separate) {
        // lib.rs:122-132: joint solve with weight[0], pweight, iterations[0].
        rc = solve_host(ctx, 3, coefs, weight[0], pweight, iterations[0], W, H, init_mode);
        if (rc) {
            cudaStreamSynchronize(ctx->stream);
            return rc;
        }
        for (int c = 0; c < 3; c++) planes[c] = ctx->final_planes + c * ctx->final_cstride;
        pitch = ctx->final_pitch;
    } else {
        // lib.rs:133-153: each component alone, compute(1, [coef], weight[c], pweight, iterations[c]),
        // so every component uses pweight[0].
        const size_t plane = (size_t)W * H;
        if ((rc = ctx->sepplanes.ensure(nout * plane * sizeof(float)))) return rc;
        for (uint32_t c = 0; c < nchannel; c++) {
            const float w = weight[c < 3 ? c : 2];
            const uint32_t its = iterations[c < 3 ? c : 2];
            rc = solve_host(ctx, 1, &coefs[c], w, pweight, its, W, H, init_mode);
            if (rc) {
                cudaStreamSynchronize(ctx->stream);
                return rc;
            }
            if (c < nout) {
                float *dst = static_cast<float *>(ctx->sepplanes.p) + c * plane;
                ART_CUDA(cudaMemcpy2DAsync(dst, (size_t)W * sizeof(float), ctx->final_planes,
                                           (size_t)ctx->final_pitch * sizeof(float), (size_t)W * sizeof(float), H,
                                           cudaMemcpyDeviceToDevice, ctx->stream));
                planes[c] = dst;
            }
            ART_CUDA(cudaStreamSynchronize(ctx->stream));
            if ((rc = check_errflag(ctx))) return rc;
        }
        pitch = W;
    }
    if (rgb_out) {
        const size_t nbytes = (size_t)real_w * real_h * 3;
        if ((rc = ctx->rgb.ensure(nbytes))) return rc;
        const long long n = (long long)real_w * real_h;
        k_rgb<<<(int)((n + 255) / 256), 256, 0, ctx->stream>>>(planes[0], planes[1], planes[2], pitch, (int)nout,
                                                               (int)real_w, (int)real_h,
                                                               static_cast<uint8_t *>(ctx->rgb.p));
        ART_CUDA(cudaGetLastError());
        ART_CUDA(cudaMemcpyAsync(rgb_out, ctx->rgb.p, nbytes, cudaMemcpyDeviceToHost, ctx->stream));
    }
    ART_CUDA(cudaStreamSynchronize(ctx->stream));
    return check_errflag(ctx);
}

}  // extern "C"

namespace art {
namespace {
// One default context per (thread, device): the reference's rayon workers
// each get their own stream and buffers.
struct ThreadContexts {
    std::vector<ArtContext *> byDevice;
    ~ThreadContexts()
    {
        for (auto c : byDevice)
            if (c) art_context_destroy(c);
    }
};
thread_local ThreadContexts t_ctx;
}  // namespace
}  // namespace art

extern "C" int32_t art_compute(uint32_t nchannel, const ArtChannel *coefs, float weight, const float pweight[3],
                               uint32_t iterations, uint32_t max_w, uint32_t max_h, uint64_t max_count,
                               float *const *out_planes, const ArtOptions *opts)
{
    if ((uint64_t)max_w * max_h != max_count)
        return fail(ART_ERR_INVALID_ARGUMENT, "max_rounded_px_count must equal width x height");
    int device = opts ? opts->device : -1;
    if (device < 0) {
        cudaError_t e = cudaGetDevice(&device);
        if (e != cudaSuccess) return fail(ART_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    }
    if (device < 0 || device > 1024) return fail(ART_ERR_INVALID_ARGUMENT, "bad device ordinal");
    auto &v = t_ctx.byDevice;
    if ((int)v.size() <= device) v.resize(device + 1, nullptr);
    if (!v[device]) {
        int rc = art_context_create(device, &v[device]);
        if (rc) return rc;
    }
    return art_context_compute(v[device], nchannel, coefs, weight, pweight, iterations, max_w, max_h, out_planes,
                               opts);
}
