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
#include <type_traits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <array>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/artefact_b200.h"
#include "art_internal.h"
#include "solver_kernels.cuh"

namespace art {

// ============================================================== kernels ====

// Gradient of the objective at the FISTA point y_k (compute_step.rs:8-48) and
// the per-channel sums of squares reduced to sigma_c = step / ||g_c||
// (compute_step.rs:52-58). One warp per strip of SWEEP_OUT output columns and
// strip_rows rows; lane L holds the column pair xs - 2 + 2L, xs - 1 + 2L as a
// float2 and the arithmetic runs on packed FP32x2 instructions. Lanes 0..31
// form the per-pixel terms, lanes 1..30 write g. Rows and columns outside the
// image are read clamped (replicated edges make the reference's last-row and
// last-column forward differences vanish, compute_step_tv.rs:105-120) and
// their terms are zero, which reproduces the reference's scatter guards. Rows
// are prefetched two ahead of use.
template <int NCH>
__global__ void __launch_bounds__(SWEEP_WARPS * 32, SWEEP_MIN_BLOCKS) k_grad_sweep(const ImgDev *__restrict__ imgs,
                                                                 const int2 *__restrict__ work, float stepmul)
{
    __shared__ float s_red[SWEEP_WARPS][NCH];
    __shared__ double s_dred[SWEEP_WARPS][NCH];
    __shared__ int s_last;
    const unsigned FULL = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int2 wk = work[blockIdx.x];
    const ImgDev &im = imgs[wk.x];
    const int W = im.W, H = im.H, pitch = im.pitch, R = im.strip_rows;
    const int strip = wk.y * SWEEP_WARPS + warp;
    float2 ssq[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) ssq[c] = make_float2(0.f, 0.f);

    if (strip < im.nstrips) {
        const int sxi = strip % im.strips_x, syi = strip / im.strips_x;
        const int xs = sxi * SWEEP_OUT, ys = syi * R;
        const int ca = xs - 2 + 2 * lane, cb = ca + 1;  // this lane's columns (ca even)
        const bool ina = ca >= 0 && ca < W, inb = cb >= 0 && cb < W;
        const bool pair = ca >= 0 && cb < W;            // both columns inside: one 8-byte load
        const int la = min(max(ca, 0), W - 1), lb = min(max(cb, 0), W - 1);
        const bool outlane = lane >= 1 && lane <= 30 && ca < W;
        const bool lft = ca > 0;                        // column a has a left neighbour in the image
        const int cs = (int)im.cstride;
        const float *ybase = im.y;
        float *gout = im.g + (outlane ? ca : 0);
        const float2 at = make_float2(im.alpha_tv, im.alpha_tv), ag = make_float2(im.alpha_tgv, im.alpha_tgv);
        const float2 half2 = make_float2(0.5f, 0.5f), two2 = make_float2(2.f, 2.f);
        // DCT-distance gradient plane of each channel at this lane's columns
        // (offsets from the first channel's plane), prefetched one row ahead.
        const float *pbase = im.ch[0].P;
        int pcol[NCH], psh[NCH], ppitch[NCH];
        bool pon[NCH], pshare[NCH];
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            const ChanDev &cd = im.ch[c];
            pon[c] = cd.alpha_p != 0.f;
            psh[c] = cd.sv - 1;
            ppitch[c] = cd.ppitch;
            pshare[c] = cd.sh == 2;  // both columns are one component sample
            pcol[c] = (int)(cd.P - pbase) + (outlane ? (ca >> (cd.sh - 1)) : 0);
        }
        const int Hm1 = H - 1;
        auto ld = [&](int c, int off) -> float2 {
            const float *p = ybase + c * cs + off;
            if (pair) return __ldg(reinterpret_cast<const float2 *>(p + ca));
            return make_float2(__ldg(p + la), __ldg(p + lb));
        };
        auto pld = [&](int c, int row) -> float2 {
            if (!pon[c]) return make_float2(0.f, 0.f);
            const float *p = pbase + pcol[c] + (row >> psh[c]) * ppitch[c];
            if (pshare[c]) {
                const float v = __ldg(p);
                return make_float2(v, v);
            }
            return __ldg(reinterpret_cast<const float2 *>(p));
        };

        // Rows in flight: ring[c][k] holds y row t + 1 + k at step t (SWEEP_PF rows
        // ahead of use), pring[c][k] the DCT-distance row t - 1 + k (the output row
        // of step t and SWEEP_PPF - 1 more).
        float2 yv[NCH], dxp[NCH], dyp[NCH], Gm[NCH], G0[NCH], Gp[NCH], ring[NCH][SWEEP_PF], pring[NCH][SWEEP_PPF];
        {
            const int o0 = min(max(ys - 2, 0), Hm1) * pitch, o1 = min(max(ys - 1, 0), Hm1) * pitch;
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                const float2 y0 = ld(c, o0);
                yv[c] = ld(c, o1);
#pragma unroll
                for (int k = 0; k < SWEEP_PF; k++) ring[c][k] = ld(c, min(ys + k, Hm1) * pitch);
#pragma unroll
                for (int k = 0; k < SWEEP_PPF; k++) pring[c][k] = pld(c, min(max(ys - 2 + k, 0), Hm1));
                const float yr = __shfl_down_sync(FULL, y0.x, 1);
                dxp[c] = f2sub(make_float2(y0.y, yr), y0);
                dyp[c] = f2sub(yv[c], y0);
                Gm[c] = G0[c] = Gp[c] = make_float2(0.f, 0.f);
            }
        }
        // The row loop in two forms, as in the narrow variant: EDGE keeps the
        // image-edge rules, interior strips run without them.
        auto rows = [&](auto edge_tag) {
        constexpr bool EDGE = decltype(edge_tag)::value;
        for (int t = ys - 1; t <= ys + R; t++) {
            float2 yn[NCH], pr[NCH];
            {
                const int o = min(t + 1 + SWEEP_PF, Hm1) * pitch;
                const int prow = min(max(t - 1 + SWEEP_PPF, 0), Hm1);
#pragma unroll
                for (int c = 0; c < NCH; c++) {
                    yn[c] = ring[c][0];
#pragma unroll
                    for (int k = 0; k + 1 < SWEEP_PF; k++) ring[c][k] = ring[c][k + 1];
                    ring[c][SWEEP_PF - 1] = ld(c, o);
                    pr[c] = pring[c][0];
#pragma unroll
                    for (int k = 0; k + 1 < SWEEP_PPF; k++) pring[c][k] = pring[c][k + 1];
                    pring[c][SWEEP_PPF - 1] = pld(c, prow);
                }
            }
            const bool rowin = !EDGE || (t >= 0 && t < H), ty0 = !EDGE || t > 0;
            float2 dx[NCH], dy[NCH], gxx[NCH], gyy[NCH], gs[NCH];
            float2 n1 = make_float2(0.f, 0.f), n2 = make_float2(0.f, 0.f);
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                const float yr = __shfl_down_sync(FULL, yv[c].x, 1);
                dx[c] = f2sub(make_float2(yv[c].y, yr), yv[c]);
                dy[c] = f2sub(yn[c], yv[c]);
                n1 = f2fma(dx[c], dx[c], n1);
                n1 = f2fma(dy[c], dy[c], n1);
            }
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                // Backward differences are zero at the left edge and the top row
                // (compute_step_tv2.rs:53-69): take the neighbour equal to self.
                const float dxs = __shfl_up_sync(FULL, dx[c].y, 1), dys = __shfl_up_sync(FULL, dy[c].y, 1);
                const float2 dxl = make_float2(!EDGE || lft ? dxs : dx[c].x, dx[c].x);
                const float2 dyl = make_float2(!EDGE || lft ? dys : dy[c].x, dy[c].x);
                const float2 dxu = ty0 ? dxp[c] : dx[c], dyu = ty0 ? dyp[c] : dy[c];
                const float2 axx = f2sub(dx[c], dxl), ayx = f2sub(dy[c], dyl);
                const float2 ayy = f2sub(dy[c], dyu), axy = f2sub(dx[c], dxu);
                const float2 s = f2mul(half2, f2add(axy, ayx));
                n2 = f2add(n2, f2fma(ayy, ayy, f2fma(two2, f2mul(s, s), f2mul(axx, axx))));
                gxx[c] = axx;
                gyy[c] = ayy;
                gs[c] = s;
            }
            float2 inv1, inv2;
            const bool ia = !EDGE || (rowin && ina), ib = !EDGE || (rowin && inb);
            inv1.x = (ia && n1.x > 0.f) ? rsqrtf(n1.x) : 0.f;
            inv1.y = (ib && n1.y > 0.f) ? rsqrtf(n1.y) : 0.f;
            inv2.x = (ia && n2.x > 0.f) ? rsqrtf(n2.x) : 0.f;
            inv2.y = (ib && n2.y > 0.f) ? rsqrtf(n2.y) : 0.f;
            const float2 at1 = f2mul(at, inv1), ag2 = f2mul(ag, inv2);
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                const float2 a = f2mul(at1, dx[c]), b = f2mul(at1, dy[c]);
                const float2 u = f2mul(ag2, f2add(gs[c], gxx[c]));
                const float2 v = f2mul(ag2, f2add(gyy[c], gs[c]));
                const float2 w = f2mul(ag2, gs[c]);
                const float2 au = f2add(a, u);
                const float aul = __shfl_up_sync(FULL, au.y, 1);
                const float ur = __shfl_down_sync(FULL, u.x, 1);
                const float wr = __shfl_down_sync(FULL, w.x, 1);
                const float wl = __shfl_up_sync(FULL, w.y, 1);
                // centre term -(a + b) - 2 (u + v - w), then the neighbours' a + u and u
                const float2 cen = f2fma(two2, f2sub(f2add(u, v), w), f2add(a, b));
                G0[c] = f2add(f2sub(G0[c], cen), f2add(make_float2(aul, au.x), make_float2(u.y, ur)));
                Gp[c] = f2add(Gp[c], f2sub(f2add(b, v), make_float2(w.y, wr)));
                Gm[c] = f2add(Gm[c], f2sub(v, make_float2(wl, w.x)));
                dxp[c] = dx[c];
                dyp[c] = dy[c];
                yv[c] = yn[c];
            }
            const int ro = t - 1;
            if (outlane && ro >= ys && ro < ys + R && ro < H) {
                const int go = ro * pitch;
#pragma unroll
                for (int c = 0; c < NCH; c++) {
                    const float2 gv = f2add(Gm[c], pr[c]);
                    *reinterpret_cast<float2 *>(gout + c * cs + go) = gv;
                    ssq[c] = f2fma(gv, gv, ssq[c]);
                }
            }
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                Gm[c] = G0[c];
                G0[c] = Gp[c];
                Gp[c] = make_float2(0.f, 0.f);
            }
        }
        };
        // Interior: every lane's two columns inside the image and off its
        // first and last columns (ca >= 1, cb <= W - 2 for all lanes), rows
        // off the first and last.
        const bool interior = xs - 2 >= 1 && xs + 61 <= W - 2 && ys - 1 >= 1 && ys + R + 1 + SWEEP_PF <= H - 1;
        if (interior)
            rows(std::false_type{});
        else
            rows(std::true_type{});
    }

    // Fixed-order reduction: warp tree, then warps in order, then blocks in order.
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        float s = ssq[c].x + ssq[c].y;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
        if (lane == 0) s_red[warp][c] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            float s = 0.f;
            for (int w = 0; w < SWEEP_WARPS; w++) s += s_red[w][c];
            im.partial[wk.y * 4 + c] = s;
        }
        __threadfence();
        const unsigned done = atomicAdd(im.counter, 1u);
        s_last = done == (unsigned)(im.ncta - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        double acc[NCH];
#pragma unroll
        for (int c = 0; c < NCH; c++) acc[c] = 0.0;
        for (int t = threadIdx.x; t < im.ncta; t += SWEEP_WARPS * 32) {
#pragma unroll
            for (int c = 0; c < NCH; c++) acc[c] += (double)__ldcg(im.partial + t * 4 + c);
        }
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            double s = acc[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
            if (lane == 0) s_dred[warp][c] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                double s = 0.0;
                for (int w = 0; w < SWEEP_WARPS; w++) s += s_dred[w][c];
                const double nrm = sqrt(s);
                im.sigma[c] = nrm > 0.0 ? (float)((double)(im.step * stepmul) / nrm) : 0.f;
            }
            atomicExch(im.counter, 0u);
        }
    }
}

// Scalar and packed-pair forms of the sweep's arithmetic: one body serves a
// single channel (float) and a pair of channels (float2, packed FP32x2, one
// instruction for both). Every operation rounds on its own, in the order of
// the wide variant, so a channel's terms are the same in either form.
__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return f2add(a, b); }
__device__ __forceinline__ float vsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float2 vsub(float2 a, float2 b) { return f2sub(a, b); }
__device__ __forceinline__ float vmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return f2mul(a, b); }
__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return f2fma(a, b, c); }
__device__ __forceinline__ void vsplat(float &d, float v) { d = v; }
__device__ __forceinline__ void vsplat(float2 &d, float v) { d = make_float2(v, v); }
__device__ __forceinline__ float vsel(bool p, float a, float b) { return p ? a : b; }
__device__ __forceinline__ float2 vsel(bool p, float2 a, float2 b) { return make_float2(p ? a.x : b.x, p ? a.y : b.y); }
__device__ __forceinline__ float vup(float v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ float2 vup(float2 v) { return make_float2(vup(v.x), vup(v.y)); }
__device__ __forceinline__ float vdn(float v) { return __shfl_down_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ float2 vdn(float2 v) { return make_float2(vdn(v.x), vdn(v.y)); }
// Channel-ordered sums over the channels of a group.
__device__ __forceinline__ float n1_acc(float n, float dx, float dy) { return __fmaf_rn(dy, dy, __fmaf_rn(dx, dx, n)); }
__device__ __forceinline__ float n1_acc(float n, float2 dx, float2 dy) { return n1_acc(n1_acc(n, dx.x, dy.x), dx.y, dy.y); }
__device__ __forceinline__ float h_acc(float n, float t) { return __fadd_rn(n, t); }
__device__ __forceinline__ float h_acc(float n, float2 t) { return __fadd_rn(__fadd_rn(n, t.x), t.y); }

// Narrow sweep state of one group of channels (one channel, or a packed pair).
template <class T>
struct NarrowGroup {
    T yv, dxp, dyp, Gm, G0, Gp, ssq, ring[SWEEP_PF_N], pring[SWEEP_PPF_N];
    T yn, pr, dx, dy, gxx, gyy, gs;
};

// Narrow variant of the gradient sweep: the same terms with one column per
// lane, so more warps cover an image and small images fill the GPU better.
// One warp per strip of SWEEP_OUT_N output columns and strip_rows rows; lane L
// holds column xs - 2 + L. Lanes 1..30 form the per-pixel terms, lanes 2..29
// write g. Rows and columns outside the image are read clamped (replicated
// edges make the reference's last-row/column forward differences vanish,
// compute_step_tv.rs:105-120) and their terms are zero, which reproduces the
// reference's scatter guards. Rows are prefetched two ahead of use. With two
// or three channels, two of them run as a packed pair (channel 0 alone with
// three), which halves their arithmetic instructions.
template <int NCH>
__global__ void __launch_bounds__(SWEEP_WARPS_N * 32, SWEEP_MIN_BLOCKS_N) k_grad_sweep_n(const ImgDev *__restrict__ imgs,
                                                                 const int2 *__restrict__ work, float stepmul)
{
    __shared__ float s_red[SWEEP_WARPS_N][NCH];
    __shared__ double s_dred[SWEEP_WARPS_N][NCH];
    __shared__ int s_last;
    const unsigned FULL = 0xffffffffu;
    constexpr bool SOLO = NCH & 1;     // channel 0 alone
    constexpr bool PAIR = NCH >= 2;    // channels P0, P0 + 1 packed
    constexpr int P0 = SOLO ? 1 : 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int2 wk = work[blockIdx.x];
    const ImgDev &im = imgs[wk.x];
    const int W = im.W, H = im.H, pitch = im.pitch, R = im.strip_rows;
    const int strip = wk.y * SWEEP_WARPS_N + warp;
    NarrowGroup<float> A;
    NarrowGroup<float2> B;
    vsplat(A.ssq, 0.f);
    vsplat(B.ssq, 0.f);

    if (strip < im.nstrips) {
        const int sxi = strip % im.strips_x, syi = strip / im.strips_x;
        const int xs = sxi * SWEEP_OUT_N, ys = syi * R;
        const int gx = xs - 2 + lane;
        const int cx = min(max(gx, 0), W - 1);
        const bool colin = gx >= 0 && gx < W;
        const bool outlane = lane >= 2 && lane < 30 && gx < W;
        const int cs = (int)im.cstride;
        const float *yp = im.y + cx;
        float *gout = im.g + (outlane ? gx : 0);
        const float at = im.alpha_tv, ag = im.alpha_tgv;
        // DCT-distance gradient plane of each channel at this lane's column
        // (offsets from the first channel's plane), prefetched one row ahead.
        const float *pbase = im.ch[0].P;
        int pcol[NCH], psh[NCH], ppitch[NCH];
        bool pon[NCH];
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            const ChanDev &cd = im.ch[c];
            pon[c] = cd.alpha_p != 0.f;
            psh[c] = cd.sv - 1;
            ppitch[c] = cd.ppitch;
            pcol[c] = (int)(cd.P - pbase) + (outlane ? (gx >> (cd.sh - 1)) : 0);
        }
        const int Hm1 = H - 1;
        auto yrow = [&](int row) -> int { return min(max(row, 0), Hm1) * pitch; };
        auto ly = [&](int c, int off) -> float { return __ldg(yp + c * cs + off); };
        auto lp = [&](int c, int row) -> float {
            return pon[c] ? __ldg(pbase + pcol[c] + (row >> psh[c]) * ppitch[c]) : 0.f;
        };
        auto ld_y = [&](auto &g, int off) {
            if constexpr (sizeof(g) == sizeof(float)) g = ly(0, off);
            else g = make_float2(ly(P0, off), ly(P0 + 1, off));
        };
        auto ld_p = [&](auto &g, int row) {
            if constexpr (sizeof(g) == sizeof(float)) g = lp(0, row);
            else g = make_float2(lp(P0, row), lp(P0 + 1, row));
        };
        // Rows in flight: ring[k] = y row t + 1 + k, pring[k] = DCT-distance
        // row t - 1 + k at step t.
        auto init = [&](auto &G) {
            using T = decltype(G.yv);
            T y0;
            ld_y(y0, yrow(ys - 2));
            ld_y(G.yv, yrow(ys - 1));
#pragma unroll
            for (int k = 0; k < SWEEP_PF_N; k++) ld_y(G.ring[k], yrow(ys + k));
#pragma unroll
            for (int k = 0; k < SWEEP_PPF_N; k++) ld_p(G.pring[k], min(max(ys - 2 + k, 0), Hm1));
            G.dxp = vsub(vdn(y0), y0);
            G.dyp = vsub(G.yv, y0);
            vsplat(G.Gm, 0.f);
            vsplat(G.G0, 0.f);
            vsplat(G.Gp, 0.f);
        };
        if constexpr (SOLO) init(A);
        if constexpr (PAIR) init(B);
        // The row loop in two forms: EDGE keeps the image-edge rules; a strip
        // whose lanes and rows all lie inside the image, away from its first
        // and last rows and columns, runs without them (warp-uniform choice).
        auto rows = [&](auto edge_tag) {
        constexpr bool EDGE = decltype(edge_tag)::value;
#pragma unroll 2
        for (int t = ys - 1; t <= ys + R; t++) {
            const int o = min(t + 1 + SWEEP_PF_N, Hm1) * pitch;
            const int pr1 = min(max(t - 1 + SWEEP_PPF_N, 0), Hm1);
            auto load = [&](auto &G) {
                G.yn = G.ring[0];
#pragma unroll
                for (int k = 0; k + 1 < SWEEP_PF_N; k++) G.ring[k] = G.ring[k + 1];
                ld_y(G.ring[SWEEP_PF_N - 1], o);
                G.pr = G.pring[0];
#pragma unroll
                for (int k = 0; k + 1 < SWEEP_PPF_N; k++) G.pring[k] = G.pring[k + 1];
                ld_p(G.pring[SWEEP_PPF_N - 1], pr1);
            };
            if constexpr (SOLO) load(A);
            if constexpr (PAIR) load(B);
            const bool inside = !EDGE || (colin && t >= 0 && t < H);
            float n1 = 0.f, n2 = 0.f;
            auto first = [&](auto &G) {
                G.dx = vsub(vdn(G.yv), G.yv);
                G.dy = vsub(G.yn, G.yv);
                n1 = n1_acc(n1, G.dx, G.dy);
            };
            if constexpr (SOLO) first(A);
            if constexpr (PAIR) first(B);
            const bool tx0 = gx > 0, ty0 = t > 0;
            auto second = [&](auto &G) {
                using T = decltype(G.yv);
                // At the left edge and the top row the backward differences are
                // zero (compute_step_tv2.rs:53-69): take the neighbour equal to self.
                T dxl = vup(G.dx), dyl = vup(G.dy), dxu = G.dxp, dyu = G.dyp;
                if constexpr (EDGE) {
                    dxl = vsel(tx0, dxl, G.dx);
                    dyl = vsel(tx0, dyl, G.dy);
                    dxu = vsel(ty0, dxu, G.dx);
                    dyu = vsel(ty0, dyu, G.dy);
                }
                const T axx = vsub(G.dx, dxl), ayx = vsub(G.dy, dyl);
                const T ayy = vsub(G.dy, dyu), axy = vsub(G.dx, dxu);
                T half, two;
                vsplat(half, 0.5f);
                vsplat(two, 2.f);
                const T sv = vmul(half, vadd(axy, ayx));
                n2 = h_acc(n2, vfma(ayy, ayy, vfma(two, vmul(sv, sv), vmul(axx, axx))));
                G.gxx = axx;
                G.gyy = ayy;
                G.gs = sv;
            };
            if constexpr (SOLO) second(A);
            if constexpr (PAIR) second(B);
            const float inv1 = (inside && n1 > 0.f) ? rsqrtf(n1) : 0.f;
            const float inv2 = (inside && n2 > 0.f) ? rsqrtf(n2) : 0.f;
            const float at1 = __fmul_rn(at, inv1), ag2 = __fmul_rn(ag, inv2);
            auto third = [&](auto &G) {
                using T = decltype(G.yv);
                T at1v, ag2v, two;
                vsplat(at1v, at1);
                vsplat(ag2v, ag2);
                vsplat(two, 2.f);
                const T a = vmul(at1v, G.dx), b = vmul(at1v, G.dy);
                const T u = vmul(ag2v, vadd(G.gs, G.gxx));
                const T v = vmul(ag2v, vadd(G.gyy, G.gs));
                const T w = vmul(ag2v, G.gs);
                const T au = vadd(a, u);
                const T aul = vup(au), ur = vdn(u), wr = vdn(w), wl = vup(w);
                // centre term -(a + b) - 2 (u + v - w), then the neighbours' a + u and u
                const T cen = vfma(two, vsub(vadd(u, v), w), vadd(a, b));
                G.G0 = vadd(vsub(G.G0, cen), vadd(aul, ur));
                G.Gp = vadd(G.Gp, vsub(vadd(b, v), wr));
                G.Gm = vadd(G.Gm, vsub(v, wl));
                G.dxp = G.dx;
                G.dyp = G.dy;
                G.yv = G.yn;
            };
            if constexpr (SOLO) third(A);
            if constexpr (PAIR) third(B);
            const int ro = t - 1;
            if (outlane && ro >= ys && ro < ys + R && ro < H) {
                const int go = ro * pitch;
                if constexpr (SOLO) {
                    const float gv = vadd(A.Gm, A.pr);
                    gout[go] = gv;
                    A.ssq = vfma(gv, gv, A.ssq);
                }
                if constexpr (PAIR) {
                    const float2 gv = vadd(B.Gm, B.pr);
                    gout[P0 * cs + go] = gv.x;
                    gout[(P0 + 1) * cs + go] = gv.y;
                    B.ssq = vfma(gv, gv, B.ssq);
                }
            }
            auto rotate = [&](auto &G) {
                G.Gm = G.G0;
                G.G0 = G.Gp;
                vsplat(G.Gp, 0.f);
            };
            if constexpr (SOLO) rotate(A);
            if constexpr (PAIR) rotate(B);
        }
        };
        const bool interior = xs - 2 >= 1 && xs + 29 <= W - 1 && ys - 1 >= 1 && ys + R + 1 + SWEEP_PF_N <= H - 1;
        if (interior)
            rows(std::false_type{});
        else
            rows(std::true_type{});
    }
    float ssq_c[NCH];
    if constexpr (SOLO) ssq_c[0] = A.ssq;
    if constexpr (PAIR) {
        ssq_c[P0] = B.ssq.x;
        ssq_c[P0 + 1] = B.ssq.y;
    }

    // Fixed-order reduction: warp tree, then warps in order, then blocks in order.
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        float s = ssq_c[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
        if (lane == 0) s_red[warp][c] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            float s = 0.f;
            for (int w = 0; w < SWEEP_WARPS_N; w++) s += s_red[w][c];
            im.partial[wk.y * 4 + c] = s;
        }
        __threadfence();
        const unsigned done = atomicAdd(im.counter, 1u);
        s_last = done == (unsigned)(im.ncta - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        double acc[NCH];
#pragma unroll
        for (int c = 0; c < NCH; c++) acc[c] = 0.0;
        for (int t = threadIdx.x; t < im.ncta; t += SWEEP_WARPS_N * 32) {
#pragma unroll
            for (int c = 0; c < NCH; c++) acc[c] += (double)__ldcg(im.partial + t * 4 + c);
        }
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            double s = acc[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
            if (lane == 0) s_dred[warp][c] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                double s = 0.0;
                for (int w = 0; w < SWEEP_WARPS_N; w++) s += s_dred[w][c];
                const double nrm = sqrt(s);
                im.sigma[c] = nrm > 0.0 ? (float)((double)(im.step * stepmul) / nrm) : 0.f;
            }
            atomicExch(im.counter, 0u);
        }
    }
}

// Quad variant of the gradient sweep: lane L holds the four columns
// x0 = xs - 4 + 4L .. x0 + 3 as two float2 pairs, loaded and stored as float4,
// with packed FP32x2 arithmetic. Horizontal neighbours inside a lane are
// registers; across lanes each row needs two shuffles for the y values (the
// next row's edge values, carried to the following step) and four for the
// gathered terms, against seven per pixel in the narrow variant. Lanes 1..30
// write g, so a warp's strip is SWEEP_OUT_Q = 120 columns and every access is
// 16-byte aligned (W is a multiple of 8, so a lane's four columns are all
// inside the image or all outside it). Every per-pixel expression is the wide
// variant's, in the same order, so both give the same g. Rows and columns
// outside the image are read clamped and their terms are zero, as in the
// other variants.
__device__ __forceinline__ float4 ldg4_clamped(const float *row, int x0, bool inside, int W)
{
    if (inside) return __ldg(reinterpret_cast<const float4 *>(row + x0));
    const float v = __ldg(row + (x0 < 0 ? 0 : W - 1));
    return make_float4(v, v, v, v);
}

template <int NCH>
__global__ void __launch_bounds__(SWEEP_WARPS_Q * 32, SWEEP_MIN_BLOCKS_Q) k_grad_sweep_q(
    const ImgDev *__restrict__ imgs, const int2 *__restrict__ work, float stepmul)
{
    __shared__ float s_red[SWEEP_WARPS_Q][NCH];
    __shared__ double s_dred[SWEEP_WARPS_Q][NCH];
    __shared__ int s_last;
    const unsigned FULL = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int2 wk = work[blockIdx.x];
    const ImgDev &im = imgs[wk.x];
    const int W = im.W, H = im.H, pitch = im.pitch, R = im.strip_rows;
    const int strip = wk.y * SWEEP_WARPS_Q + warp;
    float2 ssq[NCH];
#pragma unroll
    for (int c = 0; c < NCH; c++) ssq[c] = make_float2(0.f, 0.f);

    if (strip < im.nstrips) {
        const int sxi = strip % im.strips_x, syi = strip / im.strips_x;
        const int xs = sxi * SWEEP_OUT_Q, ys = syi * R;
        const int x0 = xs - 4 + 4 * lane;
        const bool colin = x0 >= 0 && x0 < W;      // all four columns inside (W % 8 == 0)
        const bool outlane = lane >= 1 && lane <= 30 && x0 < W;
        const bool lft = x0 > 0;                   // column x0 has a left neighbour in the image
        const int cs = (int)im.cstride;
        float *gout = im.g + (outlane ? x0 : 0);
        const float2 at = make_float2(im.alpha_tv, im.alpha_tv), ag = make_float2(im.alpha_tgv, im.alpha_tgv);
        const float2 half2 = make_float2(0.5f, 0.5f), two2 = make_float2(2.f, 2.f);
        const float *pbase = im.ch[0].P;
        int pcol[NCH], psh[NCH], ppitch[NCH];
        bool pon[NCH], pshare[NCH];
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            const ChanDev &cd = im.ch[c];
            pon[c] = cd.alpha_p != 0.f;
            psh[c] = cd.sv - 1;
            ppitch[c] = cd.ppitch;
            pshare[c] = cd.sh == 2;  // columns 2k, 2k + 1 are one component sample
            pcol[c] = (int)(cd.P - pbase) + (outlane ? (x0 >> (cd.sh - 1)) : 0);
        }
        const int Hm1 = H - 1;
        auto ld = [&](int c, int off) -> float4 { return ldg4_clamped(im.y + c * cs + off, x0, colin, W); };
        auto pld = [&](int c, int row) -> float4 {
            if (!pon[c] || !outlane) return make_float4(0.f, 0.f, 0.f, 0.f);
            const float *p = pbase + pcol[c] + (row >> psh[c]) * ppitch[c];
            if (pshare[c]) {
                const float2 v = __ldg(reinterpret_cast<const float2 *>(p));
                return make_float4(v.x, v.x, v.y, v.y);
            }
            return __ldg(reinterpret_cast<const float4 *>(p));
        };
        auto lo2 = [](float4 v) { return make_float2(v.x, v.y); };
        auto hi2 = [](float4 v) { return make_float2(v.z, v.w); };

        // Per channel: the current row yv, its neighbours' edge values yl =
        // y[x0 - 1], yr = y[x0 + 4], the previous row's differences, the three
        // output-row accumulators and the rows in flight (ring: y rows t + 1 + k,
        // pring: DCT-distance rows t - 1 + k at step t).
        float4 yv[NCH], ring[NCH][SWEEP_PF_Q], pring[NCH][SWEEP_PPF_Q];
        float yl[NCH], yr[NCH];
        float2 dxpa[NCH], dxpb[NCH], dypa[NCH], dypb[NCH];
        float2 Gma[NCH], Gmb[NCH], G0a[NCH], G0b[NCH], Gpa[NCH], Gpb[NCH];
        {
            const int o0 = min(max(ys - 2, 0), Hm1) * pitch, o1 = min(max(ys - 1, 0), Hm1) * pitch;
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                const float4 y0 = ld(c, o0);
                yv[c] = ld(c, o1);
#pragma unroll
                for (int k = 0; k < SWEEP_PF_Q; k++) ring[c][k] = ld(c, min(ys + k, Hm1) * pitch);
#pragma unroll
                for (int k = 0; k < SWEEP_PPF_Q; k++) pring[c][k] = pld(c, min(max(ys - 2 + k, 0), Hm1));
                // Differences of row ys - 2 (the first step's previous row).
                const float y0r = __shfl_down_sync(FULL, y0.x, 1);
                dxpa[c] = f2sub(make_float2(y0.y, y0.z), lo2(y0));
                dxpb[c] = f2sub(make_float2(y0.w, y0r), hi2(y0));
                dypa[c] = f2sub(lo2(yv[c]), lo2(y0));
                dypb[c] = f2sub(hi2(yv[c]), hi2(y0));
                yl[c] = __shfl_up_sync(FULL, yv[c].w, 1);
                yr[c] = __shfl_down_sync(FULL, yv[c].x, 1);
                Gma[c] = Gmb[c] = G0a[c] = G0b[c] = Gpa[c] = Gpb[c] = make_float2(0.f, 0.f);
            }
        }
#pragma unroll 1
        for (int t = ys - 1; t <= ys + R; t++) {
            float4 yn[NCH], pr[NCH];
            float nl[NCH], nr[NCH];
            {
                const int o = min(t + 1 + SWEEP_PF_Q, Hm1) * pitch;
                const int prow = min(max(t - 1 + SWEEP_PPF_Q, 0), Hm1);
#pragma unroll
                for (int c = 0; c < NCH; c++) {
                    yn[c] = ring[c][0];
#pragma unroll
                    for (int k = 0; k + 1 < SWEEP_PF_Q; k++) ring[c][k] = ring[c][k + 1];
                    ring[c][SWEEP_PF_Q - 1] = ld(c, o);
                    pr[c] = pring[c][0];
#pragma unroll
                    for (int k = 0; k + 1 < SWEEP_PPF_Q; k++) pring[c][k] = pring[c][k + 1];
                    pring[c][SWEEP_PPF_Q - 1] = pld(c, prow);
                    nl[c] = __shfl_up_sync(FULL, yn[c].w, 1);
                    nr[c] = __shfl_down_sync(FULL, yn[c].x, 1);
                }
            }
            const bool rowin = colin && t >= 0 && t < H, ty0 = t > 0;
            float2 dxa[NCH], dxb[NCH], dya[NCH], dyb[NCH], gxxa[NCH], gxxb[NCH], gyya[NCH], gyyb[NCH];
            float2 gsa[NCH], gsb[NCH];
            float2 n1a = make_float2(0.f, 0.f), n1b = n1a, n2a = n1a, n2b = n1a;
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                const float4 y = yv[c];
                dxa[c] = f2sub(make_float2(y.y, y.z), lo2(y));
                dxb[c] = f2sub(make_float2(y.w, yr[c]), hi2(y));
                dya[c] = f2sub(lo2(yn[c]), lo2(y));
                dyb[c] = f2sub(hi2(yn[c]), hi2(y));
                n1a = f2fma(dxa[c], dxa[c], n1a);
                n1a = f2fma(dya[c], dya[c], n1a);
                n1b = f2fma(dxb[c], dxb[c], n1b);
                n1b = f2fma(dyb[c], dyb[c], n1b);
            }
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                // Backward differences are zero at the left edge and the top row
                // (compute_step_tv2.rs:53-69): take the neighbour equal to self.
                const float dxs = yv[c].x - yl[c], dys = nl[c] - yl[c];  // dx, dy at x0 - 1
                const float2 dxla = make_float2(lft ? dxs : dxa[c].x, dxa[c].x);
                const float2 dyla = make_float2(lft ? dys : dya[c].x, dya[c].x);
                const float2 dxlb = make_float2(dxa[c].y, dxb[c].x);
                const float2 dylb = make_float2(dya[c].y, dyb[c].x);
                const float2 dxua = ty0 ? dxpa[c] : dxa[c], dyua = ty0 ? dypa[c] : dya[c];
                const float2 dxub = ty0 ? dxpb[c] : dxb[c], dyub = ty0 ? dypb[c] : dyb[c];
                const float2 axxa = f2sub(dxa[c], dxla), ayxa = f2sub(dya[c], dyla);
                const float2 axxb = f2sub(dxb[c], dxlb), ayxb = f2sub(dyb[c], dylb);
                const float2 ayya = f2sub(dya[c], dyua), axya = f2sub(dxa[c], dxua);
                const float2 ayyb = f2sub(dyb[c], dyub), axyb = f2sub(dxb[c], dxub);
                const float2 sa = f2mul(half2, f2add(axya, ayxa)), sb = f2mul(half2, f2add(axyb, ayxb));
                n2a = f2add(n2a, f2fma(ayya, ayya, f2fma(two2, f2mul(sa, sa), f2mul(axxa, axxa))));
                n2b = f2add(n2b, f2fma(ayyb, ayyb, f2fma(two2, f2mul(sb, sb), f2mul(axxb, axxb))));
                gxxa[c] = axxa;
                gxxb[c] = axxb;
                gyya[c] = ayya;
                gyyb[c] = ayyb;
                gsa[c] = sa;
                gsb[c] = sb;
            }
            float2 inv1a, inv1b, inv2a, inv2b;
            inv1a.x = (rowin && n1a.x > 0.f) ? rsqrtf(n1a.x) : 0.f;
            inv1a.y = (rowin && n1a.y > 0.f) ? rsqrtf(n1a.y) : 0.f;
            inv1b.x = (rowin && n1b.x > 0.f) ? rsqrtf(n1b.x) : 0.f;
            inv1b.y = (rowin && n1b.y > 0.f) ? rsqrtf(n1b.y) : 0.f;
            inv2a.x = (rowin && n2a.x > 0.f) ? rsqrtf(n2a.x) : 0.f;
            inv2a.y = (rowin && n2a.y > 0.f) ? rsqrtf(n2a.y) : 0.f;
            inv2b.x = (rowin && n2b.x > 0.f) ? rsqrtf(n2b.x) : 0.f;
            inv2b.y = (rowin && n2b.y > 0.f) ? rsqrtf(n2b.y) : 0.f;
            const float2 at1a = f2mul(at, inv1a), at1b = f2mul(at, inv1b);
            const float2 ag2a = f2mul(ag, inv2a), ag2b = f2mul(ag, inv2b);
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                const float2 aa = f2mul(at1a, dxa[c]), ab = f2mul(at1b, dxb[c]);
                const float2 ba = f2mul(at1a, dya[c]), bb = f2mul(at1b, dyb[c]);
                const float2 ua = f2mul(ag2a, f2add(gsa[c], gxxa[c])), ub = f2mul(ag2b, f2add(gsb[c], gxxb[c]));
                const float2 va = f2mul(ag2a, f2add(gyya[c], gsa[c])), vb = f2mul(ag2b, f2add(gyyb[c], gsb[c]));
                const float2 wa = f2mul(ag2a, gsa[c]), wb = f2mul(ag2b, gsb[c]);
                const float2 aua = f2add(aa, ua), aub = f2add(ab, ub);
                const float aul = __shfl_up_sync(FULL, aub.y, 1);   // (a + u) at x0 - 1
                const float ur = __shfl_down_sync(FULL, ua.x, 1);   // u at x0 + 4
                const float wr = __shfl_down_sync(FULL, wa.x, 1);   // w at x0 + 4
                const float wl = __shfl_up_sync(FULL, wb.y, 1);     // w at x0 - 1
                // centre term -(a + b) - 2 (u + v - w), then the neighbours' a + u and u
                const float2 cena = f2fma(two2, f2sub(f2add(ua, va), wa), f2add(aa, ba));
                const float2 cenb = f2fma(two2, f2sub(f2add(ub, vb), wb), f2add(ab, bb));
                G0a[c] = f2add(f2sub(G0a[c], cena), f2add(make_float2(aul, aua.x), make_float2(ua.y, ub.x)));
                G0b[c] = f2add(f2sub(G0b[c], cenb), f2add(make_float2(aua.y, aub.x), make_float2(ub.y, ur)));
                Gpa[c] = f2add(Gpa[c], f2sub(f2add(ba, va), make_float2(wa.y, wb.x)));
                Gpb[c] = f2add(Gpb[c], f2sub(f2add(bb, vb), make_float2(wb.y, wr)));
                Gma[c] = f2add(Gma[c], f2sub(va, make_float2(wl, wa.x)));
                Gmb[c] = f2add(Gmb[c], f2sub(vb, make_float2(wa.y, wb.x)));
                dxpa[c] = dxa[c];
                dxpb[c] = dxb[c];
                dypa[c] = dya[c];
                dypb[c] = dyb[c];
                yv[c] = yn[c];
                yl[c] = nl[c];
                yr[c] = nr[c];
            }
            const int ro = t - 1;
            if (outlane && ro >= ys && ro < ys + R && ro < H) {
                const int go = ro * pitch;
#pragma unroll
                for (int c = 0; c < NCH; c++) {
                    const float2 ga = f2add(Gma[c], lo2(pr[c])), gb = f2add(Gmb[c], hi2(pr[c]));
                    *reinterpret_cast<float4 *>(gout + c * cs + go) = make_float4(ga.x, ga.y, gb.x, gb.y);
                    ssq[c] = f2fma(ga, ga, ssq[c]);
                    ssq[c] = f2fma(gb, gb, ssq[c]);
                }
            }
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                Gma[c] = G0a[c];
                Gmb[c] = G0b[c];
                G0a[c] = Gpa[c];
                G0b[c] = Gpb[c];
                Gpa[c] = Gpb[c] = make_float2(0.f, 0.f);
            }
        }
    }

    // Fixed-order reduction: warp tree, then warps in order, then blocks in order.
#pragma unroll
    for (int c = 0; c < NCH; c++) {
        float s = ssq[c].x + ssq[c].y;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
        if (lane == 0) s_red[warp][c] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            float s = 0.f;
            for (int w = 0; w < SWEEP_WARPS_Q; w++) s += s_red[w][c];
            im.partial[wk.y * 4 + c] = s;
        }
        __threadfence();
        const unsigned done = atomicAdd(im.counter, 1u);
        s_last = done == (unsigned)(im.ncta - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        double acc[NCH];
#pragma unroll
        for (int c = 0; c < NCH; c++) acc[c] = 0.0;
        for (int t = threadIdx.x; t < im.ncta; t += SWEEP_WARPS_Q * 32) {
#pragma unroll
            for (int c = 0; c < NCH; c++) acc[c] += (double)__ldcg(im.partial + t * 4 + c);
        }
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            double s = acc[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
            if (lane == 0) s_dred[warp][c] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int c = 0; c < NCH; c++) {
                double s = 0.0;
                for (int w = 0; w < SWEEP_WARPS_Q; w++) s += s_dred[w][c];
                const double nrm = sqrt(s);
                im.sigma[c] = nrm > 0.0 ? (float)((double)(im.step * stepmul) / nrm) : 0.f;
            }
            atomicExch(im.counter, 0u);
        }
    }
}

// Descent step and projection of coefficient blocks (compute_step.rs:60-71,
// compute_projection.rs:8-122), the next FISTA point, and the next
// DCT-distance gradient (compute_step_prob.rs:20-57) from the clamped
// coefficients the reference keeps as cos (compute_projection.rs:82).
// One warp per task {image, channel, block row, first block} covering four
// blocks. The warp's region of y and g (8 SV rows x 32 SH columns) is staged
// into shared memory with asynchronous 16-byte copies, one round trip; once g
// is consumed (x' = y - sigma g), the same plane receives the region of x,
// again asynchronously, while the block transforms run. Lane group
// g = lane / 8 takes block first + g and lane j = lane % 8 its component
// column j (SH full-resolution columns). The separable 1-D
// transforms run on columns or rows of the block, switching with 8x8
// transposes in shared memory: the DCT in the reference's order (columns
// first), the IDCTs rows first (one transpose each).
template <int SH, int SV>
struct ProjShape {
    static constexpr int NR = 8 * SV;       // rows of the region
    static constexpr int NC = 32 * SH;      // columns of the region
    static constexpr int RS = NC + 4;       // padded row stride (floats)
    static constexpr int REGION = NR * RS;  // floats per staged plane
};

template <int SH, int SV, int PW = PROJ_WARPS>
__global__ void __launch_bounds__(PW * 32) k_project(const ImgDev *__restrict__ imgs,
                                                    const int4 *__restrict__ tasks, int ntasks, float fnext)
{
    using S = ProjShape<SH, SV>;
    constexpr bool SUB = SH * SV > 1;
    constexpr int NR = S::NR, NC = S::NC, RS = S::RS;
    extern __shared__ float4 s_dyn[];
    __shared__ float s_t[PW][2][4][8][9];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = blockIdx.x * PW + warp;
    if (w >= ntasks) return;  // warp-uniform
    float *sy_ = reinterpret_cast<float *>(s_dyn) + warp * 2 * S::REGION;  // y region; g, then x region
    float *sg_ = sy_ + S::REGION, *sx_ = sg_;
    const int4 tk = tasks[w];
    const ImgDev &im = imgs[tk.x];
    const int c = tk.y, by = tk.z, grp = lane >> 3, j = lane & 7;
    const int bx = tk.w + grp;
    const ChanDev &cd = im.ch[c];
    const int bw = cd.cw / 8;
    const bool act = bx < bw;
    const int cs = (int)im.cstride;
    const int pitch = im.pitch;
    float *xw = im.x + c * cs, *yw = im.y + c * cs;
    const float *gb = im.g + c * cs;
    // A zero step (sigma = 0: the projection of a start image, or a gradient
    // of norm zero) leaves x' = y: g is then neither staged nor read, so the
    // projection of a start needs no zeroed g plane.
    const float sg = im.sigma[c];
    const bool stepped = sg != 0.f;  // warp-uniform
    // Stage the region: rows of NC floats, 16-byte chunks; chunks of blocks
    // past the end of the block row are skipped.
    const int ncol = min(NC, (bw - tk.w) * 8 * SH);  // valid columns, a multiple of 8
    const long long r0 = (long long)(by * 8 * SV) * pitch + tk.w * 8 * SH;
    constexpr int CPR = NC / 4;  // 16-byte chunks per row
    for (int i = lane; i < NR * CPR; i += 32) {
        const int row = i / CPR, ch = i - row * CPR;
        if (ch * 4 < ncol) {
            const long long go = r0 + (long long)row * pitch + ch * 4;
            const int so = row * RS + ch * 4;
            cp_async16(sy_ + so, yw + go);
            if (stepped) cp_async16(sg_ + so, gb + go);
        }
    }
    // Meanwhile: coefficient row j of this lane's block and its quantisation steps.
    float co[8], qv[8], iq[8];
    load_coef_row(cd.coef + (by * 8 + j) * cd.cpitch + (act ? bx : 0) * 8, co);
#pragma unroll
    for (int u = 0; u < 8; u++) {
        qv[u] = __ldg(&im.q[c][j * 8 + u]);
        iq[u] = __ldg(&im.invq2[c][j * 8 + u]);
    }
    const float ap = cd.alpha_p;  // warp-uniform
    float(*T0)[9] = s_t[warp][0][grp];
    float(*T1)[9] = s_t[warp][1][grp];
    cp_async_wait_all();
    __syncwarp();

    // x' = y - sigma g (kept in the y region for a subsampled component, whose
    // residual needs it); cell means for subsampled components, summed sample
    // by sample (compute_projection.rs:18-32).
    const int cb = (grp * 8 + j) * SH;  // first region column of this lane
    float m[8], mean[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        float acc = 0.f;
#pragma unroll
        for (int sy = 0; sy < SV; sy++)
#pragma unroll
            for (int sx = 0; sx < SH; sx++) {
                const int so = (k * SV + sy) * RS + cb + sx;
                const float v = stepped ? fmaf(-sg, sg_[so], sy_[so]) : sy_[so];
                if (SUB) sy_[so] = v;  // read back for the residual of a subsampled component
                acc += v;
            }
        mean[k] = SUB ? acc / (float)(SH * SV) : acc;
        m[k] = mean[k];
    }
    // g is consumed: stage x_k into its plane while the transforms run.
    __syncwarp();
    for (int i = lane; i < NR * CPR; i += 32) {
        const int row = i / CPR, ch = i - row * CPR;
        if (ch * 4 < ncol) cp_async16(sx_ + row * RS + ch * 4, xw + r0 + (long long)row * pitch + ch * 4);
    }
    // DCT, columns then rows (dct8x8s); the lane then holds coefficient row j.
    dct8(m);
    transpose8(T0, j, m);
    dct8(m);
    // Clamp (compute_projection.rs:72-79) and (cos - c q) / q^2.
    float d[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
        const float cl = fminf(fmaxf(m[u], (co[u] - 0.5f) * qv[u]), (co[u] + 0.5f) * qv[u]);
        m[u] = cl;
        d[u] = (cl - co[u] * qv[u]) * iq[u];
    }
    // IDCT of the clamped coefficients and of d: the row pass on the
    // coefficient row this lane holds, one transpose to this lane's column,
    // then the column pass. The reference runs columns first (idct8x8s); the
    // two orders are the same transform and differ only in float rounding,
    // and this one needs one transpose per plane instead of three (the
    // transposes' shared-memory traffic bounds this kernel).
    idct8(m);
    if (ap != 0.f) idct8(d);
    transpose8(T0, j, m);
    if (ap != 0.f) transpose8(T1, j, d);
    idct8(m);
    if (ap != 0.f) idct8(d);
    cp_async_wait_all();
    __syncwarp();
    if (!act) return;
    if (ap != 0.f) {
        float *P = cd.P + by * 8 * cd.ppitch + bx * 8 + j;
#pragma unroll
        for (int k = 0; k < 8; k++) P[k * cd.ppitch] = ap * d[k];
    }
    // x_{k+1}: the projected block, or for subsampled components the residual
    // x' - mean plus the projected mean (compute_projection.rs:108-121); then
    // y_{k+1} = x_{k+1} + f (x_{k+1} - x_k) (mod.rs:54-57).
    const int o0 = by * 8 * SV * pitch + bx * 8 * SH + j * SH;
#pragma unroll
    for (int k = 0; k < NR; k++) {
        const int kc = k / SV;
        float xn[SH], yn[SH];
#pragma unroll
        for (int sx = 0; sx < SH; sx++) {
            const int so = k * RS + cb + sx;
            xn[sx] = SUB ? (sy_[so] - mean[kc]) + m[kc] : m[kc];
            yn[sx] = fmaf(fnext, xn[sx] - sx_[so], xn[sx]);
        }
        const int o = o0 + k * pitch;
        if (SH == 1) {
            xw[o] = xn[0];
            yw[o] = yn[0];
        } else {
            *reinterpret_cast<float2 *>(xw + o) = make_float2(xn[0], xn[SH - 1]);
            *reinterpret_cast<float2 *>(yw + o) = make_float2(yn[0], yn[SH - 1]);
        }
    }
}

// Initial image (coef.rs:24-92 with the single unboxing of
// pipeline_simd_adaptive/coef.rs:69-95): IDCT of c*q per block, nearest
// upsampling to full resolution, written as x_0 and y_0 (aux.rs:62-63).
// Same lane layout as k_project.
__global__ void __launch_bounds__(PROJ_WARPS * 32) k_init(const ImgDev *__restrict__ imgs,
                                                         const int4 *__restrict__ tasks, int ntasks)
{
    __shared__ float s_t[PROJ_WARPS][4][8][9];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = blockIdx.x * PROJ_WARPS + warp;
    if (w >= ntasks) return;
    const int4 tk = tasks[w];
    const ImgDev &im = imgs[tk.x];
    const int c = tk.y, by = tk.z, grp = lane >> 3, r = lane & 7;
    const int bx = tk.w + grp;
    const ChanDev &cd = im.ch[c];
    const bool act = bx < cd.cw / 8;
    float(*T)[9] = s_t[warp][grp];
    float a[8], co[8];
    load_coef_row(cd.coef + (long long)(by * 8 + r) * cd.cpitch + (act ? bx : 0) * 8, co);
#pragma unroll
    for (int u = 0; u < 8; u++) a[u] = co[u] * __ldg(&im.q[c][r * 8 + u]);
    transpose8(T, r, a);
    idct8(a);
    transpose8(T, r, a);
    idct8(a);
    if (!act) return;
    const int sh = cd.sh, sv = cd.sv;
    const long long base = c * im.cstride;
    for (int sy = 0; sy < sv; sy++) {
        const long long o = base + (long long)(by * 8 * sv + r * sv + sy) * im.pitch + bx * 8 * sh;
#pragma unroll
        for (int u = 0; u < 8; u++)
            for (int sx = 0; sx < sh; sx++) {
                im.x[o + u * sh + sx] = a[u];
                im.y[o + u * sh + sx] = a[u];
            }
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

// ---------------------------------------------------------- evaluation ----
// Objective and feasibility of an iterate in fp64 (not on the solve path).
// The objective is the function whose gradient the iteration follows: the
// coupled TV and TGV norms of compute_step_tv.rs:63-71 and
// compute_step_tv2.rs:76-90 summed over pixels, plus for each component
// (alpha_p sh sv / 2) sum ((X - c q) / q)^2 over its blocks, X the DCT of the
// (cell-averaged) plane; the sh sv factor makes the gradient of that term the
// reference's unscaled replication to subsampled pixels
// (compute_step_prob.rs:43-55).

__constant__ double c_dct_matrix[64];  // orthonormal DCT-II, row u: s(u) cos((2y + 1) u pi / 16)

constexpr int EVAL_THREADS = 256;
constexpr int EVAL_BLOCKS = 592;

__device__ __forceinline__ double block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < EVAL_THREADS / 32; w++) t += sh[w];
    __syncthreads();
    return t;
}

// Per block: sum over its pixels of n1 = sqrt(sum_c dx^2 + dy^2) and
// n2 = sqrt(sum_c gyy^2 + 2 s^2 + gxx^2), into partial[2 b], partial[2 b + 1].
__global__ void __launch_bounds__(EVAL_THREADS) k_eval_pixels(const ImgDev *__restrict__ imgs, int img,
                                                              double *__restrict__ partial)
{
    __shared__ double sh[EVAL_THREADS / 32];
    const ImgDev &im = imgs[img];
    const int W = im.W, H = im.H;
    double s1 = 0, s2 = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)W * H;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % W), y = (int)(i / W);
        double n1 = 0, n2 = 0;
        for (int c = 0; c < im.nch; c++) {
            const float *f = im.x + c * im.cstride;
            auto F = [&](int xx, int yy) { return (double)f[(long long)yy * im.pitch + xx]; };
            auto DX = [&](int xx, int yy) { return xx < W - 1 ? F(xx + 1, yy) - F(xx, yy) : 0.0; };
            auto DY = [&](int xx, int yy) { return yy < H - 1 ? F(xx, yy + 1) - F(xx, yy) : 0.0; };
            const double dx = DX(x, y), dy = DY(x, y);
            n1 += dx * dx + dy * dy;
            double gxx = 0, gyx = 0, gyy = 0, gxy = 0;
            if (x > 0) {
                gxx = dx - DX(x - 1, y);
                gyx = dy - DY(x - 1, y);
            }
            if (y > 0) {
                gyy = dy - DY(x, y - 1);
                gxy = dx - DX(x, y - 1);
            }
            const double sm = 0.5 * (gxy + gyx);
            n2 += gyy * gyy + 2.0 * sm * sm + gxx * gxx;
        }
        s1 += sqrt(n1);
        s2 += sqrt(n2);
    }
    s1 = block_sum(s1, sh);
    s2 = block_sum(s2, sh);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = s1;
        partial[2 * blockIdx.x + 1] = s2;
    }
}

// Per block: for channel c, sum over its 8x8 coefficient blocks of
// ((X - c q) / q)^2 and the largest distance of X outside [(c - 1/2) q, (c + 1/2) q]
// (X in fp64 from the cell-averaged plane, compute_projection.rs:18-32 and :72-79).
__global__ void __launch_bounds__(EVAL_THREADS) k_eval_blocks(const ImgDev *__restrict__ imgs, int img, int c,
                                                              double *__restrict__ partial)
{
    __shared__ double sh[EVAL_THREADS / 32];
    __shared__ double sm_max[EVAL_THREADS];
    const ImgDev &im = imgs[img];
    const ChanDev &cd = im.ch[c];
    const int bw = cd.cw / 8, nb = bw * (cd.chh / 8);
    const float *f = im.x + c * im.cstride;
    const double inv_cell = 1.0 / (double)(cd.sh * cd.sv);
    double acc = 0, worst = 0;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int bx = b % bw, by = b / bw;
        double blk[64], t[64];
        for (int r = 0; r < 8; r++)
            for (int u = 0; u < 8; u++) {
                double m = 0;
                for (int sy = 0; sy < cd.sv; sy++)
                    for (int sx = 0; sx < cd.sh; sx++)
                        m += (double)f[(long long)((by * 8 + r) * cd.sv + sy) * im.pitch + (bx * 8 + u) * cd.sh + sx];
                blk[r * 8 + u] = m * inv_cell;
            }
        for (int v = 0; v < 8; v++)  // t = C * blk (columns)
            for (int u = 0; u < 8; u++) {
                double a = 0;
                for (int r = 0; r < 8; r++) a += c_dct_matrix[v * 8 + r] * blk[r * 8 + u];
                t[v * 8 + u] = a;
            }
        for (int v = 0; v < 8; v++)  // X = t * C^T (rows)
            for (int u = 0; u < 8; u++) {
                double X = 0;
                for (int k = 0; k < 8; k++) X += t[v * 8 + k] * c_dct_matrix[u * 8 + k];
                const double q = im.q[c][v * 8 + u];
                const double cc = (double)cd.coef[(long long)(by * 8 + v) * cd.cpitch + bx * 8 + u];
                const double d = (X - cc * q) / q;
                acc += d * d;
                const double lo = (cc - 0.5) * q, hi = (cc + 0.5) * q;
                const double viol = X < lo ? lo - X : (X > hi ? X - hi : 0.0);
                worst = fmax(worst, viol);
            }
    }
    acc = block_sum(acc, sh);
    sm_max[threadIdx.x] = worst;
    __syncthreads();
    for (int k = EVAL_THREADS / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) sm_max[threadIdx.x] = fmax(sm_max[threadIdx.x], sm_max[threadIdx.x + k]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = acc;
        partial[2 * blockIdx.x + 1] = sm_max[0];
    }
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
    im.x[off] = v;
    im.y[off] = v;
}

// Smooth upsampling of a component image to both state buffers (the learned
// start). Along each subsampled axis, full-resolution sample 2 i + d of cell i
// takes 3/4 of cell i and 1/4 of its neighbour on that side (cell i - 1 for
// d = 0, i + 1 for d = 1), clamped at the component's edges: linear
// interpolation between cell centres, horizontal first, each product and sum
// rounded on its own (no contraction), so a float32 host restatement is exact.
// Replicating the cells instead (k_upsample) leaves a step at every cell edge
// that the second-order term prices high and the iterations are slow to
// remove; the projection that follows restores the cells' means.
__device__ __forceinline__ float tri_mix(float a, float b) { return __fadd_rn(__fmul_rn(0.75f, a), __fmul_rn(0.25f, b)); }

__global__ void k_upsample_smooth(const float *__restrict__ img, const ImgDev *__restrict__ imgs, int c)
{
    const ImgDev &im = imgs[0];
    const ChanDev &cd = im.ch[c];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)im.W * im.H) return;
    const int y = (int)(i / im.W), x = (int)(i % im.W);
    const int cy = min(y / cd.sv, cd.chh - 1), cx = min(x / cd.sh, cd.cw - 1);
    const int nx = cd.sh == 2 ? ((x & 1) ? min(cx + 1, cd.cw - 1) : max(cx - 1, 0)) : cx;
    const int ny = cd.sv == 2 ? ((y & 1) ? min(cy + 1, cd.chh - 1) : max(cy - 1, 0)) : cy;
    const float *r0 = img + (long long)cy * cd.cw, *r1 = img + (long long)ny * cd.cw;
    float v = cd.sh == 2 ? tri_mix(r0[cx], r0[nx]) : r0[cx];
    if (cd.sv == 2) v = tri_mix(v, cd.sh == 2 ? tri_mix(r1[cx], r1[nx]) : r1[cx]);
    const long long off = c * im.cstride + (long long)y * im.pitch + x;
    im.x[off] = v;
    im.y[off] = v;
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

// A device buffer that only grows. It grows by at least half its size (in
// 2 MiB steps), so a stream of solves of slowly growing size -- batches of a
// decode pipeline -- reallocates rarely: cudaFree waits for the whole device,
// which would serialise contexts working side by side, and a new address
// forces the iteration graph to be captured again.
struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
    int ensure(size_t bytes)
    {
        if (bytes <= n) return ART_OK;
        if (n) bytes = std::max(bytes, n + n / 2);
        bytes = (bytes + (2u << 20) - 1) / (2u << 20) * (2u << 20);
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

// Pinned host buffer that only grows, like DevBuf: host-device copies from it
// run asynchronously at full link speed, where pageable ones are staged by the
// driver one call at a time.
struct HostBuf {
    void *p = nullptr;
    size_t n = 0;
    int ensure(size_t bytes)
    {
        if (bytes <= n) return ART_OK;
        if (n) bytes = std::max(bytes, n + n / 2);
        bytes = (bytes + (2u << 20) - 1) / (2u << 20) * (2u << 20);
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaHostAlloc(&p, bytes, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(ART_ERR_CUDA, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
        }
        n = bytes;
        return ART_OK;
    }
    void release()
    {
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
    }
};

struct CopyJob {
    void *dst;
    const void *src;
    size_t n;
};

// Host copies of many buffers, split by bytes over up to 8 threads when they
// add up to more than a few megabytes (one thread streams ~10 GB/s).
void parallel_copy(const std::vector<CopyJob> &jobs)
{
    size_t total = 0;
    for (const auto &j : jobs) total += j.n;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = total >= (8u << 20) ? std::min(8u, hw) : 1u;
    auto run = [&](size_t lo, size_t hi) {
        size_t at = 0;
        for (const auto &j : jobs) {
            const size_t a = std::max(lo, at), b = std::min(hi, at + j.n);
            if (a < b)
                memcpy(static_cast<char *>(j.dst) + (a - at), static_cast<const char *>(j.src) + (a - at), b - a);
            at += j.n;
            if (at >= hi) break;
        }
    };
    if (nt <= 1) {
        run(0, total);
        return;
    }
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; t++) th.emplace_back(run, total * t / nt, total * (t + 1) / nt);
    run(0, total / nt);
    for (auto &t : th) t.join();
}

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
    int nimg = 0, proj_warps = 0, wcount[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    int mode_off[5] = {0, 0, 0, 0, 0};
    uint32_t iterations = 0, tail = 0;
    float tail_stepmul = 1.0f, decay = 0.0f;
    bool timing = false;
    const void *desc = nullptr, *work = nullptr, *tasks = nullptr;
    bool operator==(const GraphKey &o) const
    {
        return nimg == o.nimg && proj_warps == o.proj_warps && iterations == o.iterations && tail == o.tail &&
               tail_stepmul == o.tail_stepmul && decay == o.decay &&
               timing == o.timing && desc == o.desc &&
               work == o.work && tasks == o.tasks && std::equal(wcount, wcount + 12, o.wcount) &&
               std::equal(mode_off, mode_off + 5, o.mode_off);
    }
};

// One image of a solve: geometry, weights and device coefficient pointers.
struct ImageSpec {
    uint32_t nch;
    const ArtChannel *ch;
    const void *src[3];
    float weight;
    float pweight[3];
    uint32_t W, H;
};

}  // namespace

// Launch shapes of one geometry bucket: gradient-sweep variant (0 narrow, 1
// wide), strip rows, projection warps per block.
struct TuneChoice {
    int kind = 0, rows = 0, proj_warps = PROJ_WARPS;
};

}  // namespace art

struct ArtContext {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;      // second stream: projections of different sampling modes run side by side
    cudaEvent_t fork = nullptr, join = nullptr;
    art::DevBuf xbuf, pbuf, coefimg, stage, misc, desc, work, tasks, compat, sepplanes, rgb, pred;
    art::HostBuf hstage, hrgb;        // pinned host staging of art_context_process_batch
    ArtNet *net = nullptr;            // warm-start network for ART_INIT_LEARNED (not owned)
    ArtNet *net_joint = nullptr;      // joint 4:2:0 warm-start network, used for 4:2:0 images (not owned)
    // The learned start's launches (network, upsampling, zero-step projection)
    // as a graph: captured the second time one key is seen, then replayed.
    cudaGraphExec_t init_exec = nullptr;
    std::vector<unsigned long long> init_key, init_seen;
    bool net_used = false;            // the last solve ran the network (its error flag is checked)
    std::vector<art::ImgDev> h_desc;  // per image (pageable: copies of it are staged)
    std::vector<std::array<float, 4>> h_weights;  // per image: weight, pweight[3]
    art::DevBuf evalbuf;              // partial sums of art_context_evaluate
    std::vector<int2> h_work;         // sweep blocks {image, block in image}, grouped by variant and channel count
    int wstart[3][4] = {}, wcount[3][4] = {};  // by sweep variant (0 narrow, 1 wide, 2 quad) and channel count
    std::vector<int4> h_tasks;        // block warps {image, channel, block row, first block}
    std::vector<long long> geo_key;   // geometry h_work / h_tasks (and their device copies) were built for
    int mode_off[5] = {0, 0, 0, 0, 0};  // h_tasks grouped by sampling mode (1x1, 2x2, 2x1, 1x2)
    unsigned *errflag = nullptr;
    cudaGraphExec_t exec = nullptr;
    art::GraphKey key;
    bool timing = false;
    std::vector<cudaEvent_t> events;  // [0,1] loop; then 4 per iteration
    uint32_t timed_iterations = 0;
    int strip_rows_override = 0;      // 0 = tuning cache, else size heuristic
    int sweep_kind_override = 0;
    int proj_warps = art::PROJ_WARPS; // projection warps per block of the current solve
    int proj_warps_override = 0;      // set while the autotuner times a candidate
    std::map<std::string, art::TuneChoice> tune;  // autotuned launch shapes by geometry bucket
    ArtTuneResult last_tune{};        // the last autotune run's choice and timings
    std::vector<ArtTuneCandidate> tune_log;  // every candidate the last autotune run timed
};

namespace art {
namespace {

int pow2_bucket(uint32_t v)
{
    int b = 256;
    while ((uint32_t)b < v && b < 65536) b *= 2;
    return b;
}

// Key of a geometry bucket for the autotuner: channel count, sampling of
// each channel, width and height rounded up to a power of two.
std::string tune_key(uint32_t nch, const uint32_t *sh, const uint32_t *sv, uint32_t W, uint32_t H)
{
    std::string k = "n" + std::to_string(nch) + "-s";
    for (uint32_t c = 0; c < nch; c++) k += std::to_string(sh[c]) + std::to_string(sv[c]);
    k += "-w" + std::to_string(pow2_bucket(W)) + "-h" + std::to_string(pow2_bucket(H));
    return k;
}

// Key of a whole batch (more than one image) for the autotuner: image count
// and total pixels, each rounded up to a power of two.
std::string batch_tune_key(int nimg, long long batch_px)
{
    long long n = 1, px = 1 << 20;
    while (n < nimg) n *= 2;
    while (px < batch_px) px *= 2;
    return "batch-i" + std::to_string(n) + "-p" + std::to_string(px);
}

// Launch shapes for one image of a solve of `nimg` images: environment
// overrides (ART_SWEEP_KIND, ART_STRIP_ROWS, ART_PROJ_WARPS), the candidate
// the autotuner is timing, the autotuner's choice for the batch's bucket
// (several images) or the image's bucket (one image), else by size -- the
// narrow sweep (with its packed channel pair it is the fastest variant from
// 1080p to 6000x4000 and on the 256-image batch), strips as tall as still
// give every SM a dozen warps (the 3 extra rows a strip reads stay small), and
// 4 projection warps per block.
TuneChoice pick_shape(const ArtContext *ctx, const ImageSpec &sp, long long batch_px, int nimg)
{
    TuneChoice t;
    t.kind = 0;
    if (ctx->strip_rows_override > 0) {
        t.kind = ctx->sweep_kind_override;
        t.rows = ctx->strip_rows_override;
        t.proj_warps = ctx->proj_warps_override > 0 ? ctx->proj_warps_override : PROJ_WARPS;
        return t;
    }
    const char *ek = getenv("ART_SWEEP_KIND");
    const char *er = getenv("ART_STRIP_ROWS");
    const char *ep = getenv("ART_PROJ_WARPS");
    const int env_pw = ep ? atoi(ep) : 0;
    const bool env_pw_ok = env_pw == 2 || env_pw == 4 || env_pw == 8;
    if (ek && atoi(ek) >= 0 && atoi(ek) <= 2) t.kind = atoi(ek);
    if (er && atoi(er) > 0) {
        t.rows = atoi(er);
        if (env_pw_ok) t.proj_warps = env_pw;
        return t;
    }
    std::map<std::string, TuneChoice>::const_iterator it = ctx->tune.end();
    if (nimg > 1) it = ctx->tune.find(batch_tune_key(nimg, batch_px));
    if (it == ctx->tune.end()) {
        uint32_t sh[3], sv[3];
        for (uint32_t c = 0; c < sp.nch; c++) {
            sh[c] = sp.ch[c].samp_h;
            sv[c] = sp.ch[c].samp_v;
        }
        it = ctx->tune.find(tune_key(sp.nch, sh, sv, sp.W, sp.H));
    }
    if (it != ctx->tune.end()) {
        t = it->second;
        if (env_pw_ok) t.proj_warps = env_pw;
        return t;
    }
    const long long cols = t.kind == 2 ? SWEEP_OUT_Q : t.kind == 1 ? SWEEP_OUT : SWEEP_OUT_N;
    int R = 128;
    while (R > 16 && batch_px / (cols * R) < 148LL * 12) R /= 2;
    t.rows = R;
    if (env_pw_ok) t.proj_warps = env_pw;
    return t;
}

template <int SH, int SV, int PW = PROJ_WARPS>
constexpr int proj_smem()
{
    return PW * 2 * ProjShape<SH, SV>::REGION * (int)sizeof(float);
}

// Projection block shapes the autotuner may choose: warps per block (each
// warp takes 4 coefficient blocks of one block row).
constexpr int PROJ_WARP_CHOICES[3] = {2, 4, 8};

template <int PW>
static cudaError_t set_proj_smem()
{
    cudaError_t e = cudaFuncSetAttribute(k_project<1, 1, PW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         proj_smem<1, 1, PW>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_project<2, 2, PW>, cudaFuncAttributeMaxDynamicSharedMemorySize, proj_smem<2, 2, PW>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_project<2, 1, PW>, cudaFuncAttributeMaxDynamicSharedMemorySize, proj_smem<2, 1, PW>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_project<1, 2, PW>, cudaFuncAttributeMaxDynamicSharedMemorySize, proj_smem<1, 2, PW>());
    return e;
}

// One projection launch over n tasks of sampling mode m with PW warps per block.
template <int PW>
static void launch_project_mode(int m, int n, const ImgDev *ddesc, const int4 *tk, float fnext, cudaStream_t s)
{
    const int grid = (n + PW - 1) / PW;
    if (m == 0)
        k_project<1, 1, PW><<<grid, PW * 32, proj_smem<1, 1, PW>(), s>>>(ddesc, tk, n, fnext);
    else if (m == 1)
        k_project<2, 2, PW><<<grid, PW * 32, proj_smem<2, 2, PW>(), s>>>(ddesc, tk, n, fnext);
    else if (m == 2)
        k_project<2, 1, PW><<<grid, PW * 32, proj_smem<2, 1, PW>(), s>>>(ddesc, tk, n, fnext);
    else
        k_project<1, 2, PW><<<grid, PW * 32, proj_smem<1, 2, PW>(), s>>>(ddesc, tk, n, fnext);
}

static void launch_project(int pw, int m, int n, const ImgDev *ddesc, const int4 *tk, float fnext, cudaStream_t s)
{
    if (pw == 2)
        launch_project_mode<2>(m, n, ddesc, tk, fnext, s);
    else if (pw == 8)
        launch_project_mode<8>(m, n, ddesc, tk, fnext, s);
    else
        launch_project_mode<4>(m, n, ddesc, tk, fnext, s);
}

// Raises the dynamic shared-memory limit of the projection kernels, once per device.
int configure_kernels(int device)
{
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)done.size() <= device) done.resize(device + 1, 0);
    if (done[device]) return ART_OK;
    cudaError_t e = set_proj_smem<2>();
    if (e == cudaSuccess) e = set_proj_smem<4>();
    if (e == cudaSuccess) e = set_proj_smem<8>();
    if (e != cudaSuccess) return fail(ART_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    done[device] = 1;
    return ART_OK;
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
    if (3LL * (long long)align_up(W, 32) * (long long)align_up(H, 32) >= (1LL << 31))
        return fail(ART_ERR_INVALID_ARGUMENT, "image too large: three padded planes must stay below 2^31 floats");
    return ART_OK;
}

}  // namespace

// Sampling mode of a component: 0 = 1x1, 1 = 2x2, 2 = 2x1 (h x v), 3 = 1x2.
static int samp_mode(int sh, int sv) { return sh == 1 ? (sv == 1 ? 0 : 3) : (sv == 2 ? 1 : 2); }

// Block tasks of one image appended per sampling mode; inside a mode bottom
// rows first and channels interleaved by full-resolution row band, so the
// projection starts on the rows the gradient sweep touched last (still in L2).
static void build_tasks(const ImgDev &d, int img, std::vector<int4> per_mode[4])
{
    // Each channel's block rows, walked from the bottom, are already in
    // descending row order; merging the channels (ties to the lower channel)
    // gives the order in linear time.
    int by[3], mode[3];
    for (int c = 0; c < d.nch; c++) {
        by[c] = d.ch[c].chh / 8 - 1;
        mode[c] = samp_mode(d.ch[c].sh, d.ch[c].sv);
    }
    for (;;) {
        int best = -1, row = -1;
        for (int c = 0; c < d.nch; c++) {
            if (by[c] < 0) continue;
            const int r = by[c] * 8 * d.ch[c].sv;
            if (r > row) {
                row = r;
                best = c;
            }
        }
        if (best < 0) break;
        const int bw = d.ch[best].cw / 8;
        for (int bx0 = 0; bx0 < bw; bx0 += 4) per_mode[mode[best]].push_back(make_int4(img, best, by[best], bx0));
        by[best]--;
    }
}

// Step + projection of every image, one launch per sampling mode present.
// The launches touch disjoint channels, so with more than one mode the
// subsampled modes run on the side stream, concurrently with the full-
// resolution one (a fork and join inside the captured graph).
static void launch_projections(ArtContext *ctx, float fnext)
{
    const ImgDev *ddesc = static_cast<const ImgDev *>(ctx->desc.p);
    const int4 *tasks = static_cast<const int4 *>(ctx->tasks.p);
    int modes = 0;
    for (int m = 0; m < 4; m++) modes += ctx->mode_off[m + 1] > ctx->mode_off[m];
    const bool split = modes > 1 && ctx->mode_off[1] > ctx->mode_off[0];
    if (split) {
        cudaEventRecord(ctx->fork, ctx->stream);
        cudaStreamWaitEvent(ctx->side, ctx->fork, 0);
    }
    for (int m = 3; m >= 0; m--) {
        const int n = ctx->mode_off[m + 1] - ctx->mode_off[m];
        if (n == 0) continue;
        cudaStream_t s = split && m > 0 ? ctx->side : ctx->stream;
        launch_project(ctx->proj_warps, m, n, ddesc, tasks + ctx->mode_off[m], fnext, s);
    }
    if (split) {
        cudaEventRecord(ctx->join, ctx->side);
        cudaStreamWaitEvent(ctx->stream, ctx->join, 0);
    }
}

// Lays out the buffers of a batch of images, uploads descriptors and work
// lists, ingests coefficients and queues the initialisation.
static int prepare_batch(ArtContext *ctx, const std::vector<ImageSpec> &specs, uint32_t iterations, int init_mode,
                         uint32_t step_iterations)
{
    if (init_mode == ART_INIT_LEARNED && !ctx->net && !ctx->net_joint)
        return fail(ART_ERR_INVALID_ARGUMENT, "learned start: no network attached");
    const uint32_t step_its = step_iterations ? step_iterations : iterations;
    int rc;
    const int nimg = (int)specs.size();
    long long batch_px = 0;
    for (const auto &sp : specs) batch_px += (long long)sp.W * sp.H;
    std::vector<size_t> o_x(nimg), o_misc(nimg);
    std::vector<std::array<size_t, 3>> o_coef(nimg), o_p(nimg);
    size_t x_floats = 0, coef_bytes = 0, p_floats = 0, misc_bytes = 256;  // misc starts with the error flag
    ctx->h_desc.assign(nimg, ImgDev());
    ctx->h_weights.assign(nimg, std::array<float, 4>{});
    for (int i = 0; i < nimg; i++) {
        const ImageSpec &sp = specs[i];
        ImgDev &d = ctx->h_desc[i];
        memset(&d, 0, sizeof(d));
        ctx->h_weights[i] = {sp.weight, sp.pweight[0], sp.pweight[1], sp.pweight[2]};
        const int pitch = (int)align_up(sp.W, 32);
        const long long cstride = (long long)pitch * (long long)align_up(sp.H, 32);
        const TuneChoice sw = pick_shape(ctx, sp, batch_px, nimg);
        if (i == 0) ctx->proj_warps = sw.proj_warps;
        const int R = sw.rows;
        const int out_cols = sw.kind == 2 ? SWEEP_OUT_Q : sw.kind == 1 ? SWEEP_OUT : SWEEP_OUT_N;
        const int warps = sw.kind == 2 ? SWEEP_WARPS_Q : sw.kind == 1 ? SWEEP_WARPS : SWEEP_WARPS_N;
        d.nch = (int)sp.nch;
        d.W = (int)sp.W;
        d.H = (int)sp.H;
        d.pitch = pitch;
        d.sweep_kind = sw.kind;
        d.strip_rows = R;
        d.strips_x = (int)((sp.W + out_cols - 1) / out_cols);
        d.strips_y = (int)((sp.H + R - 1) / R);
        d.nstrips = d.strips_x * d.strips_y;
        d.ncta = (d.nstrips + warps - 1) / warps;
        d.cstride = cstride;
        // compute_step_tv.rs:130 and compute_step_tv2.rs:88-89, compute_step.rs:47.
        d.alpha_tv = 1.0f / sqrtf((float)sp.nch);
        d.alpha_tgv = (sp.weight / sqrtf(2.0f)) / sqrtf((float)sp.nch);
        // mod.rs:45 and :71.
        d.step = (sqrtf((float)((uint64_t)sp.W * sp.H)) / 2.0f) / sqrtf(1.0f + (float)step_its);
        o_x[i] = x_floats;
        x_floats += align_up((size_t)3 * sp.nch * cstride, 64);
        o_misc[i] = misc_bytes;
        misc_bytes += align_up((size_t)d.ncta * 4 * sizeof(float), 256) + 256;
        for (uint32_t c = 0; c < sp.nch; c++) {
            ChanDev &cd = d.ch[c];
            cd.cw = (int)sp.ch[c].rounded_px_w;
            cd.chh = (int)sp.ch[c].rounded_px_h;
            cd.sh = (int)sp.ch[c].samp_h;
            cd.sv = (int)sp.ch[c].samp_v;
            cd.cpitch = (int)align_up(cd.cw, 64);
            cd.ppitch = (int)align_up(cd.cw, 32);
            // compute_step.rs:20-31: alpha = pweight * 2 * 255 * sqrt(2).
            cd.alpha_p = sp.pweight[c] * 2.0f * 255.0f * sqrtf(2.0f);
            o_coef[i][c] = coef_bytes;
            coef_bytes += align_up((size_t)cd.cpitch * cd.chh * sizeof(int16_t), 256);
            o_p[i][c] = p_floats;
            p_floats += align_up((size_t)cd.ppitch * cd.chh, 64);
            for (int j = 0; j < 64; j++) {
                const float q = sp.ch[c].quant_table[j];
                d.q[c][j] = q;
                d.invq2[c][j] = 1.0f / (q * q);
            }
        }
    }
    if ((rc = ctx->xbuf.ensure(x_floats * sizeof(float)))) return rc;
    if ((rc = ctx->coefimg.ensure(coef_bytes))) return rc;
    if ((rc = ctx->pbuf.ensure(p_floats * sizeof(float)))) return rc;
    if ((rc = ctx->misc.ensure(misc_bytes))) return rc;
    if ((rc = ctx->desc.ensure(nimg * sizeof(ImgDev)))) return rc;
    float *xb = static_cast<float *>(ctx->xbuf.p);
    char *misc = static_cast<char *>(ctx->misc.p);
    ctx->errflag = reinterpret_cast<unsigned *>(misc);
    // The sweep blocks and projection tasks depend on the geometry alone: a
    // solve with the geometry of the previous one reuses them (host lists and
    // device copies) instead of rebuilding and uploading ~16 B per 4 blocks.
    std::vector<long long> geo = {nimg};
    for (int i = 0; i < nimg; i++) {
        const ImgDev &d = ctx->h_desc[i];
        geo.insert(geo.end(), {d.W, d.H, d.nch, d.sweep_kind, d.strip_rows});
        for (int c = 0; c < d.nch; c++) geo.insert(geo.end(), {d.ch[c].cw, d.ch[c].chh, d.ch[c].sh, d.ch[c].sv});
    }
    const bool same_geo = geo == ctx->geo_key && ctx->work.p && ctx->tasks.p;
    std::vector<int2> wk[3][4];
    std::vector<int4> per_mode[4];
    for (int i = 0; i < nimg; i++) {
        ImgDev &d = ctx->h_desc[i];
        d.x = xb + o_x[i];
        d.y = d.x + d.nch * d.cstride;
        d.g = d.y + d.nch * d.cstride;
        d.partial = reinterpret_cast<float *>(misc + o_misc[i]);
        d.sigma = reinterpret_cast<float *>(misc + o_misc[i] + align_up((size_t)d.ncta * 4 * sizeof(float), 256));
        d.counter = reinterpret_cast<unsigned *>(d.sigma + 4);
        for (int c = 0; c < d.nch; c++) {
            d.ch[c].coef = reinterpret_cast<const int16_t *>(static_cast<char *>(ctx->coefimg.p) + o_coef[i][c]);
            d.ch[c].P = static_cast<float *>(ctx->pbuf.p) + o_p[i][c];
        }
        if (same_geo) continue;
        for (int b = 0; b < d.ncta; b++) wk[d.sweep_kind][d.nch].push_back(make_int2(i, b));
        build_tasks(d, i, per_mode);
    }
    cudaStream_t s = ctx->stream;
    if (!same_geo) {
        ctx->geo_key.clear();
        ctx->h_work.clear();
        for (int kd = 0; kd < 3; kd++)
            for (int n = 3; n >= 1; n--) {
                ctx->wstart[kd][n] = (int)ctx->h_work.size();
                ctx->wcount[kd][n] = (int)wk[kd][n].size();
                ctx->h_work.insert(ctx->h_work.end(), wk[kd][n].begin(), wk[kd][n].end());
            }
        ctx->h_tasks.clear();
        for (int m = 0; m < 4; m++) {
            ctx->mode_off[m] = (int)ctx->h_tasks.size();
            ctx->h_tasks.insert(ctx->h_tasks.end(), per_mode[m].begin(), per_mode[m].end());
        }
        ctx->mode_off[4] = (int)ctx->h_tasks.size();
        const int nwork = (int)ctx->h_work.size(), ntasks = (int)ctx->h_tasks.size();
        if ((rc = ctx->work.ensure(nwork * sizeof(int2)))) return rc;
        if ((rc = ctx->tasks.ensure(ntasks * sizeof(int4)))) return rc;
        ART_CUDA(cudaMemcpyAsync(ctx->work.p, ctx->h_work.data(), nwork * sizeof(int2), cudaMemcpyHostToDevice, s));
        ART_CUDA(cudaMemcpyAsync(ctx->tasks.p, ctx->h_tasks.data(), ntasks * sizeof(int4), cudaMemcpyHostToDevice, s));
        ctx->geo_key = geo;
    }
    const int ntasks = (int)ctx->h_tasks.size();
    ART_CUDA(cudaMemcpyAsync(ctx->desc.p, ctx->h_desc.data(), nimg * sizeof(ImgDev), cudaMemcpyHostToDevice, s));
    ART_CUDA(cudaMemsetAsync(ctx->misc.p, 0, misc_bytes, s));
    // The first DCT-distance gradient is zero: the reference starts from cos = c q (coef.rs:94-104).
    ART_CUDA(cudaMemsetAsync(ctx->pbuf.p, 0, p_floats * sizeof(float), s));
    const ImgDev *ddesc = static_cast<const ImgDev *>(ctx->desc.p);
    for (int i = 0; i < nimg; i++) {
        const ImageSpec &sp = specs[i];
        for (uint32_t c = 0; c < sp.nch; c++) {
            const long long ncoef = (long long)sp.ch[c].block_w * sp.ch[c].block_h * 64;
            k_ingest<<<(int)((ncoef + 255) / 256), 256, 0, s>>>(
                sp.src[c], (int)sp.ch[c].coef_type, (int)sp.ch[c].block_w, ncoef,
                const_cast<int16_t *>(ctx->h_desc[i].ch[c].coef), ctx->h_desc[i].ch[c].cpitch, ctx->errflag);
        }
    }
    if (init_mode == ART_INIT_SCALAR_COMPAT) {
        size_t need = 0;
        for (const auto &sp : specs)
            for (uint32_t c = 0; c < sp.nch; c++)
                need = std::max(need, (size_t)sp.ch[c].rounded_px_w * sp.ch[c].rounded_px_h);
        if ((rc = ctx->compat.ensure(2 * need * sizeof(float)))) return rc;
        for (int i = 0; i < nimg; i++) {
            const ImageSpec &sp = specs[i];
            for (uint32_t c = 0; c < sp.nch; c++) {
                const long long nc = (long long)sp.ch[c].rounded_px_w * sp.ch[c].rounded_px_h;
                float *a = static_cast<float *>(ctx->compat.p), *b = a + need;
                ART_CUDA(cudaMemsetAsync(a, 0, nc * sizeof(float), s));
                const int nb = (int)(sp.ch[c].block_w * sp.ch[c].block_h);
                const int grid = (int)((nc + 255) / 256);
                for (int blk = 0; blk < nb; blk++) {
                    k_compat_step<<<grid, 256, 0, s>>>(a, b, ddesc + i, (int)c, blk, nc);
                    std::swap(a, b);
                }
                k_upsample<<<(int)(((long long)sp.W * sp.H + 255) / 256), 256, 0, s>>>(a, ddesc + i, (int)c);
            }
        }
    } else if (init_mode == ART_INIT_LEARNED) {
        // Prediction per component at its own resolution, upsampled smoothly
        // to full resolution into x and y, then one projection with a zero step
        // (sigma = 0): x_0 = y_0 = P(prediction), and the DCT-distance plane of
        // the projected prediction for the first gradient.
        // A 4:2:0 image (luma H x W, both chroma H/2 x W/2, H and W multiples
        // of 16) goes through the joint network when one is attached: one
        // pass predicts all three components at full resolution.
        auto joint_ok = [&](int i) {
            const ImgDev &d = ctx->h_desc[i];
            if (!ctx->net_joint || d.nch != 3 || d.W % 16 || d.H % 16) return false;
            const ChanDev *ch = d.ch;
            return ch[0].sh == 1 && ch[0].sv == 1 && ch[0].cw == d.W && ch[0].chh == d.H && ch[1].sh == 2 &&
                   ch[1].sv == 2 && ch[2].sh == 2 && ch[2].sv == 2 && ch[1].cw * 2 == d.W && ch[1].chh * 2 == d.H &&
                   ch[2].cw == ch[1].cw && ch[2].chh == ch[1].chh && ch[2].cpitch == ch[1].cpitch;
        };
        size_t need = 0;
        for (int i = 0; i < nimg; i++) {
            const ImageSpec &sp = specs[i];
            size_t img = 0;
            for (uint32_t c = 0; c < sp.nch; c++) img += (size_t)sp.ch[c].rounded_px_w * sp.ch[c].rounded_px_h;
            need = std::max(need, img);
        }
        if ((rc = ctx->pred.ensure(need * sizeof(float)))) return rc;
        float *pred = static_cast<float *>(ctx->pred.p);
        // Components of one size (the two chroma planes of 4:2:0 or 4:2:2) go
        // through the network as one batch: their coefficient images lie a
        // fixed distance apart and their quantisation tables are consecutive
        // in the descriptor.
        // Groups alternate between the network's two activation sets and the
        // context's two streams (luma and chroma of one image run side by side;
        // each group's prediction has its own region of `pred`, by channel).
        struct Group {
            int i, c, nb;
            long long stride;
            size_t poff;
            bool joint;
        };
        std::vector<Group> groups;
        for (int i = 0; i < nimg; i++) {
            const ImgDev &d = ctx->h_desc[i];
            if (joint_ok(i)) {
                const int slot = (int)(groups.size() % 2);
                groups.push_back({i, 0, 3, (long long)(d.ch[2].coef - d.ch[1].coef), 0, true});
                if ((rc = cnn::net_prepare_joint(ctx->net_joint, slot, d.H, d.W, s))) return rc;
                continue;
            }
            if (!ctx->net)
                return fail(ART_ERR_INVALID_ARGUMENT,
                            "learned start: no network attached for an image that is not 4:2:0 (art_context_set_warm_start)");
            size_t poff = 0;
            for (int c = 0; c < d.nch;) {
                const ChanDev &cd = d.ch[c];
                const long long stride = c + 1 < d.nch ? (long long)(d.ch[c + 1].coef - cd.coef) : 0;
                int nb = 1;
                while (c + nb < d.nch && d.ch[c + nb].cw == cd.cw && d.ch[c + nb].chh == cd.chh &&
                       d.ch[c + nb].cpitch == cd.cpitch && d.ch[c + nb].coef - d.ch[c + nb - 1].coef == stride)
                    nb++;
                const int slot = (int)(groups.size() % 2);
                groups.push_back({i, c, nb, stride, poff, false});
                if ((rc = cnn::net_prepare(ctx->net, slot, nb, cd.chh, cd.cw, s))) return rc;
                poff += (size_t)nb * cd.cw * cd.chh;
                c += nb;
            }
        }
        // Everything the launches below bake in: buffers, geometry, tasks.
        auto gen = [](ArtNet *n, int slot) { return n ? cnn::net_generation(n, slot) : 0ull; };
        std::vector<unsigned long long> key = {
            (unsigned long long)(uintptr_t)ctx->net, gen(ctx->net, 0), gen(ctx->net, 1),
            (unsigned long long)(uintptr_t)ctx->net_joint, gen(ctx->net_joint, 0), gen(ctx->net_joint, 1),
            (uintptr_t)ctx->desc.p, (uintptr_t)ctx->tasks.p, (uintptr_t)pred, (uintptr_t)ctx->xbuf.p,
            (uintptr_t)ctx->coefimg.p, (unsigned long long)nimg, (unsigned long long)ctx->proj_warps};
        for (int m = 0; m < 5; m++) key.push_back((unsigned long long)ctx->mode_off[m]);
        for (int i = 0; i < nimg; i++) {
            const ImgDev &d = ctx->h_desc[i];
            key.insert(key.end(), {(unsigned long long)d.W, (unsigned long long)d.H, (unsigned long long)d.nch,
                                   (unsigned long long)d.cstride, (uintptr_t)d.g});
            for (int c = 0; c < d.nch; c++)
                key.insert(key.end(), {(unsigned long long)d.ch[c].cw, (unsigned long long)d.ch[c].chh,
                                       (unsigned long long)d.ch[c].cpitch, (uintptr_t)d.ch[c].coef});
        }
        // Prediction per component at its own resolution, upsampled smoothly
        // to full resolution into x and y, then one projection with a zero step
        // (sigma = 0): x_0 = y_0 = P(prediction), and the DCT-distance plane of
        // the projected prediction for the first gradient.
        auto launch_init = [&]() -> int {
            if (groups.size() > 1) {
                ART_CUDA(cudaEventRecord(ctx->fork, s));
                ART_CUDA(cudaStreamWaitEvent(ctx->side, ctx->fork, 0));
            }
            for (size_t g = 0; g < groups.size(); g++) {
                const Group &gr = groups[g];
                const int slot = (int)(g % 2);
                cudaStream_t gs = slot ? ctx->side : s;
                const ImgDev &d = ctx->h_desc[gr.i];
                const ChanDev &cd = d.ch[gr.c];
                float *gp = pred + gr.poff;
                if (gr.joint) {
                    const int r = cnn::net_predict_joint_async(ctx->net_joint, slot, cd.coef, cd.cpitch, 0,
                                                               d.ch[1].coef, d.ch[1].cpitch, gr.stride,
                                                               &ddesc[gr.i].q[0][0], &ddesc[gr.i].q[1][0], d.H, d.W,
                                                               d.x, d.y, d.cstride, d.pitch, gs);
                    if (r) return r;
                    continue;
                }
                const int r = cnn::net_predict_async(ctx->net, slot, cd.coef, cd.cpitch, gr.stride,
                                                     &ddesc[gr.i].q[gr.c][0], gr.nb, cd.chh, cd.cw, gp, gs);
                if (r) return r;
                for (int k = 0; k < gr.nb; k++)
                    k_upsample_smooth<<<(int)(((long long)d.W * d.H + 255) / 256), 256, 0, gs>>>(
                        gp + (size_t)k * cd.cw * cd.chh, ddesc + gr.i, gr.c + k);
            }
            if (groups.size() > 1) {
                ART_CUDA(cudaEventRecord(ctx->join, ctx->side));
                ART_CUDA(cudaStreamWaitEvent(s, ctx->join, 0));
            }
            // sigma is zero (misc was cleared): the projections neither read
            // nor need g here.
            launch_projections(ctx, 0.0f);
            ART_CUDA(cudaGetLastError());
            return ART_OK;
        };
        if (ctx->init_exec && key == ctx->init_key) {
            ART_CUDA(cudaGraphLaunch(ctx->init_exec, s));
        } else if (key == ctx->init_seen) {
            if (ctx->init_exec) {
                cudaGraphExecDestroy(ctx->init_exec);
                ctx->init_exec = nullptr;
            }
            ctx->init_key.clear();
            cudaGraph_t graph = nullptr;
            ART_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            const int r = launch_init();
            const cudaError_t ce = cudaStreamEndCapture(s, &graph);
            if (r) {
                if (graph) cudaGraphDestroy(graph);
                return r;
            }
            if (ce != cudaSuccess) return fail(ART_ERR_CUDA, std::string("learned start capture: ") + cudaGetErrorString(ce));
            const cudaError_t ie = cudaGraphInstantiate(&ctx->init_exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ie != cudaSuccess) {
                ctx->init_exec = nullptr;
                return fail(ART_ERR_CUDA, std::string("learned start graph: ") + cudaGetErrorString(ie));
            }
            ctx->init_key = key;
            ART_CUDA(cudaGraphLaunch(ctx->init_exec, s));
        } else {
            if ((rc = launch_init())) return rc;
            ctx->init_seen = key;
        }
        ctx->net_used = true;
    } else {
        k_init<<<(ntasks + PROJ_WARPS - 1) / PROJ_WARPS, PROJ_WARPS * 32, 0, s>>>(
            ddesc, static_cast<const int4 *>(ctx->tasks.p), ntasks);
    }
    ART_CUDA(cudaGetLastError());
    return ART_OK;
}

// One iteration: the gradient sweeps (sigma = step * stepmul / ||g||) and the
// projections forming y_{k+1} with FISTA factor fnext.
static void launch_iteration(ArtContext *ctx, int it, float fnext, float stepmul)
{
    const ImgDev *ddesc = static_cast<const ImgDev *>(ctx->desc.p);
    const int2 *work = static_cast<const int2 *>(ctx->work.p);
    cudaStream_t s = ctx->stream;
    const bool tm = ctx->timing;
    if (tm) cudaEventRecordWithFlags(ctx->events[2 + 4 * it], s, cudaEventRecordExternal);
    if (ctx->wcount[1][3])
        k_grad_sweep<3><<<ctx->wcount[1][3], SWEEP_WARPS * 32, 0, s>>>(ddesc, work + ctx->wstart[1][3], stepmul);
    if (ctx->wcount[1][2])
        k_grad_sweep<2><<<ctx->wcount[1][2], SWEEP_WARPS * 32, 0, s>>>(ddesc, work + ctx->wstart[1][2], stepmul);
    if (ctx->wcount[1][1])
        k_grad_sweep<1><<<ctx->wcount[1][1], SWEEP_WARPS * 32, 0, s>>>(ddesc, work + ctx->wstart[1][1], stepmul);
    if (ctx->wcount[2][3])
        k_grad_sweep_q<3><<<ctx->wcount[2][3], SWEEP_WARPS_Q * 32, 0, s>>>(ddesc, work + ctx->wstart[2][3], stepmul);
    if (ctx->wcount[2][2])
        k_grad_sweep_q<2><<<ctx->wcount[2][2], SWEEP_WARPS_Q * 32, 0, s>>>(ddesc, work + ctx->wstart[2][2], stepmul);
    if (ctx->wcount[2][1])
        k_grad_sweep_q<1><<<ctx->wcount[2][1], SWEEP_WARPS_Q * 32, 0, s>>>(ddesc, work + ctx->wstart[2][1], stepmul);
    if (ctx->wcount[0][3])
        k_grad_sweep_n<3><<<ctx->wcount[0][3], SWEEP_WARPS_N * 32, 0, s>>>(ddesc, work + ctx->wstart[0][3], stepmul);
    if (ctx->wcount[0][2])
        k_grad_sweep_n<2><<<ctx->wcount[0][2], SWEEP_WARPS_N * 32, 0, s>>>(ddesc, work + ctx->wstart[0][2], stepmul);
    if (ctx->wcount[0][1])
        k_grad_sweep_n<1><<<ctx->wcount[0][1], SWEEP_WARPS_N * 32, 0, s>>>(ddesc, work + ctx->wstart[0][1], stepmul);
    if (tm) cudaEventRecordWithFlags(ctx->events[3 + 4 * it], s, cudaEventRecordExternal);
    if (tm) cudaEventRecordWithFlags(ctx->events[4 + 4 * it], s, cudaEventRecordExternal);
    launch_projections(ctx, fnext);
    if (tm) cudaEventRecordWithFlags(ctx->events[5 + 4 * it], s, cudaEventRecordExternal);
}

// Replays (capturing first if the work changed shape) the fixed-count
// iteration loop as one CUDA graph.
static int run_iterations(ArtContext *ctx, uint32_t iterations, uint32_t tail = 0, float tail_stepmul = 1.0f,
                          float decay = 0.0f)
{
    if (iterations == 0) return ART_OK;
    tail = std::min(tail, iterations);
    if (ctx->timing) {
        const size_t need = 2 + 4 * (size_t)iterations;
        while (ctx->events.size() < need) {
            cudaEvent_t e;
            ART_CUDA(cudaEventCreate(&e));
            ctx->events.push_back(e);
        }
    }
    GraphKey key;
    key.nimg = (int)ctx->h_desc.size();
    key.proj_warps = ctx->proj_warps;
    std::copy(&ctx->wcount[0][0], &ctx->wcount[0][0] + 12, key.wcount);
    std::copy(ctx->mode_off, ctx->mode_off + 5, key.mode_off);
    key.iterations = iterations;
    key.tail = tail;
    key.tail_stepmul = tail_stepmul;
    key.decay = decay;
    key.timing = ctx->timing;
    key.desc = ctx->desc.p;
    key.work = ctx->work.p;
    key.tasks = ctx->tasks.p;
    cudaStream_t s = ctx->stream;
    if (!ctx->exec || !(ctx->key == key)) {
        if (ctx->exec) {
            cudaGraphExecDestroy(ctx->exec);
            ctx->exec = nullptr;
        }
        // Two phases: iterations - tail steps of the solve's own size, then
        // `tail` steps of tail_stepmul times that size with the FISTA sequence
        // restarted (the last step of the first phase forms y = x). Without a
        // tail this is the reference's loop (mod.rs:49-75).
        const uint32_t k1 = iterations - tail;
        const std::vector<float> fs1 = fista_factors(k1), fs2 = fista_factors(tail);
        cudaGraph_t graph;
        ART_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        if (ctx->timing) cudaEventRecordWithFlags(ctx->events[0], s, cudaEventRecordExternal);
        // y_0 = x_0 (f_0 = 0); the projection of iteration k forms y_{k+1} with f_{k+1}.
        // With decay > 0 the first phase's steps shrink geometrically: step
        // k of that phase is decay^k times the solve's step (fp32 product).
        float mul = 1.0f;
        for (uint32_t it = 0; it < iterations; it++) {
            if (it < k1) {
                launch_iteration(ctx, (int)it, it + 1 < k1 ? fs1[it + 1] : 0.0f, mul);
                if (decay > 0.0f) mul *= decay;
            } else {
                launch_iteration(ctx, (int)it, it - k1 + 1 < tail ? fs2[it - k1 + 1] : 0.0f, tail_stepmul);
            }
        }
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

// Result planes of image i: base pointer, pitch and channel stride.
static void result_planes(const ArtContext *ctx, int i, const float **base, int *pitch, long long *cstride)
{
    const ImgDev &d = ctx->h_desc[i];
    *base = d.x;
    *pitch = d.pitch;
    *cstride = d.cstride;
}

static int check_errflag(ArtContext *ctx)
{
    if (!ctx->errflag) return ART_OK;
    unsigned flag = 0;
    ART_CUDA(cudaMemcpy(&flag, ctx->errflag, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (flag) return fail(ART_ERR_INVALID_DATA, "coefficients must be integers in [-32768, 32767]");
    if (ctx->net_used && ctx->net) {
        const int r = cnn::net_error(ctx->net);
        if (r) return r;
    }
    if (ctx->net_used && ctx->net_joint) return cnn::net_error(ctx->net_joint);
    return ART_OK;
}

// Start mode and step schedule of a solve.
struct InitSpec {
    int mode = ART_INIT_DECODED;
    uint32_t step_iterations = 0;
    uint32_t tail_iterations = 0, tail_step_iterations = 0;
    float step_decay = 0.0f;  // > 0: first-phase steps shrink by this factor per iteration
    // Step of the tail phase relative to the first phase's, for `iterations` in all.
    float tail_stepmul(uint32_t iterations) const
    {
        if (!tail_iterations || !tail_step_iterations) return 1.0f;
        const float s1 = (float)(step_iterations ? step_iterations : iterations);
        return sqrtf(1.0f + s1) / sqrtf(1.0f + (float)tail_step_iterations);
    }
};

static int init_spec(const ArtContext *ctx, const ArtOptions *opts, InitSpec *out)
{
    out->mode = opts ? (int)opts->init_mode : ART_INIT_DECODED;
    out->step_iterations = opts ? opts->step_iterations : 0;
    out->tail_iterations = opts ? opts->tail_iterations : 0;
    out->tail_step_iterations = opts ? opts->tail_step_iterations : 0;
    out->step_decay = opts ? opts->step_decay : 0.0f;
    if (!(out->step_decay >= 0.0f && out->step_decay <= 1.0f))
        return fail(ART_ERR_INVALID_ARGUMENT, "step_decay must lie in [0, 1]");
    if (out->mode != ART_INIT_DECODED && out->mode != ART_INIT_SCALAR_COMPAT && out->mode != ART_INIT_LEARNED)
        return fail(ART_ERR_INVALID_ARGUMENT, "unknown init mode");
    if (out->mode == ART_INIT_LEARNED && !ctx->net && !ctx->net_joint)
        return fail(ART_ERR_INVALID_ARGUMENT, "learned start: no network attached (art_context_set_warm_start)");
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
    ART_CUDA(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
    ART_CUDA(cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming));
    ART_CUDA(cudaEventCreateWithFlags(&ctx->join, cudaEventDisableTiming));
    *out = ctx.release();
    return ART_OK;
}

void art_context_destroy(ArtContext *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->exec) cudaGraphExecDestroy(ctx->exec);
    if (ctx->init_exec) cudaGraphExecDestroy(ctx->init_exec);
    for (auto e : ctx->events) cudaEventDestroy(e);
    ctx->xbuf.release();
    ctx->pbuf.release();
    ctx->work.release();
    ctx->tasks.release();
    ctx->coefimg.release();
    ctx->stage.release();
    ctx->misc.release();
    ctx->desc.release();
    ctx->compat.release();
    ctx->sepplanes.release();
    ctx->rgb.release();
    ctx->pred.release();
    ctx->evalbuf.release();
    ctx->hstage.release();
    ctx->hrgb.release();
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    if (ctx->join) cudaEventDestroy(ctx->join);
    if (ctx->side) cudaStreamDestroy(ctx->side);
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
    InitSpec ini;
    if ((rc = init_spec(ctx, opts, &ini))) return rc;
    ART_CUDA(cudaSetDevice(ctx->device));
    ctx->net_used = false;
    // `stream` NULL is the legacy default stream, as everywhere in CUDA.
    cudaStream_t user = static_cast<cudaStream_t>(stream);
    cudaEvent_t join = nullptr;
    if (user != ctx->stream) {
        // Order the context's stream after the caller's work.
        ART_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
        ART_CUDA(cudaEventRecord(join, user));
        ART_CUDA(cudaStreamWaitEvent(ctx->stream, join, 0));
    }
    ImageSpec sp{nchannel, coefs, {nullptr, nullptr, nullptr}, weight, {pweight[0], pweight[1], pweight[2]}, max_w,
                 max_h};
    for (uint32_t c = 0; c < nchannel; c++) sp.src[c] = coefs[c].dct_coefs;
    rc = prepare_batch(ctx, {sp}, iterations, ini.mode, ini.step_iterations);
    if (!rc) rc = run_iterations(ctx, iterations, ini.tail_iterations, ini.tail_stepmul(iterations), ini.step_decay);
    if (!rc) {
        const float *fb;
        int fp;
        long long fcs;
        result_planes(ctx, 0, &fb, &fp, &fcs);
        for (uint32_t c = 0; c < nchannel; c++) {
            cudaError_t e = cudaMemcpy2DAsync(out_planes_device[c], (size_t)out_pitch * sizeof(float), fb + c * fcs,
                                              (size_t)fp * sizeof(float), (size_t)max_w * sizeof(float), max_h,
                                              cudaMemcpyDeviceToDevice, ctx->stream);
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

int32_t art_context_evaluate(ArtContext *ctx, uint32_t image, double out[5])
{
    if (!ctx || !out) return fail(ART_ERR_INVALID_ARGUMENT, "null argument");
    if (image >= ctx->h_desc.size()) return fail(ART_ERR_INVALID_ARGUMENT, "no such image in the last solve");
    ART_CUDA(cudaSetDevice(ctx->device));
    static std::once_flag once;
    static double mat[64];
    std::call_once(once, [] {
        const double pi = 3.14159265358979323846;
        for (int u = 0; u < 8; u++)
            for (int y = 0; y < 8; y++)
                mat[u * 8 + y] = (u == 0 ? std::sqrt(1.0 / 8.0) : std::sqrt(2.0 / 8.0)) * std::cos((2 * y + 1) * u * pi / 16.0);
    });
    ART_CUDA(cudaMemcpyToSymbolAsync(c_dct_matrix, mat, sizeof(mat), 0, cudaMemcpyHostToDevice, ctx->stream));
    const ImgDev &d = ctx->h_desc[image];
    const int nparts = 2 * EVAL_BLOCKS * (1 + d.nch);
    int rc;
    if ((rc = ctx->evalbuf.ensure(nparts * sizeof(double)))) return rc;
    double *part = static_cast<double *>(ctx->evalbuf.p);
    const ImgDev *ddesc = static_cast<const ImgDev *>(ctx->desc.p);
    k_eval_pixels<<<EVAL_BLOCKS, EVAL_THREADS, 0, ctx->stream>>>(ddesc, (int)image, part);
    for (int c = 0; c < d.nch; c++)
        k_eval_blocks<<<EVAL_BLOCKS, EVAL_THREADS, 0, ctx->stream>>>(ddesc, (int)image, c,
                                                                      part + 2 * EVAL_BLOCKS * (1 + c));
    ART_CUDA(cudaGetLastError());
    std::vector<double> h(nparts);
    ART_CUDA(cudaMemcpyAsync(h.data(), part, nparts * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    ART_CUDA(cudaStreamSynchronize(ctx->stream));
    const std::array<float, 4> &wt = ctx->h_weights[image];
    const double nch = (double)d.nch;
    double s1 = 0, s2 = 0;
    for (int b = 0; b < EVAL_BLOCKS; b++) {
        s1 += h[2 * b];
        s2 += h[2 * b + 1];
    }
    const double tv = s1 / std::sqrt(nch), tgv = s2 * (((double)wt[0] / std::sqrt(2.0)) / std::sqrt(nch));
    double prob = 0, worst = 0;
    for (int c = 0; c < d.nch; c++) {
        double acc = 0;
        for (int b = 0; b < EVAL_BLOCKS; b++) {
            acc += h[2 * EVAL_BLOCKS * (1 + c) + 2 * b];
            worst = std::max(worst, h[2 * EVAL_BLOCKS * (1 + c) + 2 * b + 1]);
        }
        if (wt[1 + c] != 0.0f)
            prob += 0.5 * ((double)wt[1 + c] * 2.0 * 255.0 * std::sqrt(2.0) * (double)(d.ch[c].sh * d.ch[c].sv)) * acc;
    }
    out[0] = tv + tgv + prob;
    out[1] = tv;
    out[2] = tgv;
    out[3] = prob;
    out[4] = worst;
    return ART_OK;
}

int32_t art_context_set_warm_start(ArtContext *ctx, ArtNet *net)
{
    if (!ctx) return fail(ART_ERR_INVALID_ARGUMENT, "null context");
    if (net && cnn::net_device(net) != ctx->device)
        return fail(ART_ERR_INVALID_ARGUMENT, "warm-start network lives on another device than the context");
    ctx->net = net;
    ctx->net_used = false;
    return ART_OK;
}

int32_t art_context_set_joint_warm_start(ArtContext *ctx, ArtNet *net)
{
    if (!ctx) return fail(ART_ERR_INVALID_ARGUMENT, "null context");
    if (net && cnn::net_device(net) != ctx->device)
        return fail(ART_ERR_INVALID_ARGUMENT, "warm-start network lives on another device than the context");
    ctx->net_joint = net;
    ctx->net_used = false;
    return ART_OK;
}

int32_t art_context_synchronize(ArtContext *ctx)
{
    if (!ctx) return fail(ART_ERR_INVALID_ARGUMENT, "null context");
    ART_CUDA(cudaSetDevice(ctx->device));
    ART_CUDA(cudaStreamSynchronize(ctx->stream));
    return check_errflag(ctx);
}

static int solve_host(ArtContext *ctx, uint32_t nchannel, const ArtChannel *coefs, float weight,
                      const float pweight[3], uint32_t iterations, uint32_t max_w, uint32_t max_h,
                      const ArtOptions *opts)
{
    int rc = validate(nchannel, coefs, weight, pweight, max_w, max_h);
    if (rc) return rc;
    InitSpec ini;
    if ((rc = init_spec(ctx, opts, &ini))) return rc;
    ctx->net_used = false;
    // Host coefficients go through a device staging buffer.
    size_t off[3], total = 0;
    for (uint32_t c = 0; c < nchannel; c++) {
        off[c] = total;
        const size_t es = coefs[c].coef_type == ART_COEF_I16 ? 2 : 4;
        total += align_up((size_t)coefs[c].block_w * coefs[c].block_h * 64 * es, 256);
    }
    if ((rc = ctx->stage.ensure(total))) return rc;
    ImageSpec sp{nchannel, coefs, {nullptr, nullptr, nullptr}, weight, {pweight[0], pweight[1], pweight[2]}, max_w,
                 max_h};
    for (uint32_t c = 0; c < nchannel; c++) {
        const size_t es = coefs[c].coef_type == ART_COEF_I16 ? 2 : 4;
        char *dst = static_cast<char *>(ctx->stage.p) + off[c];
        ART_CUDA(cudaMemcpyAsync(dst, coefs[c].dct_coefs, (size_t)coefs[c].block_w * coefs[c].block_h * 64 * es,
                                 cudaMemcpyHostToDevice, ctx->stream));
        sp.src[c] = dst;
    }
    rc = prepare_batch(ctx, {sp}, iterations, ini.mode, ini.step_iterations);
    if (!rc) rc = run_iterations(ctx, iterations, ini.tail_iterations, ini.tail_stepmul(iterations), ini.step_decay);
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
    int rc = solve_host(ctx, nchannel, coefs, weight, pweight, iterations, max_w, max_h, opts);
    if (rc) {
        cudaStreamSynchronize(ctx->stream);
        return rc;
    }
    const float *fb;
    int fp;
    long long fcs;
    result_planes(ctx, 0, &fb, &fp, &fcs);
    for (uint32_t c = 0; c < nchannel; c++)
        ART_CUDA(cudaMemcpy2DAsync(out_planes[c], (size_t)max_w * sizeof(float), fb + c * fcs,
                                   (size_t)fp * sizeof(float), (size_t)max_w * sizeof(float), max_h,
                                   cudaMemcpyDeviceToHost, ctx->stream));
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
        rc = solve_host(ctx, 3, coefs, weight[0], pweight, iterations[0], W, H, opts);
        if (rc) {
            cudaStreamSynchronize(ctx->stream);
            return rc;
        }
        const float *fb;
        int fp;
        long long fcs;
        result_planes(ctx, 0, &fb, &fp, &fcs);
        for (int c = 0; c < 3; c++) planes[c] = fb + c * fcs;
        pitch = fp;
    } else {
        // lib.rs:133-153: each component alone, compute(1, [coef], weight[c], pweight, iterations[c]),
        // so every component uses pweight[0].
        const size_t plane = (size_t)W * H;
        if ((rc = ctx->sepplanes.ensure(nout * plane * sizeof(float)))) return rc;
        for (uint32_t c = 0; c < nchannel; c++) {
            const float w = weight[c < 3 ? c : 2];
            const uint32_t its = iterations[c < 3 ? c : 2];
            rc = solve_host(ctx, 1, &coefs[c], w, pweight, its, W, H, opts);
            if (rc) {
                cudaStreamSynchronize(ctx->stream);
                return rc;
            }
            if (c < nout) {
                float *dst = static_cast<float *>(ctx->sepplanes.p) + c * plane;
                const float *fb;
                int fp;
                long long fcs;
                result_planes(ctx, 0, &fb, &fp, &fcs);
                ART_CUDA(cudaMemcpy2DAsync(dst, (size_t)W * sizeof(float), fb, (size_t)fp * sizeof(float),
                                           (size_t)W * sizeof(float), H, cudaMemcpyDeviceToDevice, ctx->stream));
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


// ---------------------------------------------------------------- batches --

static int batch_specs(const ArtImage *images, uint32_t nimages, std::vector<ImageSpec> &specs)
{
    specs.clear();
    for (uint32_t i = 0; i < nimages; i++) {
        const ArtImage &im = images[i];
        int rc = validate(im.nchannel, im.channels, im.weight, im.pweight, im.max_rounded_px_w, im.max_rounded_px_h);
        if (rc) return fail(rc, "image " + std::to_string(i) + ": " + g_err);
        if (!im.out_planes) return fail(ART_ERR_INVALID_ARGUMENT, "image " + std::to_string(i) + ": null output planes");
        for (uint32_t c = 0; c < im.nchannel; c++)
            if (!im.out_planes[c]) return fail(ART_ERR_INVALID_ARGUMENT, "image " + std::to_string(i) + ": null plane");
        ImageSpec sp{im.nchannel, im.channels, {nullptr, nullptr, nullptr}, im.weight,
                     {im.pweight[0], im.pweight[1], im.pweight[2]}, im.max_rounded_px_w, im.max_rounded_px_h};
        for (uint32_t c = 0; c < im.nchannel; c++) sp.src[c] = im.channels[c].dct_coefs;
        specs.push_back(sp);
    }
    return ART_OK;
}

int32_t art_context_compute_batch(ArtContext *ctx, uint32_t nimages, const ArtImage *images, uint32_t iterations,
                                  const ArtOptions *opts)
{
    if (!ctx || !images || nimages == 0) return fail(ART_ERR_INVALID_ARGUMENT, "null context or empty batch");
    ART_CUDA(cudaSetDevice(ctx->device));
    InitSpec ini;
    int rc = init_spec(ctx, opts, &ini);
    if (rc) return rc;
    ctx->net_used = false;
    std::vector<ImageSpec> specs;
    rc = batch_specs(images, nimages, specs);
    if (rc) return rc;
    // Host coefficients of every image through one device staging buffer.
    size_t total = 0;
    for (auto &sp : specs)
        for (uint32_t c = 0; c < sp.nch; c++)
            total += align_up((size_t)sp.ch[c].block_w * sp.ch[c].block_h * 64 *
                                  (sp.ch[c].coef_type == ART_COEF_I16 ? 2 : 4), 256);
    if ((rc = ctx->stage.ensure(total))) return rc;
    size_t off = 0;
    for (auto &sp : specs)
        for (uint32_t c = 0; c < sp.nch; c++) {
            const size_t n = (size_t)sp.ch[c].block_w * sp.ch[c].block_h * 64 * (sp.ch[c].coef_type == ART_COEF_I16 ? 2 : 4);
            char *dst = static_cast<char *>(ctx->stage.p) + off;
            ART_CUDA(cudaMemcpyAsync(dst, sp.ch[c].dct_coefs, n, cudaMemcpyHostToDevice, ctx->stream));
            sp.src[c] = dst;
            off += align_up(n, 256);
        }
    rc = prepare_batch(ctx, specs, iterations, ini.mode, ini.step_iterations);
    if (!rc) rc = run_iterations(ctx, iterations, ini.tail_iterations, ini.tail_stepmul(iterations), ini.step_decay);
    if (rc) {
        cudaStreamSynchronize(ctx->stream);
        return rc;
    }
    for (uint32_t i = 0; i < nimages; i++) {
        const float *fb;
        int fp;
        long long fcs;
        result_planes(ctx, (int)i, &fb, &fp, &fcs);
        const ArtImage &im = images[i];
        for (uint32_t c = 0; c < im.nchannel; c++)
            ART_CUDA(cudaMemcpy2DAsync(im.out_planes[c], (size_t)im.max_rounded_px_w * sizeof(float), fb + c * fcs,
                                       (size_t)fp * sizeof(float), (size_t)im.max_rounded_px_w * sizeof(float),
                                       im.max_rounded_px_h, cudaMemcpyDeviceToHost, ctx->stream));
    }
    ART_CUDA(cudaStreamSynchronize(ctx->stream));
    return check_errflag(ctx);
}

int32_t art_context_compute_batch_device(ArtContext *ctx, uint32_t nimages, const ArtImage *images,
                                         uint32_t iterations, const ArtOptions *opts, void *stream)
{
    if (!ctx || !images || nimages == 0) return fail(ART_ERR_INVALID_ARGUMENT, "null context or empty batch");
    ART_CUDA(cudaSetDevice(ctx->device));
    InitSpec ini;
    int rc = init_spec(ctx, opts, &ini);
    if (rc) return rc;
    ctx->net_used = false;
    std::vector<ImageSpec> specs;
    rc = batch_specs(images, nimages, specs);
    if (rc) return rc;
    for (uint32_t i = 0; i < nimages; i++)
        if (images[i].out_pitch < images[i].max_rounded_px_w)
            return fail(ART_ERR_INVALID_ARGUMENT, "image " + std::to_string(i) + ": out_pitch below width");
    cudaStream_t user = static_cast<cudaStream_t>(stream);
    cudaEvent_t join = nullptr;
    if (user != ctx->stream) {
        ART_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
        ART_CUDA(cudaEventRecord(join, user));
        ART_CUDA(cudaStreamWaitEvent(ctx->stream, join, 0));
    }
    rc = prepare_batch(ctx, specs, iterations, ini.mode, ini.step_iterations);
    if (!rc) rc = run_iterations(ctx, iterations, ini.tail_iterations, ini.tail_stepmul(iterations), ini.step_decay);
    for (uint32_t i = 0; !rc && i < nimages; i++) {
        const float *fb;
        int fp;
        long long fcs;
        result_planes(ctx, (int)i, &fb, &fp, &fcs);
        const ArtImage &im = images[i];
        for (uint32_t c = 0; c < im.nchannel && !rc; c++) {
            cudaError_t e = cudaMemcpy2DAsync(im.out_planes[c], (size_t)im.out_pitch * sizeof(float), fb + c * fcs,
                                              (size_t)fp * sizeof(float), (size_t)im.max_rounded_px_w * sizeof(float),
                                              im.max_rounded_px_h, cudaMemcpyDeviceToDevice, ctx->stream);
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

int32_t art_context_process_batch(ArtContext *ctx, uint32_t nimages, const ArtProcessImage *images,
                                  uint32_t iterations, int32_t separate, const ArtOptions *opts)
{
    if (!ctx || !images || nimages == 0) return fail(ART_ERR_INVALID_ARGUMENT, "null context or empty batch");
    ART_CUDA(cudaSetDevice(ctx->device));
    InitSpec ini;
    int rc = init_spec(ctx, opts, &ini);
    if (rc) return rc;
    ctx->net_used = false;
    // lib.rs:122-153 per image: a joint solve of a 3-component image, else one
    // solve per component (each reads pweight[0], as compute(1, ...) does).
    // Every solve becomes one image of the batch.
    struct Out {
        uint32_t first, nout;  // first batch image of this input, planes to convert
        bool joint;
    };
    std::vector<ImageSpec> specs;
    std::vector<Out> outs(nimages);
    for (uint32_t i = 0; i < nimages; i++) {
        const ArtProcessImage &im = images[i];
        const std::string at = "image " + std::to_string(i) + ": ";
        if (im.nchannel < 1 || im.nchannel > 4 || !im.channels)
            return fail(ART_ERR_INVALID_ARGUMENT, at + "nchannel must be 1 to 4 with channels given");
        uint32_t W = 0, H = 0;
        for (uint32_t c = 0; c < im.nchannel; c++) {
            W = std::max(W, im.channels[c].rounded_px_w);
            H = std::max(H, im.channels[c].rounded_px_h);
        }
        if (im.real_w == 0 || im.real_h == 0 || im.real_w > W || im.real_h > H)
            return fail(ART_ERR_INVALID_ARGUMENT, at + "real size must be positive and within the rounded size");
        const bool joint = im.nchannel == 3 && !separate;
        outs[i] = {(uint32_t)specs.size(), im.nchannel == 3 ? 3u : 1u, joint};
        const uint32_t njobs = joint ? 1 : im.nchannel;
        for (uint32_t k = 0; k < njobs; k++) {
            const uint32_t nch = joint ? 3 : 1;
            const ArtChannel *ch = joint ? im.channels : &im.channels[k];
            const float w = joint ? im.weight[0] : im.weight[std::min(k, 2u)];
            if ((rc = validate(nch, ch, w, im.pweight, W, H))) return fail(rc, at + g_err);
            ImageSpec sp{nch, ch, {nullptr, nullptr, nullptr}, w, {im.pweight[0], im.pweight[1], im.pweight[2]},
                         W, H};
            for (uint32_t c = 0; c < nch; c++) sp.src[c] = ch[c].dct_coefs;
            specs.push_back(sp);
        }
    }
    // Host coefficients through one device staging buffer.
    size_t total = 0;
    for (auto &sp : specs)
        for (uint32_t c = 0; c < sp.nch; c++)
            total += align_up((size_t)sp.ch[c].block_w * sp.ch[c].block_h * 64 *
                                  (sp.ch[c].coef_type == ART_COEF_I16 ? 2 : 4), 256);
    if ((rc = ctx->stage.ensure(total)) || (rc = ctx->hstage.ensure(total))) return rc;
    // Gathered into pinned memory by host threads, then one asynchronous copy.
    // The previous call on this context returned only after its copies ended,
    // so the pinned buffer is free.
    std::vector<CopyJob> up;
    size_t off = 0;
    for (auto &sp : specs)
        for (uint32_t c = 0; c < sp.nch; c++) {
            const size_t n = (size_t)sp.ch[c].block_w * sp.ch[c].block_h * 64 * (sp.ch[c].coef_type == ART_COEF_I16 ? 2 : 4);
            up.push_back({static_cast<char *>(ctx->hstage.p) + off, sp.ch[c].dct_coefs, n});
            sp.src[c] = static_cast<char *>(ctx->stage.p) + off;
            off += align_up(n, 256);
        }
    parallel_copy(up);
    ART_CUDA(cudaMemcpyAsync(ctx->stage.p, ctx->hstage.p, off, cudaMemcpyHostToDevice, ctx->stream));
    rc = prepare_batch(ctx, specs, iterations, ini.mode, ini.step_iterations);
    if (!rc) rc = run_iterations(ctx, iterations, ini.tail_iterations, ini.tail_stepmul(iterations), ini.step_decay);
    if (rc) {
        cudaStreamSynchronize(ctx->stream);
        return rc;
    }
    // Output stage per image (lib.rs:159-211) into one device buffer, one
    // copy of it to pinned memory, then host threads copy each image out.
    size_t rgb_total = 0;
    for (uint32_t i = 0; i < nimages; i++)
        if (images[i].rgb_out) rgb_total += align_up((size_t)images[i].real_w * images[i].real_h * 3, 256);
    std::vector<CopyJob> down;
    if (rgb_total) {
        if ((rc = ctx->rgb.ensure(rgb_total)) || (rc = ctx->hrgb.ensure(rgb_total))) {
            cudaStreamSynchronize(ctx->stream);
            return rc;
        }
        size_t ro = 0;
        for (uint32_t i = 0; i < nimages; i++) {
            const ArtProcessImage &im = images[i];
            if (!im.rgb_out) continue;
            const float *pl[3] = {nullptr, nullptr, nullptr};
            long long pitch = 0;
            for (uint32_t c = 0; c < outs[i].nout; c++) {
                const float *fb;
                int fp;
                long long fcs;
                result_planes(ctx, (int)(outs[i].first + (outs[i].joint ? 0 : c)), &fb, &fp, &fcs);
                pl[c] = outs[i].joint ? fb + c * fcs : fb;
                pitch = fp;
            }
            const long long n = (long long)im.real_w * im.real_h;
            uint8_t *dst = static_cast<uint8_t *>(ctx->rgb.p) + ro;
            k_rgb<<<(int)((n + 255) / 256), 256, 0, ctx->stream>>>(pl[0], pl[1], pl[2], pitch, (int)outs[i].nout,
                                                                   (int)im.real_w, (int)im.real_h, dst);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) {
                cudaStreamSynchronize(ctx->stream);
                return fail(ART_ERR_CUDA, std::string("output stage: ") + cudaGetErrorString(e));
            }
            down.push_back({im.rgb_out, static_cast<char *>(ctx->hrgb.p) + ro, (size_t)n * 3});
            ro += align_up((size_t)n * 3, 256);
        }
        const cudaError_t e = cudaMemcpyAsync(ctx->hrgb.p, ctx->rgb.p, ro, cudaMemcpyDeviceToHost, ctx->stream);
        if (e != cudaSuccess) {
            cudaStreamSynchronize(ctx->stream);
            return fail(ART_ERR_CUDA, std::string("output copy: ") + cudaGetErrorString(e));
        }
    }
    ART_CUDA(cudaStreamSynchronize(ctx->stream));
    if ((rc = check_errflag(ctx))) return rc;
    parallel_copy(down);
    return ART_OK;
}

// -------------------------------------------------------------- autotuner --

}  // extern "C"

namespace art {
namespace {

constexpr int TUNE_REPS = 5;          // timed repetitions per candidate (median)
constexpr float TUNE_TIE = 0.02f;     // candidates within 2 % of the fastest count as ties

// Times the launch-shape candidates on prepared specs (coefficients already on
// the device): first the gradient sweep (variant x strip rows, projection at 4
// warps), then the projection's warps per block with the chosen sweep. Each
// candidate is captured and warmed once, then timed TUNE_REPS times; its time
// is the median. Candidates are tried in a fixed order that starts with the
// size heuristic's choice, and the first one within TUNE_TIE of the fastest
// wins, so a choice changes only for a clear gain.
int tune_specs(ArtContext *ctx, const std::vector<ImageSpec> &specs, uint32_t iterations, bool skip_tall,
               TuneChoice *best, ArtTuneResult *res)
{
    long long batch_px = 0;
    uint32_t max_h = 0;
    for (const auto &sp : specs) {
        batch_px += (long long)sp.W * sp.H;
        max_h = std::max(max_h, sp.H);
    }
    const TuneChoice heur = pick_shape(ctx, specs[0], batch_px, (int)specs.size());
    ctx->tune_log.clear();
    cudaEvent_t e0, e1;
    ART_CUDA(cudaEventCreate(&e0));
    ART_CUDA(cudaEventCreate(&e1));
    const bool timing = ctx->timing;
    ctx->timing = false;
    int rc = ART_OK;
    auto time_one = [&](const TuneChoice &t, float *ms) -> int {
        ctx->sweep_kind_override = t.kind;
        ctx->strip_rows_override = t.rows;
        ctx->proj_warps_override = t.proj_warps;
        int r = prepare_batch(ctx, specs, iterations, ART_INIT_DECODED, 0);
        if (!r) r = run_iterations(ctx, iterations);  // captures and warms up
        std::vector<float> v;
        for (int rep = 0; rep < TUNE_REPS && !r; rep++) {
            cudaEventRecord(e0, ctx->stream);
            r = run_iterations(ctx, iterations);
            cudaEventRecord(e1, ctx->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) r = fail(ART_ERR_CUDA, "autotune: timing failed");
            float t_ms = 0.f;
            cudaEventElapsedTime(&t_ms, e0, e1);
            v.push_back(t_ms);
        }
        if (!r) {
            std::sort(v.begin(), v.end());
            *ms = v[v.size() / 2];
        }
        return r;
    };
    auto pick = [](const std::vector<std::pair<TuneChoice, float>> &c) {
        float lo = c[0].second;
        for (const auto &x : c) lo = std::min(lo, x.second);
        for (const auto &x : c)
            if (x.second <= lo * (1.0f + TUNE_TIE)) return x;
        return c[0];
    };
    // Phase 1: the sweep, heuristic first.
    std::vector<TuneChoice> cands = {TuneChoice{heur.kind, heur.rows, PROJ_WARPS}};
    for (int kind = 0; kind < 3; kind++)
        for (int R : {16, 32, 64, 128}) {
            if (skip_tall && (int)max_h < R && R > 16) continue;
            if (kind == heur.kind && R == heur.rows) continue;
            cands.push_back(TuneChoice{kind, R, PROJ_WARPS});
        }
    std::vector<std::pair<TuneChoice, float>> timed1, timed2;
    for (const auto &t : cands) {
        float ms = 0.f;
        if ((rc = time_one(t, &ms))) break;
        timed1.push_back({t, ms});
        ctx->tune_log.push_back(ArtTuneCandidate{(uint32_t)t.kind, (uint32_t)t.rows, (uint32_t)t.proj_warps, ms});
    }
    TuneChoice chosen;
    float chosen_ms = 0.f, default_ms = 0.f;
    if (!rc) {
        const auto p1 = pick(timed1);
        // Phase 2: projection warps per block, 4 (already timed) first.
        timed2.push_back(p1);
        for (int pw : PROJ_WARP_CHOICES) {
            if (pw == PROJ_WARPS) continue;
            TuneChoice t = p1.first;
            t.proj_warps = pw;
            float ms = 0.f;
            if ((rc = time_one(t, &ms))) break;
            timed2.push_back({t, ms});
            ctx->tune_log.push_back(ArtTuneCandidate{(uint32_t)t.kind, (uint32_t)t.rows, (uint32_t)t.proj_warps, ms});
        }
        if (!rc) {
            const auto p2 = pick(timed2);
            chosen = p2.first;
            chosen_ms = p2.second;
            default_ms = timed1[0].second;
        }
    }
    ctx->strip_rows_override = 0;
    ctx->sweep_kind_override = 0;
    ctx->proj_warps_override = 0;
    ctx->timing = timing;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    ART_CUDA(cudaStreamSynchronize(ctx->stream));
    *best = chosen;
    if (res) {
        memset(res, 0, sizeof(*res));
        res->variant = (uint32_t)chosen.kind;
        res->strip_rows = (uint32_t)chosen.rows;
        res->proj_warps = (uint32_t)chosen.proj_warps;
        res->candidates = (uint32_t)(timed1.size() + timed2.size() - 1);
        res->best_ms = chosen_ms;
        res->heuristic_ms = default_ms;
        res->heuristic_variant = (uint32_t)heur.kind;
        res->heuristic_strip_rows = (uint32_t)heur.rows;
    }
    return ART_OK;
}

}  // namespace
}  // namespace art

extern "C" {

int32_t art_context_autotune(ArtContext *ctx, uint32_t nchannel, const uint32_t *samp_h, const uint32_t *samp_v,
                             uint32_t max_w, uint32_t max_h, uint32_t iterations, uint32_t *variant_out,
                             uint32_t *strip_rows_out)
{
    if (!ctx || !samp_h || !samp_v || nchannel < 1 || nchannel > 3)
        return fail(ART_ERR_INVALID_ARGUMENT, "bad autotune arguments");
    ART_CUDA(cudaSetDevice(ctx->device));
    if (iterations == 0) iterations = 10;
    // A deterministic synthetic image of this geometry: sparse small
    // coefficients, quantisation steps of 8.
    ArtChannel ch[3];
    std::vector<int16_t> host[3];
    float q[64];
    for (int j = 0; j < 64; j++) q[j] = 8.0f;
    uint32_t lcg = 12345u;
    size_t total = 0;
    for (uint32_t c = 0; c < nchannel; c++) {
        if ((samp_h[c] != 1 && samp_h[c] != 2) || (samp_v[c] != 1 && samp_v[c] != 2) || max_w % (8 * samp_h[c]) ||
            max_h % (8 * samp_v[c]))
            return fail(ART_ERR_INVALID_ARGUMENT, "autotune geometry does not fit the sampling factors");
        memset(&ch[c], 0, sizeof(ArtChannel));
        ch[c].rounded_px_w = max_w / samp_h[c];
        ch[c].rounded_px_h = max_h / samp_v[c];
        ch[c].block_w = ch[c].rounded_px_w / 8;
        ch[c].block_h = ch[c].rounded_px_h / 8;
        ch[c].samp_h = samp_h[c];
        ch[c].samp_v = samp_v[c];
        ch[c].coef_type = ART_COEF_I16;
        ch[c].quant_table = q;
        host[c].assign((size_t)ch[c].block_w * ch[c].block_h * 64, 0);
        ch[c].dct_coefs = host[c].data();  // host values; staged to the device below
        for (size_t i = 0; i < host[c].size(); i++) {
            lcg = lcg * 1664525u + 1013904223u;
            if ((i & 63) == 0 || (lcg >> 28) == 0) host[c][i] = (int16_t)((int)((lcg >> 16) & 255) - 128);
        }
        total += align_up(host[c].size() * 2, 256);
    }
    const float pw3[3] = {0.001f, 0.001f, 0.001f};
    int rc = validate(nchannel, ch, 0.3f, pw3, max_w, max_h);
    if (rc) return rc;
    if ((rc = ctx->stage.ensure(total))) return rc;
    ImageSpec sp{nchannel, ch, {nullptr, nullptr, nullptr}, 0.3f, {0.001f, 0.001f, 0.001f}, max_w, max_h};
    size_t off = 0;
    for (uint32_t c = 0; c < nchannel; c++) {
        char *dst = static_cast<char *>(ctx->stage.p) + off;
        ART_CUDA(cudaMemcpyAsync(dst, host[c].data(), host[c].size() * 2, cudaMemcpyHostToDevice, ctx->stream));
        sp.src[c] = dst;
        off += align_up(host[c].size() * 2, 256);
    }
    TuneChoice best;
    if ((rc = tune_specs(ctx, {sp}, iterations, true, &best, &ctx->last_tune))) return rc;
    ctx->tune[tune_key(nchannel, samp_h, samp_v, max_w, max_h)] = best;
    if (variant_out) *variant_out = (uint32_t)best.kind;
    if (strip_rows_out) *strip_rows_out = (uint32_t)best.rows;
    return ART_OK;
}

int32_t art_context_autotune_batch(ArtContext *ctx, uint32_t nimages, const ArtImage *images, uint32_t iterations,
                                   ArtTuneResult *out)
{
    if (!ctx || !images || nimages == 0) return fail(ART_ERR_INVALID_ARGUMENT, "null context or empty batch");
    ART_CUDA(cudaSetDevice(ctx->device));
    if (iterations == 0) iterations = 10;
    std::vector<ImageSpec> specs;
    int rc = batch_specs(images, nimages, specs);
    if (rc) return rc;
    size_t total = 0;
    for (auto &sp : specs)
        for (uint32_t c = 0; c < sp.nch; c++)
            total += align_up((size_t)sp.ch[c].block_w * sp.ch[c].block_h * 64 *
                                  (sp.ch[c].coef_type == ART_COEF_I16 ? 2 : 4), 256);
    if ((rc = ctx->stage.ensure(total))) return rc;
    size_t off = 0;
    for (auto &sp : specs)
        for (uint32_t c = 0; c < sp.nch; c++) {
            const size_t n = (size_t)sp.ch[c].block_w * sp.ch[c].block_h * 64 * (sp.ch[c].coef_type == ART_COEF_I16 ? 2 : 4);
            char *dst = static_cast<char *>(ctx->stage.p) + off;
            ART_CUDA(cudaMemcpyAsync(dst, sp.ch[c].dct_coefs, n, cudaMemcpyHostToDevice, ctx->stream));
            sp.src[c] = dst;
            off += align_up(n, 256);
        }
    TuneChoice best;
    if ((rc = tune_specs(ctx, specs, iterations, false, &best, &ctx->last_tune))) return rc;
    long long batch_px = 0;
    for (const auto &sp : specs) batch_px += (long long)sp.W * sp.H;
    if (nimages > 1) {
        ctx->tune[batch_tune_key((int)nimages, batch_px)] = best;
    } else {
        uint32_t sh[3], sv[3];
        for (uint32_t c = 0; c < specs[0].nch; c++) {
            sh[c] = specs[0].ch[c].samp_h;
            sv[c] = specs[0].ch[c].samp_v;
        }
        ctx->tune[tune_key(specs[0].nch, sh, sv, specs[0].W, specs[0].H)] = best;
    }
    if (out) *out = ctx->last_tune;
    return ART_OK;
}

int32_t art_context_tune_candidates(ArtContext *ctx, ArtTuneCandidate *out, uint32_t capacity, uint32_t *count)
{
    if (!ctx || !count || (capacity && !out)) return fail(ART_ERR_INVALID_ARGUMENT, "null argument");
    *count = (uint32_t)ctx->tune_log.size();
    for (uint32_t i = 0; i < capacity && i < *count; i++) out[i] = ctx->tune_log[i];
    return ART_OK;
}

int32_t art_context_last_tune(ArtContext *ctx, ArtTuneResult *out)
{
    if (!ctx || !out) return fail(ART_ERR_INVALID_ARGUMENT, "null argument");
    if (!ctx->last_tune.candidates) return fail(ART_ERR_INVALID_ARGUMENT, "no autotune run on this context");
    *out = ctx->last_tune;
    return ART_OK;
}

int32_t art_context_tune_cache(ArtContext *ctx, const char *path, int32_t save)
{
    if (!ctx || !path) return fail(ART_ERR_INVALID_ARGUMENT, "null context or path");
    if (save) {
        std::ofstream f(path);
        if (!f) return fail(ART_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
        f << "# artefact_b200 autotune cache: <geometry bucket> <sweep variant 0|1|2> <strip rows> <projection warps>\n";
        for (const auto &kv : ctx->tune)
            f << kv.first << " " << kv.second.kind << " " << kv.second.rows << " " << kv.second.proj_warps << "\n";
        return f.good() ? ART_OK : fail(ART_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
    }
    std::ifstream f(path);
    if (!f) return fail(ART_ERR_INVALID_ARGUMENT, std::string("cannot read ") + path);
    std::string line;
    while (std::getline(f, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream ls(line);
        std::string key;
        int kind = -1, rows = 0, pw = PROJ_WARPS;
        if (!(ls >> key >> kind >> rows) || kind < 0 || kind > 2 ||
            (rows != 16 && rows != 32 && rows != 64 && rows != 128))
            return fail(ART_ERR_INVALID_ARGUMENT, "malformed tune cache line: " + line);
        if (!(ls >> pw)) pw = PROJ_WARPS;  // three-field lines: the default projection shape
        if (pw != 2 && pw != 4 && pw != 8) return fail(ART_ERR_INVALID_ARGUMENT, "malformed tune cache line: " + line);
        ctx->tune[key] = TuneChoice{kind, rows, pw};
    }
    return ART_OK;
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

// ============================================ allocation-free entry point ====
//
// art_solve_noalloc runs the iteration of a default-options
// art_context_compute_device solve (decoded start, one FISTA phase) with the
// narrow gradient sweep and 32-row strips at every size -- equal to it within
// the parity tolerance, not bit for bit, since the sweep variant and strip
// height set the summation order -- and takes every scratch buffer (iterate,
// FISTA point, gradient, DCT-distance and
// coefficient planes, norm partials, descriptor, work lists) from one
// file-scope device array of ART_NOALLOC_SCRATCH_BYTES instead of cudaMalloc.
// It is for callers that must not allocate device memory themselves: callers
// whose device memory is owned by another allocator (a framework's caching
// allocator, a server that partitions each GPU up front) and callers that
// cannot afford the device-wide synchronisation cudaMalloc and cudaFree may
// imply. Every GPU that loads this library holds the array until the process
// exits. All calls share it and it keeps the last call's contents, so each call
// clears what must start at zero; calls whose GPU work overlaps (from two host
// threads, or on two streams) race on it.

#define ART_NOALLOC_SCRATCH_BYTES (64ull << 20)

static __device__ __align__(256) unsigned char g_noalloc_scratch[ART_NOALLOC_SCRATCH_BYTES];

namespace art {
namespace {

struct NoallocSeg {
    int c, base, bw4, bh;  // channel, first task, tasks per block row, block rows
};

struct NoallocPlan {
    NoallocSeg seg[3];
    int nseg;
};

// Writes the descriptor and the two work lists into the scratch array (the
// descriptor arrives by value as a kernel parameter, so no host buffer is copied).
__global__ void k_noalloc_setup(ImgDev d, ImgDev *dst, int2 *work, int ncta, int4 *tasks, int ntasks,
                                NoallocPlan plan)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *dst = d;
    if (i < ncta) work[i] = make_int2(0, i);
    if (i < ntasks) {
        int s = 0;
        while (s + 1 < plan.nseg && i >= plan.seg[s + 1].base) s++;
        const NoallocSeg &g = plan.seg[s];
        const int k = i - g.base, by = k / g.bw4, bx0 = (k % g.bw4) * 4;
        tasks[i] = make_int4(0, g.c, by, bx0);
    }
}

std::mutex g_noalloc_mu;
std::vector<void *> g_noalloc_base;  // per device, resolved once

// Device address of the scratch array on the current device, resolved once
// per device with that device current.
int noalloc_scratch(int device, unsigned char **out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if ((int)g_noalloc_base.size() <= device) g_noalloc_base.resize(device + 1, nullptr);
    if (!g_noalloc_base[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(ART_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_noalloc_base[device] = p;
    }
    *out = static_cast<unsigned char *>(g_noalloc_base[device]);
    return ART_OK;
}

}  // namespace
}  // namespace art

// Once work is queued on the caller's stream, an error return first waits for
// that work (ignoring its status), so a later call cannot overlap it on the
// shared scratch array.
#define NOALLOC_CUDA(call)                                                                   \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            cudaStreamSynchronize(s);                                                        \
            return fail(ART_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
        }                                                                                    \
    } while (0)

extern "C" int32_t art_solve_noalloc(uint32_t nchannel, const ArtChannel *coefs, float weight,
                                     const float pweight[3], uint32_t iterations, uint32_t max_w, uint32_t max_h,
                                     float *const *out_planes_device, uint32_t out_pitch, void *stream)
{
    using namespace art;
    int rc = validate(nchannel, coefs, weight, pweight, max_w, max_h);
    if (rc) return rc;
    if (!out_planes_device || out_pitch < max_w) return fail(ART_ERR_INVALID_ARGUMENT, "bad output planes");
    for (uint32_t c = 0; c < nchannel; c++)
        if (!out_planes_device[c]) return fail(ART_ERR_INVALID_ARGUMENT, "null output plane");
    int device = 0;
    ART_CUDA(cudaGetDevice(&device));
    unsigned char *base = nullptr;
    if ((rc = noalloc_scratch(device, &base))) return rc;
    if ((rc = configure_kernels(device))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // Layout inside the scratch array (the same geometry prepare() uses).
    const uint32_t W = max_w, H = max_h, nch = nchannel;
    const int pitch = (int)align_up(W, 32);
    const long long cstride = (long long)pitch * (long long)align_up(H, 32);
    if (3 * cstride >= (1LL << 31))
        return fail(ART_ERR_INVALID_ARGUMENT, "image too large: three padded planes must stay below 2^31 floats");
    const int R = 32;
    const int strips_x = (int)((W + SWEEP_OUT_N - 1) / SWEEP_OUT_N), strips_y = (int)((H + R - 1) / R);
    const int nstrips = strips_x * strips_y, ncta = (nstrips + SWEEP_WARPS_N - 1) / SWEEP_WARPS_N;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    const size_t o_x = take(3 * nch * cstride * sizeof(float));
    size_t o_coef[3], o_p[3];
    int cpitch[3], ppitch[3];
    for (uint32_t c = 0; c < nch; c++) {
        cpitch[c] = (int)align_up(coefs[c].rounded_px_w, 64);
        ppitch[c] = (int)align_up(coefs[c].rounded_px_w, 32);
        o_coef[c] = take((size_t)cpitch[c] * coefs[c].rounded_px_h * sizeof(int16_t));
        o_p[c] = take((size_t)ppitch[c] * coefs[c].rounded_px_h * sizeof(float));
    }
    const size_t o_misc = take(align_up((size_t)ncta * 4 * sizeof(float), 256) + 256);
    const size_t o_desc = take(sizeof(ImgDev));
    const size_t o_work = take((size_t)ncta * sizeof(int2));
    // Tasks grouped by sampling mode (channels of one mode in channel order).
    NoallocPlan plan{};
    int mode_off[5] = {0, 0, 0, 0, 0};
    int ntasks = 0;
    for (int m = 0; m < 4; m++) {
        mode_off[m] = ntasks;
        for (uint32_t c = 0; c < nch; c++) {
            if (samp_mode((int)coefs[c].samp_h, (int)coefs[c].samp_v) != m) continue;
            const int bw4 = (int)((coefs[c].block_w + 3) / 4);
            plan.seg[plan.nseg++] = NoallocSeg{(int)c, ntasks, bw4, (int)coefs[c].block_h};
            ntasks += bw4 * (int)coefs[c].block_h;
        }
    }
    mode_off[4] = ntasks;
    const size_t o_tasks = take((size_t)ntasks * sizeof(int4));
    if (off > ART_NOALLOC_SCRATCH_BYTES)
        return fail(ART_ERR_INVALID_ARGUMENT, "image needs " + std::to_string(off >> 20) +
                                                  " MiB of scratch; art_solve_noalloc has " +
                                                  std::to_string(ART_NOALLOC_SCRATCH_BYTES >> 20) + " MiB");

    ImgDev d;
    memset(&d, 0, sizeof(d));
    d.nch = (int)nch;
    d.W = (int)W;
    d.H = (int)H;
    d.pitch = pitch;
    d.strips_x = strips_x;
    d.strips_y = strips_y;
    d.nstrips = nstrips;
    d.strip_rows = R;
    d.ncta = ncta;
    d.cstride = cstride;
    d.x = reinterpret_cast<float *>(base + o_x);
    d.y = d.x + nch * cstride;
    d.g = d.y + nch * cstride;
    d.alpha_tv = 1.0f / sqrtf((float)nch);
    d.alpha_tgv = (weight / sqrtf(2.0f)) / sqrtf((float)nch);
    d.step = (sqrtf((float)((uint64_t)W * H)) / 2.0f) / sqrtf(1.0f + (float)iterations);
    unsigned char *misc = base + o_misc;
    d.partial = reinterpret_cast<float *>(misc);
    d.sigma = reinterpret_cast<float *>(misc + align_up((size_t)ncta * 4 * sizeof(float), 256));
    d.counter = reinterpret_cast<unsigned *>(d.sigma + 4);
    unsigned *errflag = d.counter + 1;
    for (uint32_t c = 0; c < nch; c++) {
        ChanDev &cd = d.ch[c];
        cd.cw = (int)coefs[c].rounded_px_w;
        cd.chh = (int)coefs[c].rounded_px_h;
        cd.sh = (int)coefs[c].samp_h;
        cd.sv = (int)coefs[c].samp_v;
        cd.cpitch = cpitch[c];
        cd.ppitch = ppitch[c];
        cd.coef = reinterpret_cast<const int16_t *>(base + o_coef[c]);
        cd.P = reinterpret_cast<float *>(base + o_p[c]);
        cd.alpha_p = pweight[c] * 2.0f * 255.0f * sqrtf(2.0f);
        for (int j = 0; j < 64; j++) {
            const float q = coefs[c].quant_table[j];
            d.q[c][j] = q;
            d.invq2[c][j] = 1.0f / (q * q);
        }
    }
    ImgDev *ddesc = reinterpret_cast<ImgDev *>(base + o_desc);
    int2 *work = reinterpret_cast<int2 *>(base + o_work);
    int4 *tasks = reinterpret_cast<int4 *>(base + o_tasks);

    // Clear what must start at zero: the norm partials, counter and error flag,
    // and the first DCT-distance gradient planes.
    NOALLOC_CUDA(cudaMemsetAsync(misc, 0, o_desc - o_misc, s));
    for (uint32_t c = 0; c < nch; c++)
        NOALLOC_CUDA(cudaMemsetAsync(d.ch[c].P, 0, (size_t)ppitch[c] * coefs[c].rounded_px_h * sizeof(float), s));
    const int nset = std::max(ncta, ntasks);
    k_noalloc_setup<<<(nset + 255) / 256, 256, 0, s>>>(d, ddesc, work, ncta, tasks, ntasks, plan);
    for (uint32_t c = 0; c < nch; c++) {
        const long long ncoef = (long long)coefs[c].block_w * coefs[c].block_h * 64;
        k_ingest<<<(int)((ncoef + 255) / 256), 256, 0, s>>>(coefs[c].dct_coefs, (int)coefs[c].coef_type,
                                                             (int)coefs[c].block_w, ncoef,
                                                             const_cast<int16_t *>(d.ch[c].coef), cpitch[c], errflag);
    }
    k_init<<<(ntasks + PROJ_WARPS - 1) / PROJ_WARPS, PROJ_WARPS * 32, 0, s>>>(ddesc, tasks, ntasks);
    // FISTA factors as fista_factors() forms them, one step ahead (no host buffer).
    float term = 1.0f;
    auto next_factor = [&term]() {
        volatile float t2 = term * term;
        volatile float inner = 4.0f * t2 + 1.0f;
        const float next = (float)(((double)1.0f + (double)sqrtf(inner)) / 2.0);
        const float f = (term - 1.0f) / next;
        term = next;
        return f;
    };
    next_factor();  // f_0 = 0: y_0 = x_0
    for (uint32_t it = 0; it < iterations; it++) {
        const float fnext = it + 1 < iterations ? next_factor() : 0.0f;
        if (nch == 3)
            k_grad_sweep_n<3><<<ncta, SWEEP_WARPS_N * 32, 0, s>>>(ddesc, work, 1.0f);
        else if (nch == 2)
            k_grad_sweep_n<2><<<ncta, SWEEP_WARPS_N * 32, 0, s>>>(ddesc, work, 1.0f);
        else
            k_grad_sweep_n<1><<<ncta, SWEEP_WARPS_N * 32, 0, s>>>(ddesc, work, 1.0f);
        for (int m = 3; m >= 0; m--) {
            const int n = mode_off[m + 1] - mode_off[m];
            if (n == 0) continue;
            const int4 *tk = tasks + mode_off[m];
            const int grid = (n + PROJ_WARPS - 1) / PROJ_WARPS;
            if (m == 0)
                k_project<1, 1><<<grid, PROJ_WARPS * 32, proj_smem<1, 1>(), s>>>(ddesc, tk, n, fnext);
            else if (m == 1)
                k_project<2, 2><<<grid, PROJ_WARPS * 32, proj_smem<2, 2>(), s>>>(ddesc, tk, n, fnext);
            else if (m == 2)
                k_project<2, 1><<<grid, PROJ_WARPS * 32, proj_smem<2, 1>(), s>>>(ddesc, tk, n, fnext);
            else
                k_project<1, 2><<<grid, PROJ_WARPS * 32, proj_smem<1, 2>(), s>>>(ddesc, tk, n, fnext);
        }
    }
    NOALLOC_CUDA(cudaGetLastError());
    for (uint32_t c = 0; c < nch; c++)
        NOALLOC_CUDA(cudaMemcpy2DAsync(out_planes_device[c], (size_t)out_pitch * sizeof(float), d.x + c * cstride,
                                   (size_t)pitch * sizeof(float), (size_t)W * sizeof(float), H,
                                   cudaMemcpyDeviceToDevice, s));
    unsigned flag = 0;
    NOALLOC_CUDA(cudaMemcpyAsync(&flag, errflag, sizeof(flag), cudaMemcpyDeviceToHost, s));
    NOALLOC_CUDA(cudaStreamSynchronize(s));
    if (flag) return fail(ART_ERR_INVALID_DATA, "coefficients must be integers in [-32768, 32767]");
    return ART_OK;
}
