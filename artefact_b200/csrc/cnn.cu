// Warm-start network of the restoration solver: BF16 tensor-core kernels for
// sm_100a (tcgen05 MMA with TMEM accumulators, TMA-staged operands) and the
// memory-bound glue around them. The network has no counterpart in the
// reference; it only chooses where the reference's iteration starts.
//
// Tensors are NHWC bf16: element (b, y, x, c) at ((b * H + y) * W + x) * C + c.
//
// k_conv3x3   3x3 convolution, stride 1, zero padding 1, as an implicit GEMM:
//             D[pixel][n] = sum_{tap, c} X[pixel + d(tap)][c] * Wt[n][tap][c].
//             A tile is 2 output rows x 128 pixels. TMA loads the input halo
//             (4 rows x 130 pixels, 8 channels per box, zero fill outside the
//             image) so that, with pixels stored 16 bytes apart, the A
//             operand of every tap is the same shared-memory matrix started
//             (dy + 1) * 130 + dx + 1 rows further on. The weights of one
//             channel chunk for all 9 taps come in by one bulk copy. Warp 0
//             issues the loads, warp 1 the MMAs (accumulators in TMEM, two
//             tiles in flight), warps 2-5 the epilogue (bias, ReLU, ReLU-mask,
//             accumulate, bf16 or fp32 store). Backward-data is the same kernel
//             on the output gradient with the weights flipped and transposed.
// k_wgrad3x3  weight gradient dW[n][tap][c] = sum_pixel dY[pixel][n] *
//             X[pixel + d(tap)][c]: both operands MN-major from the same kind
//             of TMA tiles; 9 tap accumulators in TMEM; one partial per band
//             of tiles, reduced in a fixed order by k_wgrad_reduce.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>

#include "art_internal.h"
#include "artefact_b200.h"
#include "solver_kernels.cuh"
#include "tc_ptx.cuh"

namespace art {
namespace cnn {

using bf16 = __nv_bfloat16;

constexpr int TPX = 128;                    // output pixels per tile row (MMA M)
constexpr int TROWS = 2;                    // weight gradient: output rows per tile (the convolution takes 2 or 4)
constexpr int HPX = TPX + 2;                // halo tile width
constexpr int HROWS = TROWS + 2;            // weight gradient: halo tile height
constexpr uint32_t KCOL = HROWS * HPX * 16; // weight gradient: bytes of one 8-channel halo column (8320, 65 x 128)
constexpr uint32_t DYREG = TROWS * TPX * 16;// bytes of one 8-channel region of a gradient tile (4096)
constexpr int THREADS = 192;                // weight gradient: warp 0 loads, warp 1 MMA, warps 2-5 epilogue
constexpr int CONV_THREADS = 320;           // convolution: warp 0 loads, warp 1 MMA, warps 2-9 epilogue
constexpr int EPI_THREADS = CONV_THREADS - 64;
constexpr uint32_t SMEM_BUDGET = 220 * 1024;  // pipeline stages; 1 KB more is requested for alignment
constexpr int MAX_STAGES = 4;
constexpr int RSTRIDE = 4;                  // channels per pixel of the head's fp32 residual output
constexpr int JOINT_RSTRIDE = 12;           // the same for the joint 4:2:0 network (three components' 2x2 cells)

struct ConvArgs {
    int B, H, W;
    int cin, ck;      // input channels (multiple of ck), channels per pipeline stage (16 or 32)
    int n, n_store;   // MMA N (multiple of 16, <= 128), channels stored (multiple of 16, <= n)
    const bf16 *wpack;  // [cin/ck][3 tap columns][ck/8][3 tap rows][n][8]
    const float *bias;  // [n] or null
    bf16 *out;
    int out_cstride, out_coff;
    float *out_f32;
    int f32_cstride, f32_n;  // fp32 output: channel stride, channels written (multiple of 4)
    const bf16 *mask;   // optional: zero where mask <= 0 (ReLU backward)
    int mask_cstride;
    int relu, accumulate;
    bf16 *pool_out;     // optional: 2x2 average of the stored output, [B][H/2][W/2][n_store]
    int up2;            // out is 2H x 2W: each pixel stored to its 2x2 cell
    int stages;
    uint32_t stage_bytes, halo_bytes;
    uint32_t tx_bytes;  // bytes the TMA and bulk copies of one stage deliver
    int *err;
};

struct WgradArgs {
    int B, H, W;
    int cout, cin, nci;  // gradient channels (<= 128), input channels, input channels per CTA (16 or 32)
    int tiles_per_band;
    float *partial;      // [bands][cin/nci][9][cout][nci]
    int stages;
    uint32_t stage_bytes;
    int *err;
};

__device__ __forceinline__ void tile_coords(int tile, int tiles_x, int tiles_y, int trows, int &b, int &y0, int &x0)
{
    const int per = tiles_x * tiles_y;
    b = tile / per;
    const int r = tile - b * per;
    y0 = (r / tiles_x) * trows;
    x0 = (r % tiles_x) * TPX;
}

// Waits without honouring the abort flag (used to drain in-flight work
// before TMEM is freed), still bounded.
__device__ __forceinline__ bool drain_wait(uint64_t *bar, uint32_t parity)
{
    int dummy = 0;
    return tc::mbar_wait(bar, parity, &dummy);
}

__device__ __forceinline__ unsigned char *aligned_smem(unsigned char *p)
{
    const uint32_t a = tc::smem_u32(p);
    return p + ((1024 - (a & 1023)) & 1023);
}

// Halo tile of one input-channel chunk (ck = 16 or 32 channels) for TR output
// rows: (TR + 2) x HPX pixels, one row of ck x 2 bytes per pixel, written by one
// TMA box with the 32- or 64-byte swizzle and read by the MMAs through swizzled
// K-major descriptors. Rounded up to 1 KB so that every stage starts on a 1 KB
// boundary.
__host__ __device__ constexpr uint32_t halo_rows(int tr) { return (uint32_t)(tr + 2) * HPX; }
__host__ __device__ constexpr uint32_t halo_bytes(int tr, int ck) { return (halo_rows(tr) * (uint32_t)ck * 2u + 1023u) / 1024u * 1024u; }

// The stacked MMAs of one (tap column, K slice) for TR output rows: halo row r
// times tap rows lo..hi (those with 0 <= r - ty < TR, from tap row LO0 on),
// into the accumulators of output rows r - hi .. r - lo (reverse column order,
// see the MMA warp in k_conv3x3). All bounds are compile-time.
template <int TR, int LO0>
__device__ __forceinline__ void issue_halo_rows(uint32_t dbase, uint64_t at, uint64_t bt, uint32_t n, uint32_t rstep,
                                                const uint32_t (&idesc)[3])
{
#pragma unroll
    for (int r = 0; r < TR + 2; r++) {
        const int lo = r - TR + 1 > LO0 ? r - TR + 1 : LO0;
        const int hi = r < 2 ? r : 2;
        if (lo > hi) continue;
        tc::mma_bf16(dbase + (uint32_t)(TR - 1 - r + lo) * n, at + (uint64_t)(r * rstep), bt + (uint64_t)lo * n,
                     idesc[hi - lo], 1);
    }
}

template <int TR>
__global__ void __launch_bounds__(CONV_THREADS, 1) k_conv3x3(const __grid_constant__ CUtensorMap xmap, const ConvArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = aligned_smem(smem_raw);
    __shared__ __align__(8) uint64_t full_bar[MAX_STAGES], empty_bar[MAX_STAGES], accf_bar[2], acce_bar[2],
        done_bar;
    __shared__ uint32_t tmem_base;
    __shared__ int abort_s;
    volatile int *abort_p = &abort_s;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_x = (a.W + TPX - 1) / TPX, tiles_y = (a.H + TR - 1) / TR;
    const int ntiles = a.B * tiles_x * tiles_y;
    const int nchunks = a.cin / a.ck;
    const int S = a.stages;

    if (threadIdx.x == 0) {
        abort_s = 0;
        for (int s = 0; s < S; s++) {
            tc::mbar_init(&full_bar[s], 1);
            tc::mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            tc::mbar_init(&accf_bar[b], 1);
            tc::mbar_init(&acce_bar[b], EPI_THREADS);
        }
        tc::mbar_init(&done_bar, 1);
        tc::fence_barrier_init();
    }
    if (warp == 1) tc::tmem_alloc(&tmem_base, 512);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tbase = tmem_base;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                int b, y0, x0;
                tile_coords(tile, tiles_x, tiles_y, TR, b, y0, x0);
                for (int c = 0; c < nchunks; c++, it++) {
                    const int s = it % S;
                    const uint32_t use = it / S;
                    if (use > 0 && !tc::mbar_wait(&empty_bar[s], (use - 1) & 1, abort_p)) {
                        ok = false;
                        break;
                    }
                    unsigned char *st = smem + (size_t)s * a.stage_bytes;
                    tc::mbar_arrive_expect_tx(&full_bar[s], a.tx_bytes);
                    tc::tma_load_4d(st, &xmap, c * a.ck, x0 - 1, y0 - 1, b, &full_bar[s]);
                    tc::bulk_load(st + a.halo_bytes, a.wpack + (size_t)c * 9 * a.ck * a.n, 18u * a.ck * a.n,
                                  &full_bar[s]);
                }
            }
            // Let the copies still in flight land before the block can exit.
            const uint32_t last = it;
            for (uint32_t k = (last > (uint32_t)S ? last - S : 0); k < last; k++)
                drain_wait(&full_bar[k % S], (k / S) & 1);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // Accumulator of output row t: TMEM columns (ab * TR + TR - 1 - t) * n,
            // n wide (rows in reverse order). Halo row r times the three tap rows
            // of one tap column stacked along N (weights of tap row ty in operand
            // rows ty*n..) adds tap row ty's products to output row r - ty, whose
            // accumulator sits ty * n columns after row r's: one MMA of up to 3n
            // columns covers every (output row, tap row) pair of that halo row
            // (the rows with r - ty outside the tile are left out of the N range).
            // A halo row meets at most min(3, TR) tap rows, and 4-row tiles have
            // n <= 64, so one MMA spans at most 256 columns.
            const uint32_t n = (uint32_t)a.n;
            const uint32_t idesc[3] = {tc::idesc_bf16(128, a.n, 0, 0),
                                       tc::idesc_bf16(128, TR >= 2 ? 2 * a.n : a.n, 0, 0),
                                       tc::idesc_bf16(128, TR >= 3 ? 3 * a.n : a.n, 0, 0)};
            // Descriptors are built once with address 0 and offset per MMA by
            // adding the operand's address / 16 to the low 14-bit field (shared
            // memory addresses stay below 256 KB, so the add never carries), which
            // keeps the issuing thread to a few instructions per MMA. The halo's
            // pixel rows are ck x 2 bytes (ru descriptor units): tap column tx and
            // halo row r start r x HPX + tx rows in. Weights: 8-channel columns
            // 3n x 16 bytes apart, tap row ty at + ty * n units.
            const uint32_t ru = (uint32_t)a.ck / 8;
            const uint64_t adesc0 = tc::smem_desc_sw(0, 8u * (uint32_t)a.ck * 2u, a.ck == 32 ? 4u : 6u);
            const uint64_t bdesc0 = tc::smem_desc(0, 3u * n * 16u, 128);
            const uint32_t nk = (uint32_t)a.ck / 16;     // K = 16 slices per chunk
            const uint32_t kcols = (uint32_t)a.ck / 8;
            uint32_t it = 0, tcount = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, tcount++) {
                const int ab = tcount & 1;
                const uint32_t ause = tcount >> 1;
                if (ause > 0 && !tc::mbar_wait(&acce_bar[ab], (ause - 1) & 1, abort_p)) break;
                tc::tc_fence_after();
                const uint32_t dbase = tbase + (uint32_t)(ab * TR) * n;
                for (int c = 0; c < nchunks; c++, it++) {
                    const int s = it % S;
                    if (!tc::mbar_wait(&full_bar[s], (it / S) & 1, abort_p)) {
                        ok = false;
                        break;
                    }
                    tc::tc_fence_after();
                    const uint32_t st4 = tc::smem_u32(smem + (size_t)s * a.stage_bytes) >> 4;
                    const uint32_t wst4 = st4 + (a.halo_bytes >> 4);
#pragma unroll
                    for (uint32_t tx = 0; tx < 3; tx++) {
#pragma unroll
                        for (uint32_t kk = 0; kk < 2; kk++) {
                            if (kk >= nk) continue;
                            const uint64_t at = adesc0 + (uint64_t)(st4 + 2 * kk + tx * ru);
                            const uint64_t bt = bdesc0 + (uint64_t)(wst4 + (tx * kcols + 2 * kk) * 3u * n);
                            // The first K slice of a tile initialises every accumulator
                            // with tap row 0 alone; everything after accumulates.
                            const uint32_t rstep = HPX * ru;
                            if (c == 0 && tx == 0 && kk == 0) {
#pragma unroll
                                for (int t = 0; t < TR; t++)
                                    tc::mma_bf16(dbase + (uint32_t)(TR - 1 - t) * n, at + (uint64_t)(t * rstep), bt,
                                                 idesc[0], 0);
                                issue_halo_rows<TR, 1>(dbase, at, bt, n, rstep, idesc);
                            } else {
                                issue_halo_rows<TR, 0>(dbase, at, bt, n, rstep, idesc);
                            }
                        }
                    }
                    tc::mma_commit(&empty_bar[s]);
                }
                if (ok) tc::mma_commit(&accf_bar[ab]);
            }
            tc::mma_commit(&done_bar);
            drain_wait(&done_bar, 0);
        }
        __syncwarp();
    } else {
        // Two warps per TMEM lane quarter (a warp reaches lanes 32 (warp % 4) ..
        // + 31 only), splitting the 16-channel groups between them.
        const int q = warp & 3;  // TMEM lanes 32q..32q+31 belong to this warp
        const int half = (warp - 2) >> 2;
        const int px = q * 32 + lane;
        constexpr int G = TR < 4 ? TR : 4;
        uint32_t tcount = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, tcount++) {
            const int ab = tcount & 1;
            // One lane waits and the warp follows its verdict, so the warp-wide
            // TMEM loads below never run with part of the warp gone.
            int ok = lane == 0 ? (int)tc::mbar_wait(&accf_bar[ab], (tcount >> 1) & 1, abort_p) : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) break;
            tc::mbar_wait(&accf_bar[ab], (tcount >> 1) & 1, abort_p);  // completes at once: every lane observes the phase
            tc::tc_fence_after();
            int b, y0, x0;
            tile_coords(tile, tiles_x, tiles_y, TR, b, y0, x0);
            const int x = x0 + px;
#pragma unroll 1
            for (int c0 = half * 16; c0 < a.n_store; c0 += 32) {
                float bias[16];
#pragma unroll
                for (int i = 0; i < 16; i++) bias[i] = a.bias ? __ldg(a.bias + c0 + i) : 0.f;
                // Rows of this channel group in groups of G (accumulator of row t
                // at column (ab * TR + TR - 1 - t) * n + c0), one wait per group.
                const uint32_t lane_base = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)c0;
#pragma unroll
                for (int g = 0; g < TR; g += G) {
                    float v[G][16];
                    if constexpr (G == 1) {
                        tc::tmem_ld16(lane_base + (uint32_t)(ab * a.n), v[0]);
                    } else if constexpr (G == 2) {
                        const uint32_t ad[2] = {lane_base + (uint32_t)((ab * TR + TR - 1 - g) * a.n),
                                                lane_base + (uint32_t)((ab * TR + TR - 2 - g) * a.n)};
                        tc::tmem_ld16x2(ad, v);
                    } else {
                        uint32_t ad[4];
#pragma unroll
                        for (int k = 0; k < 4; k++) ad[k] = lane_base + (uint32_t)((ab * TR + TR - 1 - (g + k)) * a.n);
                        tc::tmem_ld16x4(ad, v);
                    }
#pragma unroll
                    for (int t = 0; t < G; t++) {
                        const int y = y0 + g + t;
                        const bool in = y < a.H && x < a.W;
#pragma unroll
                        for (int i = 0; i < 16; i++) v[t][i] += bias[i];
                        if (a.relu) {
#pragma unroll
                            for (int i = 0; i < 16; i++) v[t][i] = fmaxf(v[t][i], 0.f);
                        }
                        if (!in) continue;
                        const size_t pix = ((size_t)b * a.H + y) * a.W + x;
                        if (a.mask) {
                            const uint4 *mp = reinterpret_cast<const uint4 *>(a.mask + pix * a.mask_cstride + c0);
                            const uint4 m2[2] = {__ldg(mp), __ldg(mp + 1)};
                            const bf16 *m = reinterpret_cast<const bf16 *>(m2);
#pragma unroll
                            for (int i = 0; i < 16; i++) v[t][i] = __bfloat162float(m[i]) > 0.f ? v[t][i] : 0.f;
                        }
                        if (a.out_f32 && c0 < a.f32_n) {
                            float4 *o = reinterpret_cast<float4 *>(a.out_f32 + pix * a.f32_cstride + c0);
#pragma unroll
                            for (int i = 0; i < 4; i++)
                                if (c0 + 4 * i < a.f32_n)
                                    o[i] = make_float4(v[t][4 * i], v[t][4 * i + 1], v[t][4 * i + 2], v[t][4 * i + 3]);
                        }
                        if (a.out) {
                            uint4 w2[2];
                            __nv_bfloat162 *w = reinterpret_cast<__nv_bfloat162 *>(w2);
                            if (a.up2) {
#pragma unroll
                                for (int i = 0; i < 8; i++) w[i] = __floats2bfloat162_rn(v[t][2 * i], v[t][2 * i + 1]);
#pragma unroll
                                for (int dy = 0; dy < 2; dy++)
#pragma unroll
                                    for (int dx = 0; dx < 2; dx++) {
                                        uint4 *o = reinterpret_cast<uint4 *>(
                                            a.out + (((size_t)b * 2 * a.H + 2 * y + dy) * 2 * a.W + 2 * x + dx) * a.out_cstride +
                                            a.out_coff + c0);
                                        o[0] = w2[0];
                                        o[1] = w2[1];
                                    }
                            } else {
                                uint4 *o = reinterpret_cast<uint4 *>(a.out + pix * a.out_cstride + a.out_coff + c0);
                                if (a.accumulate) {
                                    const uint4 p2[2] = {o[0], o[1]};
                                    const bf16 *p = reinterpret_cast<const bf16 *>(p2);
#pragma unroll
                                    for (int i = 0; i < 16; i++) v[t][i] += __bfloat162float(p[i]);
                                }
#pragma unroll
                                for (int i = 0; i < 8; i++) w[i] = __floats2bfloat162_rn(v[t][2 * i], v[t][2 * i + 1]);
                                o[0] = w2[0];
                                o[1] = w2[1];
                            }
                        }
                    }
                    if (G >= 2 && a.pool_out) {
                        // 2x2 average of the stored (bf16-rounded) values: each row pair
                        // (2 tp, 2 tp + 1) is this thread's, the column pair is this lane and
                        // its neighbour (tiles start at even rows and columns; H, W even).
#pragma unroll
                        for (int tp = 0; tp < G / 2; tp++) {
                            float pv[16];
#pragma unroll
                            for (int i = 0; i < 16; i++) {
                                const float sum = __bfloat162float(__float2bfloat16_rn(v[2 * tp][i])) +
                                                  __bfloat162float(__float2bfloat16_rn(v[2 * tp + 1][i]));
                                pv[i] = sum + __shfl_xor_sync(0xffffffffu, sum, 1);
                            }
                            const int yp = y0 + g + 2 * tp;
                            if (yp < a.H && x < a.W && (x & 1) == 0) {
                                uint4 w2[2];
                                __nv_bfloat162 *w = reinterpret_cast<__nv_bfloat162 *>(w2);
#pragma unroll
                                for (int i = 0; i < 8; i++)
                                    w[i] = __floats2bfloat162_rn(0.25f * pv[2 * i], 0.25f * pv[2 * i + 1]);
                                uint4 *o = reinterpret_cast<uint4 *>(
                                    a.pool_out + (((size_t)b * (a.H / 2) + yp / 2) * (a.W / 2) + x / 2) * a.n_store + c0);
                                o[0] = w2[0];
                                o[1] = w2[1];
                            }
                        }
                    }
                }
            }
            tc::tc_fence_before();
            tc::mbar_arrive(&acce_bar[ab]);
        }
    }

    tc::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tbase, 512);
    }
    if (threadIdx.x == 0 && abort_s) atomicExch(a.err, 1);
}

__global__ void __launch_bounds__(THREADS, 1) k_wgrad3x3(const __grid_constant__ CUtensorMap dymap,
                                                         const __grid_constant__ CUtensorMap xmap, const WgradArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = aligned_smem(smem_raw);
    __shared__ __align__(8) uint64_t full_bar[MAX_STAGES], empty_bar[MAX_STAGES], accf_bar, done_bar;
    __shared__ uint32_t tmem_base;
    __shared__ int abort_s;
    volatile int *abort_p = &abort_s;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_x = (a.W + TPX - 1) / TPX, tiles_y = (a.H + TROWS - 1) / TROWS;
    const int ntiles = a.B * tiles_x * tiles_y;
    const int band = blockIdx.x, chunk = blockIdx.y, nchunk = gridDim.y;
    const int t_begin = band * a.tiles_per_band, t_end = min(ntiles, t_begin + a.tiles_per_band);
    const int S = a.stages;
    const uint32_t dy_bytes = 16 * DYREG;  // M = 128 gradient channels: 16 regions (unused ones are never read back)

    if (threadIdx.x == 0) {
        abort_s = 0;
        for (int s = 0; s < S; s++) {
            tc::mbar_init(&full_bar[s], 1);
            tc::mbar_init(&empty_bar[s], 1);
        }
        tc::mbar_init(&accf_bar, 1);
        tc::mbar_init(&done_bar, 1);
        tc::fence_barrier_init();
    }
    if (warp == 1) tc::tmem_alloc(&tmem_base, 512);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tbase = tmem_base;

    if (warp == 0) {
        if (lane == 0) {
            const uint32_t tx_bytes = (uint32_t)(a.cout / 8) * DYREG + (uint32_t)(a.nci / 8) * KCOL;
            uint32_t it = 0;
            for (int tile = t_begin; tile < t_end; tile++, it++) {
                const int s = it % S;
                const uint32_t use = it / S;
                if (use > 0 && !tc::mbar_wait(&empty_bar[s], (use - 1) & 1, abort_p)) break;
                int b, y0, x0;
                tile_coords(tile, tiles_x, tiles_y, TROWS, b, y0, x0);
                unsigned char *st = smem + (size_t)s * a.stage_bytes;
                tc::mbar_arrive_expect_tx(&full_bar[s], tx_bytes);
                for (int g = 0; g < a.cout / 8; g++)
                    tc::tma_load_4d(st + g * DYREG, &dymap, 8 * g, x0, y0, b, &full_bar[s]);
                for (int j = 0; j < a.nci / 8; j++)
                    tc::tma_load_4d(st + dy_bytes + j * KCOL, &xmap, chunk * a.nci + 8 * j, x0 - 1, y0 - 1, b,
                                    &full_bar[s]);
            }
            const uint32_t last = it;
            for (uint32_t k = (last > (uint32_t)S ? last - S : 0); k < last; k++)
                drain_wait(&full_bar[k % S], (k / S) & 1);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_bf16(128, a.nci, 1, 1);
            uint32_t it = 0;
            bool ok = true;
            for (int tile = t_begin; tile < t_end; tile++, it++) {
                const int s = it % S;
                if (!tc::mbar_wait(&full_bar[s], (it / S) & 1, abort_p)) {
                    ok = false;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t st = tc::smem_u32(smem + (size_t)s * a.stage_bytes);
                const uint32_t xs = st + dy_bytes;
                for (int tap = 0; tap < 9; tap++) {
                    const int ty = tap / 3, tx = tap % 3;
#pragma unroll
                    for (int r = 0; r < TROWS; r++)
#pragma unroll
                        for (int k0 = 0; k0 < TPX; k0 += 16) {
                            const uint64_t adesc = tc::smem_desc(st + (uint32_t)((r * TPX + k0) * 16), 128, DYREG);
                            const uint64_t bdesc =
                                tc::smem_desc(xs + (uint32_t)(((r + ty) * HPX + k0 + tx) * 16), 128, KCOL);
                            tc::mma_bf16(tbase + (uint32_t)(tap * a.nci), adesc, bdesc, idesc,
                                         (it | r | k0) != 0);
                        }
                }
                tc::mma_commit(&empty_bar[s]);
            }
            if (ok) tc::mma_commit(&accf_bar);
            tc::mma_commit(&done_bar);
            drain_wait(&done_bar, 0);
        }
        __syncwarp();
    } else {
        const int q = warp & 3;
        const int co = q * 32 + lane;
        int ok = lane == 0 ? (int)tc::mbar_wait(&accf_bar, 0, abort_p) : 0;
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (ok) tc::mbar_wait(&accf_bar, 0, abort_p);
        if (ok) {
            tc::tc_fence_after();
            float *dst = a.partial + ((size_t)(band * nchunk + chunk) * 9) * a.cout * a.nci;
#pragma unroll 1
            for (int tap = 0; tap < 9; tap++)
#pragma unroll 1
                for (int c0 = 0; c0 < a.nci; c0 += 16) {
                    float v[16];
                    tc::tmem_ld16(tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(tap * a.nci + c0), v);
                    if (co < a.cout) {
                        float4 *o = reinterpret_cast<float4 *>(dst + ((size_t)tap * a.cout + co) * a.nci + c0);
#pragma unroll
                        for (int i = 0; i < 4; i++)
                            o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                    }
                }
        }
    }

    tc::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tbase, 512);
    }
    if (threadIdx.x == 0 && abort_s) atomicExch(a.err, 1);
}

// dW[n][tap][c] (+)= sum over bands of the partials, in band order.
__global__ void k_wgrad_reduce(const float *__restrict__ partial, int bands, int cout, int cin, int nci,
                               float *__restrict__ dw, int accumulate)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int total = cout * 9 * cin;
    if (i >= total) return;
    const int c = i % cin, tap = (i / cin) % 9, n = i / (9 * cin);
    const int chunk = c / nci, cc = c % nci, nchunk = cin / nci;
    float s = 0.f;
    for (int b = 0; b < bands; b++)
        s += partial[(((size_t)(b * nchunk + chunk) * 9 + tap) * cout + n) * nci + cc];
    dw[i] = accumulate ? dw[i] + s : s;
}

// Packs fp32 master weights W[cout][9][cin] into the bf16 layout a conv stage
// copies in one piece: [chunk][tx][ck/8][ty][n][8] with tap = 3 ty + tx, so
// the three tap rows of a tap column are one K-major operand of 3n rows.
// Forward: n = output channel, k = input channel. Transposed (backward-data):
// n = input channel ci0 + n, k = output channel, taps mirrored.
__global__ void k_pack(const float *__restrict__ w, int cout, int cin, int transpose, int ci0, int n_out, int ck,
                       bf16 *__restrict__ out)
{
    const int K = transpose ? cout : cin;
    const int total = n_out * 9 * K;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int e = i % 8;
    const int n = (i / 8) % n_out;
    const int rest = i / (8 * n_out);  // ((chunk * 3 + tx) * (ck/8) + kcol) * 3 + ty
    const int ty = rest % 3;
    const int kcol = (rest / 3) % (ck / 8);
    const int tx = (rest / (3 * (ck / 8))) % 3;
    const int chunk = rest / (9 * (ck / 8));
    const int tap = 3 * ty + tx;
    const int k = chunk * ck + kcol * 8 + e;
    float v;
    if (!transpose)
        v = (n < cout && k < cin) ? w[((size_t)n * 9 + tap) * cin + k] : 0.f;
    else
        v = (k < cout && ci0 + n < cin) ? w[((size_t)k * 9 + (8 - tap)) * cin + ci0 + n] : 0.f;
    out[i] = __float2bfloat16_rn(v);
}

// 2x2 average pooling (NHWC, 8 channels per thread) of channels
// [in_coff, in_coff + C) of a tensor with in_cstride channels.
__global__ void k_pool2(const bf16 *__restrict__ in, int B, int H, int W, int C, int in_cstride, int in_coff,
                        bf16 *__restrict__ out)
{
    const int Ho = H / 2, Wo = W / 2, cg = C / 8;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long total = (long long)B * Ho * Wo * cg;
    if (i >= total) return;
    const int g = (int)(i % cg);
    const long long p = i / cg;
    const int x = (int)(p % Wo), y = (int)((p / Wo) % Ho), b = (int)(p / ((long long)Wo * Ho));
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
#pragma unroll
        for (int dx = 0; dx < 2; dx++) {
            const uint4 r =
                __ldg(reinterpret_cast<const uint4 *>(in + (((size_t)b * H + 2 * y + dy) * W + 2 * x + dx) * in_cstride +
                                                      in_coff + 8 * g));
            const bf16 *v = reinterpret_cast<const bf16 *>(&r);
#pragma unroll
            for (int k = 0; k < 8; k++) acc[k] += __bfloat162float(v[k]);
        }
    uint4 o;
    __nv_bfloat162 *w = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
    for (int k = 0; k < 4; k++) w[k] = __floats2bfloat162_rn(0.25f * acc[2 * k], 0.25f * acc[2 * k + 1]);
    *reinterpret_cast<uint4 *>(out + (((size_t)b * Ho + y) * Wo + x) * C + 8 * g) = o;
}

// Nearest 2x upsampling of in[B][H/2][W/2][C] into channels [coff, coff + C)
// of out[B][H][W][Cs].
__global__ void k_upsample2(const bf16 *__restrict__ in, int B, int H, int W, int C, bf16 *__restrict__ out,
                            int Cs, int coff)
{
    const int cg = C / 8;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long total = (long long)B * H * W * cg;
    if (i >= total) return;
    const int g = (int)(i % cg);
    const long long p = i / cg;
    const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    const uint4 r = __ldg(
        reinterpret_cast<const uint4 *>(in + (((size_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + 8 * g));
    *reinterpret_cast<uint4 *>(out + (((size_t)b * H + y) * W + x) * Cs + coff + 8 * g) = r;
}

// Backward of nearest upsampling followed by the ReLU mask of the upsampled
// activation: out[b][y][x][c] = (sum of the 2x2 cell of g) * (act > 0).
__global__ void k_downsum2_mask(const bf16 *__restrict__ g, int B, int H, int W, int C, const bf16 *__restrict__ act,
                                bf16 *__restrict__ out)
{
    const int Ho = H / 2, Wo = W / 2, cg = C / 8;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long total = (long long)B * Ho * Wo * cg;
    if (i >= total) return;
    const int k8 = (int)(i % cg);
    const long long p = i / cg;
    const int x = (int)(p % Wo), y = (int)((p / Wo) % Ho), b = (int)(p / ((long long)Wo * Ho));
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
#pragma unroll
        for (int dx = 0; dx < 2; dx++) {
            const uint4 r =
                __ldg(reinterpret_cast<const uint4 *>(g + (((size_t)b * H + 2 * y + dy) * W + 2 * x + dx) * C + 8 * k8));
            const bf16 *v = reinterpret_cast<const bf16 *>(&r);
#pragma unroll
            for (int k = 0; k < 8; k++) acc[k] += __bfloat162float(v[k]);
        }
    const size_t o = (((size_t)b * Ho + y) * Wo + x) * C + 8 * k8;
    const uint4 ra = __ldg(reinterpret_cast<const uint4 *>(act + o));
    const bf16 *av = reinterpret_cast<const bf16 *>(&ra);
    uint4 res;
    __nv_bfloat162 *w = reinterpret_cast<__nv_bfloat162 *>(&res);
#pragma unroll
    for (int k = 0; k < 4; k++)
        w[k] = __floats2bfloat162_rn(__bfloat162float(av[2 * k]) > 0.f ? acc[2 * k] : 0.f,
                                     __bfloat162float(av[2 * k + 1]) > 0.f ? acc[2 * k + 1] : 0.f);
    *reinterpret_cast<uint4 *>(out + o) = res;
}

// Gradient of an encoder activation used both as a skip connection (gradient
// already in g) and through 2x2 average pooling (gradient gp at half
// resolution, may be null), then its ReLU mask, in place:
// g = (g + gp[up] / 4) * (act > 0); act = channels [act_coff, act_coff + C)
// of a tensor with act_cstride channels.
__global__ void k_unpool_add_mask(bf16 *__restrict__ g, const bf16 *__restrict__ gp, int B, int H, int W, int C,
                                  const bf16 *__restrict__ act, int act_cstride, int act_coff)
{
    const int cg = C / 8;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long total = (long long)B * H * W * cg;
    if (i >= total) return;
    const int k8 = (int)(i % cg);
    const long long p = i / cg;
    const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    const size_t o = (size_t)p * C + 8 * k8;
    uint4 rg = *reinterpret_cast<const uint4 *>(g + o);
    const uint4 ra = __ldg(reinterpret_cast<const uint4 *>(act + (size_t)p * act_cstride + act_coff + 8 * k8));
    uint4 rp = make_uint4(0, 0, 0, 0);
    if (gp) rp = __ldg(reinterpret_cast<const uint4 *>(gp + (((size_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + 8 * k8));
    const bf16 *gv = reinterpret_cast<const bf16 *>(&rg), *av = reinterpret_cast<const bf16 *>(&ra),
               *pv = reinterpret_cast<const bf16 *>(&rp);
    uint4 res;
    __nv_bfloat162 *w = reinterpret_cast<__nv_bfloat162 *>(&res);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        float v0 = __bfloat162float(gv[2 * k]) + 0.25f * __bfloat162float(pv[2 * k]);
        float v1 = __bfloat162float(gv[2 * k + 1]) + 0.25f * __bfloat162float(pv[2 * k + 1]);
        v0 = __bfloat162float(av[2 * k]) > 0.f ? v0 : 0.f;
        v1 = __bfloat162float(av[2 * k + 1]) > 0.f ? v1 : 0.f;
        w[k] = __floats2bfloat162_rn(v0, v1);
    }
    *reinterpret_cast<uint4 *>(g + o) = res;
}

// Per-channel sums over all pixels of g[npix][C] (bias gradient), two passes
// with a fixed order: blocks write partials, one block adds them.
__global__ void k_colsum_partial(const bf16 *__restrict__ g, long long npix, int C, float *__restrict__ partial)
{
    __shared__ float s[256];
    const int per_row = 256 / C;  // pixels handled per step by the block
    const int c = threadIdx.x % C, r = threadIdx.x / C;
    float acc = 0.f;
    if (r < per_row)
        for (long long p = (long long)blockIdx.x * per_row + r; p < npix; p += (long long)gridDim.x * per_row)
            acc += __bfloat162float(g[p * C + c]);
    s[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < C) {
        float t = 0.f;
        for (int k = 0; k < per_row; k++) t += s[k * C + threadIdx.x];
        partial[(size_t)blockIdx.x * C + threadIdx.x] = t;
    }
}

__global__ void k_colsum_final(const float *__restrict__ partial, int nblk, int C, float *__restrict__ out,
                               int accumulate)
{
    const int c = threadIdx.x;
    if (c >= C) return;
    float t = 0.f;
    for (int b = 0; b < nblk; b++) t += partial[(size_t)b * C + c];
    out[c] = accumulate ? out[c] + t : t;
}

// Network input from a coefficient image: per 8x8 block the decoded samples
// IDCT(c * q) (level-shifted, as the solver's start) into dec (fp32
// [B][H][W]) and the feature tensor F[B][H0][W0][16] (bf16) on the network's
// half-resolution grid (H0 = ceil(H / 16) * 8, W0 likewise): level-0 pixel
// (y, x) holds the 2x2 cell of samples (2y + dy, 2x + dx) -- channel 2 dy + dx
// = decoded / 128, channel 4 + 2 dy + dx = the quantisation step of that
// sample's frequency position / 64, channels 8-15 = 0; cells outside the
// component are zero. One warp per four 8x8 blocks of a row of the padded
// block grid (4x4 level-0 pixels each): lane group g = lane / 8 takes block
// 4 w + g, lane r = lane % 8 its sample row r; the 2-D IDCT runs columns then
// rows with 8x8 transposes in shared memory (the same operations, in the same
// order, as idct8x8_regs). Lane r then writes level-0 row r / 2, columns
// 2 (r % 2) and 2 (r % 2) + 1 of its block, taking the other sample row of
// each cell from lane r ^ 1.
__global__ void __launch_bounds__(128) k_features(const int16_t *__restrict__ coef, int cpitch, long long img_stride,
                                                  const float *__restrict__ q, int B, int H, int W,
                                                  float *__restrict__ dec, bf16 *__restrict__ feat)
{
    __shared__ float s_t[4][4][8][9];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bw = W / 8, bh = H / 8;
    const int W0 = (W + 15) / 16 * 8, H0 = (H + 15) / 16 * 8;
    const int pbw = W0 / 4, pbh = H0 / 4;  // padded block grid
    const int gx = (pbw + 3) / 4;          // warps per padded block row
    const long long wi = blockIdx.x * 4LL + warp;
    if (wi >= (long long)B * pbh * gx) return;  // warp-uniform
    const int grp = lane >> 3, r = lane & 7;
    const int bx = (int)(wi % gx) * 4 + grp, by = (int)((wi / gx) % pbh), b = (int)(wi / ((long long)gx * pbh));
    const bool real = bx < bw && by < bh;
    const float *qt = q + (size_t)b * 64;
    float(*T)[9] = s_t[warp][grp];
    float a[8];
    if (real) {
        load_coef_row(coef + b * img_stride + (size_t)(by * 8 + r) * cpitch + bx * 8, a);
#pragma unroll
        for (int u = 0; u < 8; u++) a[u] *= __ldg(qt + r * 8 + u);
    } else {
#pragma unroll
        for (int u = 0; u < 8; u++) a[u] = 0.f;
    }
    transpose8(T, r, a);
    idct8(a);
    transpose8(T, r, a);
    idct8(a);
    if (real) {
        float4 *d = reinterpret_cast<float4 *>(dec + ((size_t)b * H + by * 8 + r) * W + bx * 8);
        d[0] = make_float4(a[0], a[1], a[2], a[3]);
        d[1] = make_float4(a[4], a[5], a[6], a[7]);
    }
    float o8[8];
#pragma unroll
    for (int u = 0; u < 8; u++) o8[u] = __shfl_xor_sync(0xffffffffu, a[u], 1);
    if (bx >= pbw || !feat) return;
    const int yy = r >> 1, h = r & 1;
#pragma unroll
    for (int k2 = 0; k2 < 2; k2++) {
        const int xx = 2 * h + k2;
        uint4 o[2] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
        if (real) {
            bf16 *w = reinterpret_cast<bf16 *>(o);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int dy = k >> 1, dx = k & 1;
                const int clo = 2 * k2 + dx, chi = 4 + 2 * k2 + dx;  // sample column for h = 0 / 1
                // Row 2 yy is this lane's for h = 0, its partner's for h = 1.
                const float v = dy == 0 ? (h ? o8[chi] : a[clo]) : (h ? a[chi] : o8[clo]);
                w[k] = __float2bfloat16_rn(v * (1.f / 128.f));
                w[4 + k] = __float2bfloat16_rn(__ldg(qt + (2 * yy + dy) * 8 + 2 * xx + dx) * (1.f / 64.f));
            }
        }
        uint4 *f = reinterpret_cast<uint4 *>(feat + (((size_t)b * H0 + by * 4 + yy) * W0 + bx * 4 + xx) * 16);
        f[0] = o[0];
        f[1] = o[1];
    }
}

// Residual head output r (fp32 [B][H0][W0][rstride], channels 0-3 = the 2x2
// cell of a level-0 pixel, channel 2 dy + dx) -> prediction x = dec + 16 r at
// full resolution [B][H][W]; with a target: gradient of the mean squared error
// over the B H W samples (in units of 16 levels) into grad[B][H0][W0][16]
// (channels 0-3; the rest and cells outside the component zero) and per-block
// partial sums of the squared error. One thread per level-0 pixel.
__global__ void k_residual(const float *__restrict__ r, int rstride, const float *__restrict__ dec,
                           const float *__restrict__ target, int B, int H, int W, float inv_count,
                           float *__restrict__ pred, bf16 *__restrict__ grad, float *__restrict__ loss_partial)
{
    __shared__ float s[256];
    const int W0 = (W + 15) / 16 * 8, H0 = (H + 15) / 16 * 8;
    const long long n0 = (long long)B * H0 * W0;
    float acc = 0.f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n0; p += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(p % W0), y = (int)((p / W0) % H0), b = (int)(p / ((long long)W0 * H0));
        uint4 o[2] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
        bf16 *gv = reinterpret_cast<bf16 *>(o);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int Y = 2 * y + (k >> 1), X = 2 * x + (k & 1);
            if (Y >= H || X >= W) continue;
            const size_t q = ((size_t)b * H + Y) * W + X;
            const float rv = r[p * rstride + k];
            const float d = dec[q];
            if (pred) pred[q] = d + 16.f * rv;
            if (target) {
                const float e = rv - (target[q] - d) * (1.f / 16.f);
                acc += e * e;
                gv[k] = __float2bfloat16_rn(2.f * e * inv_count);
            }
        }
        if (target) {
            uint4 *g = reinterpret_cast<uint4 *>(grad + p * 16);
            g[0] = o[0];
            g[1] = o[1];
        }
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss_partial) loss_partial[blockIdx.x] = s[0];
}

// Self-test of the bounded wait every tensor-core pipeline uses: thread 0
// waits on an mbarrier phase that nothing completes. After `limit` clock
// cycles the wait gives up and raises the abort flag, and the kernel writes
// 1 to *err and returns -- what the pipelines do when a partner role stalls,
// leaving the context usable. 0 would mean the phase completed (impossible here).
__global__ void k_wait_selftest(int *err, long long limit)
{
    __shared__ __align__(8) uint64_t bar;
    __shared__ int abort_s;
    if (threadIdx.x == 0) {
        abort_s = 0;
        tc::mbar_init(&bar, 1);
        tc::fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile int *ab = &abort_s;
        const bool ok = tc::mbar_wait_limit(&bar, 0, ab, limit);
        *err = ok ? 0 : 1;
    }
}

// Gradient of the training loss with a smoothness term: with e = (pred -
// target) / 16 per sample, L = (sum e^2 + lambda sum over horizontally and
// vertically adjacent pairs (e_p - e_q)^2) / n, so dL/de_p = (2 e_p + 2 lambda
// sum_{q adjacent to p} (e_p - e_q)) / n. Overwrites channels 0-3 of
// grad[B][H0][W0][16] and writes per-block partial sums of the pair term
// (times lambda). One thread per level-0 pixel (its 2x2 cell).
__global__ void k_residual_smooth_grad(const float *__restrict__ pred, const float *__restrict__ target, int B, int H,
                                       int W, float lambda, float inv_count, bf16 *__restrict__ grad,
                                       float *__restrict__ loss_partial)
{
    __shared__ float s[256];
    const int W0 = (W + 15) / 16 * 8, H0 = (H + 15) / 16 * 8;
    const long long n0 = (long long)B * H0 * W0;
    auto err = [&](int b, int Y, int X) {
        const size_t q = ((size_t)b * H + Y) * W + X;
        return (pred[q] - target[q]) * (1.f / 16.f);
    };
    float acc = 0.f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n0; p += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(p % W0), y = (int)((p / W0) % H0), b = (int)(p / ((long long)W0 * H0));
        uint4 o[2] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
        bf16 *gv = reinterpret_cast<bf16 *>(o);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int Y = 2 * y + (k >> 1), X = 2 * x + (k & 1);
            if (Y >= H || X >= W) continue;
            const float e = err(b, Y, X);
            float lap = 0.f;
            if (X > 0) lap += e - err(b, Y, X - 1);
            if (X < W - 1) {
                const float d = e - err(b, Y, X + 1);
                lap += d;
                acc += d * d;
            }
            if (Y > 0) lap += e - err(b, Y - 1, X);
            if (Y < H - 1) {
                const float d = e - err(b, Y + 1, X);
                lap += d;
                acc += d * d;
            }
            gv[k] = __float2bfloat16_rn((2.f * e + 2.f * lambda * lap) * inv_count);
        }
        uint4 *g = reinterpret_cast<uint4 *>(grad + p * 16);
        g[0] = o[0];
        g[1] = o[1];
    }
    s[threadIdx.x] = lambda * acc;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss_partial[blockIdx.x] = s[0];
}

// ---------------------------------------------------------------------------
// Joint 4:2:0 network input and output. The luma's level-0 grid (a 2x2 luma
// cell per pixel) is the chroma components' sample grid, so one pass over it
// sees all three components: each level-0 pixel also carries one sample of
// Cb and of Cr, and the head's outputs 4-7 / 8-11 are the 2x2 full-resolution
// chroma cells, which the chroma's own resolution cannot express.

// Smooth 2x upsampling weights of the solver's learned start: 3/4 of the own
// cell, 1/4 of the neighbour on the sample's side, each product and sum
// rounded on its own.
__device__ __forceinline__ float tri_mix(float a, float b) { return __fadd_rn(__fmul_rn(0.75f, a), __fmul_rn(0.25f, b)); }

// One thread per level-0 pixel (y, x) of image b: channels 8-11 of feat
// [B][H0][W0][16] = decoded Cb sample / 128, its quantisation step / 64 (the
// step of its frequency position in its block), the same for Cr; and the
// chroma bases, the decoded chroma upsampled smoothly to full resolution,
// into planes 1 and 2 of dec[3][B][H][W]. decC[B][2][H/2][W/2] holds the
// decoded chroma, qc[B][2][64] their tables. H, W multiples of 16.
__global__ void k_features_joint(const float *__restrict__ decC, const float *__restrict__ qc, int B, int H, int W,
                                 float *__restrict__ dec, bf16 *__restrict__ feat)
{
    const int Wc = W / 2, Hc = H / 2;
    const long long n0 = (long long)B * Hc * Wc, plane = (long long)B * H * W;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n0; p += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(p % Wc), y = (int)((p / Wc) % Hc), b = (int)(p / ((long long)Wc * Hc));
        bf16 f[4];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const float *c = decC + ((size_t)b * 2 + k) * Hc * Wc;
            f[2 * k] = __float2bfloat16_rn(c[(size_t)y * Wc + x] * (1.f / 128.f));
            f[2 * k + 1] = __float2bfloat16_rn(__ldg(qc + ((size_t)b * 2 + k) * 64 + (y & 7) * 8 + (x & 7)) * (1.f / 64.f));
#pragma unroll
            for (int d = 0; d < 4; d++) {
                const int dy = d >> 1, dx = d & 1;
                const int nx = dx ? min(x + 1, Wc - 1) : max(x - 1, 0), ny = dy ? min(y + 1, Hc - 1) : max(y - 1, 0);
                const float *r0 = c + (size_t)y * Wc, *r1 = c + (size_t)ny * Wc;
                const float v = tri_mix(tri_mix(r0[x], r0[nx]), tri_mix(r1[x], r1[nx]));
                dec[(1 + k) * plane + ((size_t)b * H + 2 * y + dy) * W + 2 * x + dx] = v;
            }
        }
        uint2 o;
        memcpy(&o, f, 8);
        *reinterpret_cast<uint2 *>(feat + p * 16 + 8) = o;
    }
}

// Joint residual head output r (fp32 [B][H0][W0][rstride], channels 4 c + 2 dy
// + dx = sample (2 y + dy, 2 x + dx) of component c) -> prediction dec + 16 r
// of sample (c, b, Y, X) at pred[c ocs + (b H + Y) opitch + X] (and at the
// same place of pred2 when given: the solver's two state buffers); with a
// target [3][B][H][W]: gradient of the mean squared error over the 3 B H W
// samples (the luma's weighted by luma_w) into channels 0-11 of
// grad[B][H0][W0][16], per-block partial sums of the weighted squared error.
__global__ void k_residual_joint(const float *__restrict__ r, int rstride, const float *__restrict__ dec,
                                 const float *__restrict__ target, int B, int H, int W, float inv_count, float luma_w,
                                 float *__restrict__ pred, float *__restrict__ pred2, long long ocs, int opitch,
                                 bf16 *__restrict__ grad, float *__restrict__ loss_partial)
{
    __shared__ float s[256];
    const int W0 = W / 2, H0 = H / 2;
    const long long n0 = (long long)B * H0 * W0, plane = (long long)B * H * W;
    float acc = 0.f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n0; p += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(p % W0), y = (int)((p / W0) % H0), b = (int)(p / ((long long)W0 * H0));
        uint4 o[2] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
        bf16 *gv = reinterpret_cast<bf16 *>(o);
#pragma unroll
        for (int c = 0; c < 3; c++) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int Y = 2 * y + (k >> 1), X = 2 * x + (k & 1);
                const size_t q = c * plane + ((size_t)b * H + Y) * W + X;
                const float rv = r[p * rstride + 4 * c + k];
                const float d = dec[q];
                if (pred) {
                    const size_t o = c * ocs + ((size_t)b * H + Y) * opitch + X;
                    const float v = d + 16.f * rv;
                    pred[o] = v;
                    if (pred2) pred2[o] = v;
                }
                if (target) {
                    const float e = rv - (target[q] - d) * (1.f / 16.f), wc = c == 0 ? luma_w : 1.f;
                    acc += wc * e * e;
                    gv[4 * c + k] = __float2bfloat16_rn(2.f * wc * e * inv_count);
                }
            }
        }
        if (target) {
            uint4 *g = reinterpret_cast<uint4 *>(grad + p * 16);
            g[0] = o[0];
            g[1] = o[1];
        }
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss_partial) loss_partial[blockIdx.x] = s[0];
}

// ---------------------------------------------------------------------------
// Objective term of the training loss. The solver judges a start by its
// objective, not by its distance to a converged image, so training can add
// lambda E(x) / n to the mean squared error, where x = proj(pred) is the
// prediction projected onto the quantisation box per 8x8 block (DCT, clamp to
// [(c - 1/2) q, (c + 1/2) q], IDCT: compute_projection.rs:8-122 on a component
// at its own resolution) and E is the solver's objective of one channel:
// a_tv sum |grad x| (compute_step_tv.rs:29-93), a_tgv sum of the second-order
// norm (compute_step_tv2.rs:32-136) and a_p sum (DCT(x) - c q)^2 / (2 q^2)
// (compute_step_prob.rs:5-60). Its gradient with respect to pred is
// J^T grad E(x) with J = IDCT diag(m) DCT, m = 1 on the coefficients the clamp
// left alone; the transform is orthonormal, so J^T = J. Three kernels:
// project (per block), terms (per sample), gather + back-projection.

__device__ __forceinline__ void block_reduce_store(float acc, float *out)
{
    __shared__ float s[256];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

// One thread per 8x8 block: x = proj(pred), the DCT-distance gradient plane
// P = a_p IDCT((cos - c q) / q^2) of the clamped coefficients cos, the mask of
// unclamped coefficients, and partial sums of the DCT-distance value.
__global__ void __launch_bounds__(256) k_obj_project(const float *__restrict__ pred, const int16_t *__restrict__ coef,
                                                     int cpitch, long long img_stride, const float *__restrict__ q,
                                                     int B, int H, int W, float a_p, float *__restrict__ x,
                                                     float *__restrict__ P, unsigned long long *__restrict__ mask,
                                                     float *__restrict__ partial)
{
    const int bw = W / 8, bh = H / 8;
    const long long nblk = (long long)B * bw * bh;
    float acc = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nblk; i += (long long)gridDim.x * blockDim.x) {
        const int bx = (int)(i % bw), by = (int)((i / bw) % bh), b = (int)(i / ((long long)bw * bh));
        const size_t o = ((size_t)b * H + by * 8) * W + bx * 8;
        float a[64], d[64];
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const float4 *s = reinterpret_cast<const float4 *>(pred + o + (size_t)r * W);
            const float4 u = s[0], v = s[1];
            a[r * 8 + 0] = u.x, a[r * 8 + 1] = u.y, a[r * 8 + 2] = u.z, a[r * 8 + 3] = u.w;
            a[r * 8 + 4] = v.x, a[r * 8 + 5] = v.y, a[r * 8 + 6] = v.z, a[r * 8 + 7] = v.w;
        }
        dct8x8_regs(a);
        const float *qt = q + (size_t)b * 64;
        unsigned long long m = 0;
#pragma unroll
        for (int r = 0; r < 8; r++) {
            float c[8];
            load_coef_row(coef + b * img_stride + (size_t)(by * 8 + r) * cpitch + bx * 8, c);
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int j = r * 8 + u;
                const float qj = __ldg(qt + j), cq = c[u] * qj;
                const float lo = (c[u] - 0.5f) * qj, hi = (c[u] + 0.5f) * qj;
                const float v = fminf(fmaxf(a[j], lo), hi);
                if (v == a[j]) m |= 1ull << j;
                a[j] = v;
                d[j] = (v - cq) / (qj * qj);
                acc += 0.5f * a_p * d[j] * (v - cq);
            }
        }
        idct8x8_regs(a);
        idct8x8_regs(d);
#pragma unroll
        for (int r = 0; r < 8; r++) {
            float4 *xs = reinterpret_cast<float4 *>(x + o + (size_t)r * W);
            float4 *ps = reinterpret_cast<float4 *>(P + o + (size_t)r * W);
            xs[0] = make_float4(a[r * 8 + 0], a[r * 8 + 1], a[r * 8 + 2], a[r * 8 + 3]);
            xs[1] = make_float4(a[r * 8 + 4], a[r * 8 + 5], a[r * 8 + 6], a[r * 8 + 7]);
            ps[0] = make_float4(a_p * d[r * 8 + 0], a_p * d[r * 8 + 1], a_p * d[r * 8 + 2], a_p * d[r * 8 + 3]);
            ps[1] = make_float4(a_p * d[r * 8 + 4], a_p * d[r * 8 + 5], a_p * d[r * 8 + 6], a_p * d[r * 8 + 7]);
        }
        mask[i] = m;
    }
    block_reduce_store(acc, partial);
}

// One thread per sample of x: the TV and TGV terms centred on it, scaled by
// their weights and divided by their norms, as five planes
// T = [a_tv dx/n, a_tv dy/n, a_tgv xx/n2, a_tgv yy/n2, a_tgv s/n2] (zero where a
// norm is zero), with the edge rules of the reference's scatter: forward
// differences vanish on the last column / row, backward ones on the first.
// Partial sums of a_tv n + a_tgv n2.
__global__ void __launch_bounds__(256) k_obj_terms(const float *__restrict__ x, int B, int H, int W, float a_tv,
                                                   float a_tgv, float *__restrict__ T, float *__restrict__ partial)
{
    const long long n = (long long)B * H * W;
    float acc = 0.f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const int X = (int)(p % W), Y = (int)((p / W) % H);
        const float *im = x + (p - (long long)Y * W - X);
        auto at = [&](int yy, int xx) { return __ldg(im + (size_t)yy * W + xx); };
        const float v = at(Y, X);
        const float dX = X < W - 1 ? at(Y, X + 1) - v : 0.f, dY = Y < H - 1 ? at(Y + 1, X) - v : 0.f;
        float xx = 0.f, yy = 0.f, gyx = 0.f, gxy = 0.f;
        if (X > 0) {
            const float l = at(Y, X - 1);
            const float dYl = Y < H - 1 ? at(Y + 1, X - 1) - l : 0.f;
            xx = dX - (v - l);
            gyx = dY - dYl;
        }
        if (Y > 0) {
            const float u = at(Y - 1, X);
            const float dXu = X < W - 1 ? at(Y - 1, X + 1) - u : 0.f;
            yy = dY - (v - u);
            gxy = dX - dXu;
        }
        const float s = 0.5f * (gxy + gyx);
        const float n1 = sqrtf(dX * dX + dY * dY), n2 = sqrtf(yy * yy + 2.f * s * s + xx * xx);
        const float i1 = n1 > 0.f ? a_tv / n1 : 0.f, i2 = n2 > 0.f ? a_tgv / n2 : 0.f;
        T[p] = i1 * dX;
        T[n + p] = i1 * dY;
        T[2 * n + p] = i2 * xx;
        T[3 * n + p] = i2 * yy;
        T[4 * n + p] = i2 * s;
        acc += a_tv * n1 + a_tgv * n2;
    }
    block_reduce_store(acc, partial);
}

// One thread per 8x8 block: g = grad E(x) at its 64 samples (the gather of the
// terms' scatter, plus P), then J g = IDCT(m DCT(g)), and the loss gradient
// with respect to the residual head's four cell outputs,
// 2 e / n + lambda 16 (J g) / n with e = (pred - target) / 16, written over
// channels 0-3 of grad[B][H0][W0][16].
__global__ void __launch_bounds__(256) k_obj_back(const float *__restrict__ T, const float *__restrict__ P,
                                                  const unsigned long long *__restrict__ mask,
                                                  const float *__restrict__ pred, const float *__restrict__ target,
                                                  int B, int H, int W, float lambda, float inv_count,
                                                  bf16 *__restrict__ grad)
{
    const int bw = W / 8, bh = H / 8;
    const int W0 = (W + 15) / 16 * 8, H0 = (H + 15) / 16 * 8;
    const long long nblk = (long long)B * bw * bh, n = (long long)B * H * W;
    const float *T0 = T, *T1 = T + n, *T2 = T + 2 * n, *T3 = T + 3 * n, *T4 = T + 4 * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nblk; i += (long long)gridDim.x * blockDim.x) {
        const int bx = (int)(i % bw), by = (int)((i / bw) % bh), b = (int)(i / ((long long)bw * bh));
        const size_t base = (size_t)b * H * W;
        float a[64];
#pragma unroll
        for (int r = 0; r < 8; r++) {
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int Y = by * 8 + r, X = bx * 8 + u;
                const size_t p = base + (size_t)Y * W + X;
                float g = -(T0[p] + T1[p]) - 2.f * (T3[p] + T2[p] + T4[p]) + P[p];
                if (X > 0) g += T0[p - 1] + T4[p - 1] + T2[p - 1];
                if (Y > 0) g += T1[p - W] + T3[p - W] + T4[p - W];
                if (X < W - 1) g += T4[p + 1] + T2[p + 1];
                if (Y < H - 1) g += T3[p + W] + T4[p + W];
                if (X > 0 && Y < H - 1) g -= T4[p + W - 1];
                if (X < W - 1 && Y > 0) g -= T4[p - W + 1];
                a[r * 8 + u] = g;
            }
        }
        dct8x8_regs(a);
        const unsigned long long m = mask[i];
#pragma unroll
        for (int j = 0; j < 64; j++)
            if (!((m >> j) & 1ull)) a[j] = 0.f;
        idct8x8_regs(a);
#pragma unroll
        for (int r = 0; r < 8; r++) {
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int Y = by * 8 + r, X = bx * 8 + u;
                const size_t p = base + (size_t)Y * W + X;
                const float e = (pred[p] - target[p]) * (1.f / 16.f);
                const float gr = (2.f * e + lambda * 16.f * a[r * 8 + u]) * inv_count;
                grad[(((size_t)b * H0 + (Y >> 1)) * W0 + (X >> 1)) * 16 + ((Y & 1) << 1) + (X & 1)] =
                    __float2bfloat16_rn(gr);
            }
        }
    }
}

// Adam on flat fp32 parameters (decoupled from the bf16 copies the convs read).
__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

// ---------------------------------------------------------------------------
// Host side.

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Tensor map over an NHWC bf16 tensor [B][H][W][C] with box {8, bw, bh, 1}.
// NHWC bf16 tensor map with boxes of bc channels x bw pixels x bh rows; bc = 8
// unswizzled, 16 with the 32-byte swizzle, 32 with the 64-byte swizzle.
bool make_map(CUtensorMap *m, const void *base, int B, int H, int W, int C, int bw, int bh, std::string &err,
              int bc = 8)
{
    auto fn = encode_fn();
    if (!fn) {
        err = "cuTensorMapEncodeTiled is unavailable";
        return false;
    }
    if ((reinterpret_cast<uintptr_t>(base) & 15) || C % 8) {
        err = "tensor base must be 16-byte aligned and channels a multiple of 8";
        return false;
    }
    cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    cuuint32_t box[4] = {(cuuint32_t)bc, (cuuint32_t)bw, (cuuint32_t)bh, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    const CUtensorMapSwizzle sw = bc == 32 ? CU_TENSOR_MAP_SWIZZLE_64B
                                  : bc == 16 ? CU_TENSOR_MAP_SWIZZLE_32B
                                             : CU_TENSOR_MAP_SWIZZLE_NONE;
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
        return false;
    }
    return true;
}

// Raises a kernel's dynamic shared-memory limit to the pipeline budget, once
// per device (slot: which kernel).
void set_smem_attribute_once(const void *fn, int slot)
{
    static std::mutex mu;
    static bool done[64][5] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && done[dev][slot]) return;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(SMEM_BUDGET + 1024));
    if (dev >= 0 && dev < 64) done[dev][slot] = true;
}

int num_sms()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

int32_t fail(int32_t code, const std::string &msg)
{
    set_error(msg);
    return code;
}

int32_t check_launch(const char *what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ART_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return ART_OK;
}

// Output rows per tile when the caller leaves it open. Taller tiles re-read
// fewer halo rows, reload the chunk's weights for more output rows and give
// the stacked tap-row MMAs more rows to span; shorter ones give small layers
// enough tiles to occupy the SMs. Two tiles' accumulators (2 x rows x n
// columns) fit TMEM's 512. Measured on the network's 1080p layers: 8 rows
// best or tied for n <= 32 without a pooled output, 4 rows for n <= 64, and
// for n > 64 one row where 2-row tiles would cover under half the SMs.
int auto_tile_rows(int B, int H, int W, int n, bool pooled)
{
    const long long tiles2 = (long long)B * ((H + 1) / 2) * ((W + TPX - 1) / TPX);
    if (n <= 32 && !pooled) return 8;
    if (n <= 64) return 4;
    if (2 * tiles2 < num_sms() && !pooled) return 1;
    return 2;
}

int32_t conv3x3(const ArtCnnConv *d, cudaStream_t s)
{
    if (!d || !d->x || !d->wpack || !d->err) return fail(ART_ERR_INVALID_ARGUMENT, "conv: null pointer");
    if (d->B < 1 || d->H < 1 || d->W < 1) return fail(ART_ERR_INVALID_ARGUMENT, "conv: empty tensor");
    if (d->ck != 16 && d->ck != 32) return fail(ART_ERR_INVALID_ARGUMENT, "conv: ck must be 16 or 32");
    if (d->cin < d->ck || d->cin % d->ck) return fail(ART_ERR_INVALID_ARGUMENT, "conv: cin must be a multiple of ck");
    if (d->n < 16 || d->n > 128 || d->n % 16) return fail(ART_ERR_INVALID_ARGUMENT, "conv: n must be 16..128, multiple of 16");
    if (d->n_store < 16 || d->n_store > d->n || d->n_store % 16)
        return fail(ART_ERR_INVALID_ARGUMENT, "conv: n_store must be a multiple of 16 and at most n");
    if (!d->out && !d->out_f32) return fail(ART_ERR_INVALID_ARGUMENT, "conv: no output");
    if (d->out && (d->out_cstride % 8 || d->out_coff % 8 || d->out_coff + d->n_store > d->out_cstride))
        return fail(ART_ERR_INVALID_ARGUMENT, "conv: bad output channel stride/offset");
    const int f32_n = d->f32_channels ? d->f32_channels : d->n_store;
    if (d->out_f32 && (d->f32_channels < 0 || f32_n % 4 || f32_n > d->n_store || d->f32_cstride % 4 ||
                       d->f32_cstride < f32_n))
        return fail(ART_ERR_INVALID_ARGUMENT, "conv: bad fp32 output channels or stride");
    if (d->mask && (d->mask_cstride % 8 || d->mask_cstride < d->n_store))
        return fail(ART_ERR_INVALID_ARGUMENT, "conv: bad mask stride");
    if ((long long)d->B * d->H * d->W * (long long)d->cin >= (1LL << 40))
        return fail(ART_ERR_INVALID_ARGUMENT, "conv: tensor too large");
    if (d->pool_out && (d->H % 2 || d->W % 2 || d->mask))
        return fail(ART_ERR_INVALID_ARGUMENT, "conv: pooled output needs even H and W and no mask");
    if (d->up2 && (!d->out || d->accumulate || d->mask))
        return fail(ART_ERR_INVALID_ARGUMENT, "conv: upsampled output needs out, no accumulate and no mask");
    if (d->tile_rows != 0 && d->tile_rows != 1 && d->tile_rows != 2 && d->tile_rows != 4 && d->tile_rows != 8)
        return fail(ART_ERR_INVALID_ARGUMENT, "conv: tile_rows must be 0, 1, 2, 4 or 8");
    if (d->tile_rows * d->n > 256)
        return fail(ART_ERR_INVALID_ARGUMENT, "conv: tile_rows x n must be at most 256 (TMEM holds 2 tiles' accumulators)");
    if (d->tile_rows == 1 && d->pool_out)
        return fail(ART_ERR_INVALID_ARGUMENT, "conv: a pooled output needs 2- or 4-row tiles");
    const int trows = d->tile_rows ? d->tile_rows : auto_tile_rows(d->B, d->H, d->W, d->n, d->pool_out != nullptr);
    CUtensorMap map;
    std::string err;
    if (!make_map(&map, d->x, d->B, d->H, d->W, d->cin, HPX, trows + 2, err, d->ck))
        return fail(ART_ERR_CUDA, "conv: " + err);
    ConvArgs a{};
    a.B = d->B;
    a.H = d->H;
    a.W = d->W;
    a.cin = d->cin;
    a.ck = d->ck;
    a.n = d->n;
    a.n_store = d->n_store;
    a.wpack = static_cast<const bf16 *>(d->wpack);
    a.bias = d->bias;
    a.out = static_cast<bf16 *>(d->out);
    a.out_cstride = d->out_cstride;
    a.out_coff = d->out_coff;
    a.out_f32 = d->out_f32;
    a.f32_cstride = d->f32_cstride;
    a.f32_n = f32_n;
    a.mask = static_cast<const bf16 *>(d->mask);
    a.mask_cstride = d->mask_cstride;
    a.relu = d->relu;
    a.accumulate = d->accumulate;
    a.pool_out = static_cast<bf16 *>(d->pool_out);
    a.up2 = d->up2;
    a.halo_bytes = halo_bytes(trows, d->ck);
    a.stage_bytes = (a.halo_bytes + 18u * d->ck * d->n + 1023u) / 1024u * 1024u;
    a.tx_bytes = halo_rows(trows) * (uint32_t)d->ck * 2u + 18u * d->ck * d->n;
    a.stages = (int)std::min<uint32_t>(MAX_STAGES, SMEM_BUDGET / a.stage_bytes);
    a.err = d->err;
    if (a.stages < 2) return fail(ART_ERR_INVALID_ARGUMENT, "conv: stage does not fit shared memory");
    const uint32_t smem = a.stages * a.stage_bytes + 1024;
    const long long ntiles = (long long)d->B * ((d->H + trows - 1) / trows) * ((d->W + TPX - 1) / TPX);
    const int grid = (int)std::min<long long>(ntiles, num_sms());
    if (trows == 8) {
        set_smem_attribute_once(reinterpret_cast<const void *>(k_conv3x3<8>), 4);
        k_conv3x3<8><<<grid, CONV_THREADS, smem, s>>>(map, a);
    } else if (trows == 4) {
        set_smem_attribute_once(reinterpret_cast<const void *>(k_conv3x3<4>), 2);
        k_conv3x3<4><<<grid, CONV_THREADS, smem, s>>>(map, a);
    } else if (trows == 1) {
        set_smem_attribute_once(reinterpret_cast<const void *>(k_conv3x3<1>), 3);
        k_conv3x3<1><<<grid, CONV_THREADS, smem, s>>>(map, a);
    } else {
        set_smem_attribute_once(reinterpret_cast<const void *>(k_conv3x3<2>), 0);
        k_conv3x3<2><<<grid, CONV_THREADS, smem, s>>>(map, a);
    }
    return check_launch("k_conv3x3");
}

int32_t wgrad3x3(const ArtCnnWgrad *d, cudaStream_t s)
{
    if (!d || !d->x || !d->dy || !d->dw || !d->workspace || !d->err)
        return fail(ART_ERR_INVALID_ARGUMENT, "wgrad: null pointer");
    if (d->B < 1 || d->H < 1 || d->W < 1) return fail(ART_ERR_INVALID_ARGUMENT, "wgrad: empty tensor");
    if (d->cout < 8 || d->cout > 128 || d->cout % 8) return fail(ART_ERR_INVALID_ARGUMENT, "wgrad: cout must be 8..128, multiple of 8");
    const int nci = d->cin % 32 == 0 ? 32 : 16;
    if (d->cin < 16 || d->cin % 16) return fail(ART_ERR_INVALID_ARGUMENT, "wgrad: cin must be a multiple of 16");
    const long long ntiles = (long long)d->B * ((d->H + TROWS - 1) / TROWS) * ((d->W + TPX - 1) / TPX);
    const int nchunk = d->cin / nci;
    int bands = (int)std::max<long long>(1, std::min<long long>(ntiles, (2LL * num_sms() + nchunk - 1) / nchunk));
    const long long per_band_bytes = (long long)nchunk * 9 * d->cout * nci * 4;
    bands = (int)std::min<long long>(bands, std::max<long long>(1, (long long)d->workspace_bytes / per_band_bytes));
    if (per_band_bytes > (long long)d->workspace_bytes) return fail(ART_ERR_INVALID_ARGUMENT, "wgrad: workspace too small");
    const int tpb = (int)((ntiles + bands - 1) / bands);
    bands = (int)((ntiles + tpb - 1) / tpb);
    CUtensorMap dymap, xmap;
    std::string err;
    if (!make_map(&dymap, d->dy, d->B, d->H, d->W, d->cout, TPX, TROWS, err)) return fail(ART_ERR_CUDA, "wgrad: " + err);
    if (!make_map(&xmap, d->x, d->B, d->H, d->W, d->cin, HPX, HROWS, err)) return fail(ART_ERR_CUDA, "wgrad: " + err);
    WgradArgs a{};
    a.B = d->B;
    a.H = d->H;
    a.W = d->W;
    a.cout = d->cout;
    a.cin = d->cin;
    a.nci = nci;
    a.tiles_per_band = tpb;
    a.partial = static_cast<float *>(d->workspace);
    a.stage_bytes = 16 * DYREG + (uint32_t)(nci / 8) * KCOL;
    a.stages = (int)std::min<uint32_t>(MAX_STAGES, SMEM_BUDGET / a.stage_bytes);
    a.err = d->err;
    set_smem_attribute_once(reinterpret_cast<const void *>(k_wgrad3x3), 1);
    k_wgrad3x3<<<dim3(bands, nchunk), THREADS, a.stages * a.stage_bytes + 1024, s>>>(dymap, xmap, a);
    int32_t rc = check_launch("k_wgrad3x3");
    if (rc) return rc;
    const int total = d->cout * 9 * d->cin;
    k_wgrad_reduce<<<(total + 255) / 256, 256, 0, s>>>(a.partial, bands, d->cout, d->cin, nci, d->dw, d->accumulate);
    return check_launch("k_wgrad_reduce");
}

inline unsigned blocks_for(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace cnn
}  // namespace art

using namespace art::cnn;

extern "C" {

int32_t art_cnn_conv3x3(const ArtCnnConv *desc, void *stream)
{
    return conv3x3(desc, static_cast<cudaStream_t>(stream));
}

int32_t art_cnn_wgrad3x3(const ArtCnnWgrad *desc, void *stream)
{
    return wgrad3x3(desc, static_cast<cudaStream_t>(stream));
}

int32_t art_cnn_pack_weights(const float *w, int32_t cout, int32_t cin, int32_t transpose, int32_t ci0, int32_t n,
                             int32_t ck, void *out, void *stream)
{
    if (!w || !out || cout < 1 || cin < 1 || n < 16 || n % 16 || (ck != 16 && ck != 32))
        return fail(ART_ERR_INVALID_ARGUMENT, "pack_weights: bad arguments");
    const int K = transpose ? cout : cin;
    if (K % ck) return fail(ART_ERR_INVALID_ARGUMENT, "pack_weights: reduction size must be a multiple of ck");
    const int total = n * 9 * K;
    k_pack<<<blocks_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(w, cout, cin, transpose, ci0, n, ck,
                                                                             static_cast<bf16 *>(out));
    return check_launch("k_pack");
}

int32_t art_cnn_pool2(const void *in, int32_t B, int32_t H, int32_t W, int32_t C, int32_t in_cstride,
                      int32_t in_coff, void *out, void *stream)
{
    if (!in || !out || H % 2 || W % 2 || C % 8 || in_cstride % 8 || in_coff % 8 || in_coff + C > in_cstride)
        return fail(ART_ERR_INVALID_ARGUMENT, "pool2: bad arguments");
    const long long n = (long long)B * (H / 2) * (W / 2) * (C / 8);
    k_pool2<<<blocks_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const bf16 *>(in), B, H, W, C,
                                                                          in_cstride, in_coff, static_cast<bf16 *>(out));
    return check_launch("k_pool2");
}

int32_t art_cnn_upsample2(const void *in, int32_t B, int32_t H, int32_t W, int32_t C, void *out, int32_t out_cstride,
                          int32_t out_coff, void *stream)
{
    if (!in || !out || H % 2 || W % 2 || C % 8 || out_cstride % 8 || out_coff % 8 || out_coff + C > out_cstride)
        return fail(ART_ERR_INVALID_ARGUMENT, "upsample2: bad arguments");
    const long long n = (long long)B * H * W * (C / 8);
    k_upsample2<<<blocks_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const bf16 *>(in), B, H, W, C, static_cast<bf16 *>(out), out_cstride, out_coff);
    return check_launch("k_upsample2");
}

int32_t art_cnn_downsum2_mask(const void *g, int32_t B, int32_t H, int32_t W, int32_t C, const void *act, void *out,
                              void *stream)
{
    if (!g || !act || !out || H % 2 || W % 2 || C % 8) return fail(ART_ERR_INVALID_ARGUMENT, "downsum2_mask: bad arguments");
    const long long n = (long long)B * (H / 2) * (W / 2) * (C / 8);
    k_downsum2_mask<<<blocks_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const bf16 *>(g), B, H, W, C, static_cast<const bf16 *>(act), static_cast<bf16 *>(out));
    return check_launch("k_downsum2_mask");
}

int32_t art_cnn_unpool_add_mask(void *g, const void *gp, int32_t B, int32_t H, int32_t W, int32_t C, const void *act,
                                int32_t act_cstride, int32_t act_coff, void *stream)
{
    if (!g || !act || H % 2 || W % 2 || C % 8 || act_cstride % 8 || act_coff % 8 || act_coff + C > act_cstride)
        return fail(ART_ERR_INVALID_ARGUMENT, "unpool_add_mask: bad arguments");
    const long long n = (long long)B * H * W * (C / 8);
    k_unpool_add_mask<<<blocks_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<bf16 *>(g), static_cast<const bf16 *>(gp), B, H, W, C, static_cast<const bf16 *>(act), act_cstride,
        act_coff);
    return check_launch("k_unpool_add_mask");
}

int32_t art_cnn_bias_grad(const void *g, int64_t npix, int32_t C, float *workspace, int64_t workspace_bytes,
                          float *out, int32_t accumulate, void *stream)
{
    if (!g || !workspace || !out || C < 1 || C > 256) return fail(ART_ERR_INVALID_ARGUMENT, "bias_grad: bad arguments");
    int nblk = (int)std::min<long long>(2 * num_sms(), workspace_bytes / (4LL * C));
    if (nblk < 1) return fail(ART_ERR_INVALID_ARGUMENT, "bias_grad: workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_colsum_partial<<<nblk, 256, 0, s>>>(static_cast<const bf16 *>(g), npix, C, workspace);
    int32_t rc = check_launch("k_colsum_partial");
    if (rc) return rc;
    k_colsum_final<<<1, 256, 0, s>>>(workspace, nblk, C, out, accumulate);
    return check_launch("k_colsum_final");
}

int32_t art_cnn_features(const int16_t *coef, int32_t cpitch, int64_t img_stride, const float *q, int32_t B,
                         int32_t H, int32_t W, float *dec, void *feat, void *stream)
{
    if (!coef || !q || !dec || H % 8 || W % 8 || cpitch < W || cpitch % 8 || img_stride % 8)
        return fail(ART_ERR_INVALID_ARGUMENT, "features: bad arguments");
    if ((reinterpret_cast<uintptr_t>(coef) | reinterpret_cast<uintptr_t>(dec) | reinterpret_cast<uintptr_t>(feat)) & 15)
        return fail(ART_ERR_INVALID_ARGUMENT, "features: coef, dec and feat must be 16-byte aligned");
    // One warp per 4 blocks of a padded block row (ceil(W / 16) * 2 blocks wide).
    const long long warps = (long long)B * ((H + 15) / 16 * 2) * (((W + 15) / 16 * 2 + 3) / 4);
    k_features<<<blocks_for(warps * 32, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        coef, cpitch, img_stride, q, B, H, W, dec, static_cast<bf16 *>(feat));
    return check_launch("k_features");
}

int32_t art_cnn_residual(const float *r, int32_t rstride, const float *dec, const float *target, int32_t B,
                         int32_t H, int32_t W, float *pred, void *grad, float *loss_partial, int32_t loss_blocks,
                         void *stream)
{
    if (!r || !dec || (target && (!grad || !loss_partial)) || loss_blocks < 1 || rstride < 4 || B < 1 || H < 1 ||
        W < 1)
        return fail(ART_ERR_INVALID_ARGUMENT, "residual: bad arguments");
    const long long npix = (long long)B * H * W;
    k_residual<<<loss_blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        r, rstride, dec, target, B, H, W, 1.f / (float)npix, pred, static_cast<bf16 *>(grad), loss_partial);
    return check_launch("k_residual");
}

int32_t art_cnn_wait_selftest(int32_t *err, int64_t limit_cycles, void *stream)
{
    if (!err || limit_cycles < 1 || limit_cycles > 8000000000LL)
        return fail(ART_ERR_INVALID_ARGUMENT, "wait_selftest: bad arguments");
    k_wait_selftest<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(err, (long long)limit_cycles);
    return check_launch("k_wait_selftest");
}

int32_t art_cnn_adam(float *w, const float *g, float *m, float *v, int64_t n, float lr, float beta1, float beta2,
                     float eps, int32_t step, void *stream)
{
    if (!w || !g || !m || !v || n < 0 || step < 1) return fail(ART_ERR_INVALID_ARGUMENT, "adam: bad arguments");
    const float c1 = 1.f / (1.f - std::pow(beta1, (float)step)), c2 = 1.f / (1.f - std::pow(beta2, (float)step));
    k_adam<<<blocks_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(w, g, m, v, n, lr, beta1, beta2, eps, c1, c2);
    return check_launch("k_adam");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The network: a 4-level encoder-decoder, one 3x3 convolution per level and
// direction. Level l has H >> l rows. Encoder activations are written into
// the first channels of the decoder's concatenation buffers (skip | upsampled):
//   e1 = relu(conv(F, 16 -> 32))            -> cat1[0:32]     level 0
//   e2 = relu(conv(pool(e1), 32 -> 64))     -> cat2[0:64]     level 1
//   e3 = relu(conv(pool(e2), 64 -> 96))     -> cat3[0:96]     level 2
//   e4 = relu(conv(pool(e3), 96 -> 128))                      level 3
//   d3 = relu(conv(cat3 = [e3 | up(e4)], 224 -> 96))          level 2
//   d2 = relu(conv(cat2 = [e2 | up(d3)], 160 -> 64))          level 1
//   d1 = relu(conv(cat1 = [e1 | up(d2)], 96 -> 32))           level 0
//   r  = conv(d1, 32 -> 16), channel 0 used; prediction = decoded + 16 r.
namespace art {
namespace cnn {

struct LayerDef {
    int cin, cout, level, relu, skip;  // skip: channels of cin that come from the encoder (decoder layers)
};
constexpr int NLAYER = 8;
constexpr LayerDef LAYERS[NLAYER] = {
    {16, 32, 0, 1, 0},   {32, 64, 1, 1, 0},  {64, 96, 2, 1, 0},  {96, 128, 3, 1, 0},
    {224, 96, 2, 1, 96}, {160, 64, 1, 1, 64}, {96, 32, 0, 1, 32}, {32, 16, 0, 0, 0},
};
enum { E1, E2, E3, E4, D3, D2, D1, HEAD };

inline int ck_for(int k) { return k % 32 == 0 ? 32 : 16; }

long long param_count()
{
    long long n = 0;
    for (const auto &l : LAYERS) n += (long long)l.cout * 9 * l.cin + l.cout;
    return n;
}

struct Buf {
    void *p = nullptr;
    size_t n = 0;
    bool ensure(size_t bytes)
    {
        if (bytes <= n) return true;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            p = nullptr;
            return false;
        }
        n = bytes;
        return true;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    template <class T>
    T *as() const
    {
        return static_cast<T *>(p);
    }
};

}  // namespace cnn
}  // namespace art

namespace art {
namespace cnn {
// One set of forward activations. A network holds two, so that two
// predictions (e.g. the luma and the chroma planes of one image) can run on
// two streams at once; training uses set 0 (its gradients live in ArtNet).
struct NetActs {
    Buf feat, dec, cat1, cat2, cat3, p1, p2, p3, e4, d3, d2, d1, r, pred;
    unsigned long long gen = 0;  // process-wide serial, renewed whenever these buffers are (re)allocated
    long long cap_px = 0;        // level-0 pixels the activation buffers hold
    long long cap_full = 0;      // full-resolution samples the decoded/prediction buffers hold
};
constexpr int NSLOT = 2;
}  // namespace cnn
}  // namespace art

struct ArtNet {
    int device = 0;
    long long nparam = 0;
    int step = 0;
    size_t w_off[art::cnn::NLAYER], b_off[art::cnn::NLAYER];
    art::cnn::Buf params, grads, adam_m, adam_v, errflag, workspace, loss_partial;
    art::cnn::Buf wf[art::cnn::NLAYER];     // forward packs
    art::cnn::Buf wb[art::cnn::NLAYER][2];  // backward-data packs (skip part, upsampled part or whole input)
    bool packed = false;
    art::cnn::NetActs act[art::cnn::NSLOT];  // forward activations
    // gradients (training, with activation set 0)
    art::cnn::Buf dr, gd1, ge1, gup1, gd2, ge2, gup2, gd3, ge3, gup3, ge4, gp3, gp2, gp1;
    float smooth_weight = 0.f;  // lambda of the training loss's smoothness term (art_net_set_loss)
    // Objective term of the training loss (art_net_set_objective): its weight
    // and the objective's term weights; obj holds x, P, the five term planes
    // and the clamp masks.
    float obj_lambda = 0.f, obj_tv = 0.f, obj_tgv = 0.f, obj_p = 0.f;
    float joint_luma_w = 1.f;  // weight of the luma's squared errors in the joint loss (art_net_set_joint_loss)
    art::cnn::Buf obj;
    bool cap_train = false;     // the gradient buffers match act[0]
};

namespace art {
namespace cnn {

constexpr int LOSS_BLOCKS = 296;
constexpr size_t WORKSPACE_BYTES = 64ull << 20;

// Activation set `slot` for px level-0 pixels and full full-resolution
// samples (decoded image, prediction); with train, also the gradient
// buffers (slot 0 only).
int32_t net_alloc(ArtNet *net, int slot, long long px, long long full, bool train)
{
    if (slot < 0 || slot >= NSLOT || (train && slot != 0)) return fail(ART_ERR_INVALID_ARGUMENT, "network: bad activation set");
    NetActs &A = net->act[slot];
    if (px <= A.cap_px && full <= A.cap_full && (!train || net->cap_train)) return ART_OK;
    px = std::max(px, A.cap_px);
    full = std::max(full, A.cap_full);
    train = train || (slot == 0 && net->cap_train);
    const size_t P0 = (size_t)px, P1 = P0 / 4 + 64, P2 = P0 / 16 + 64, P3 = P0 / 64 + 64, PF = (size_t)full;
    struct Req {
        Buf *b;
        size_t bytes;
    };
    std::vector<Req> req = {
        {&A.feat, P0 * 16 * 2}, {&A.dec, PF * 4},       {&A.cat1, P0 * 96 * 2}, {&A.cat2, P1 * 160 * 2},
        {&A.cat3, P2 * 224 * 2}, {&A.p1, P1 * 32 * 2},   {&A.p2, P2 * 64 * 2},   {&A.p3, P3 * 96 * 2},
        {&A.e4, P3 * 128 * 2},  {&A.d3, P2 * 96 * 2},   {&A.d2, P1 * 64 * 2},   {&A.d1, P0 * 32 * 2},
        {&A.r, P0 * JOINT_RSTRIDE * 4}, {&A.pred, PF * 4},
    };
    if (train) {
        std::vector<Req> t = {
            {&net->dr, P0 * 16 * 2},  {&net->gd1, P0 * 32 * 2}, {&net->ge1, P0 * 32 * 2},  {&net->gup1, P0 * 64 * 2},
            {&net->gd2, P1 * 64 * 2}, {&net->ge2, P1 * 64 * 2}, {&net->gup2, P1 * 96 * 2}, {&net->gd3, P2 * 96 * 2},
            {&net->ge3, P2 * 96 * 2}, {&net->gup3, P2 * 128 * 2}, {&net->ge4, P3 * 128 * 2}, {&net->gp3, P3 * 96 * 2},
            {&net->gp2, P2 * 64 * 2}, {&net->gp1, P1 * 32 * 2},
        };
        req.insert(req.end(), t.begin(), t.end());
    }
    // A process-wide serial, not a per-network count: a network created later
    // at the same host address must never match a graph recorded with another
    // network's (freed) buffers.
    static std::atomic<unsigned long long> serial{0};
    A.gen = ++serial;
    for (auto &q : req)
        if (!q.b->ensure(q.bytes)) return fail(ART_ERR_CUDA, "network buffers: cudaMalloc failed");
    A.cap_px = px;
    A.cap_full = full;
    if (slot == 0) net->cap_train = train;
    return ART_OK;
}

int32_t net_pack(ArtNet *net, bool backward, cudaStream_t s)
{
    const float *w = net->params.as<float>();
    for (int i = 0; i < NLAYER; i++) {
        const LayerDef &L = LAYERS[i];
        const size_t fbytes = (size_t)L.cout * 9 * L.cin * 2;
        if (!net->wf[i].ensure(fbytes)) return fail(ART_ERR_CUDA, "weight packs: cudaMalloc failed");
        int32_t rc = art_cnn_pack_weights(w + net->w_off[i], L.cout, L.cin, 0, 0, L.cout, ck_for(L.cin), net->wf[i].p, s);
        if (rc) return rc;
        if (!backward || i == E1) continue;
        // Backward-data packs: decoder layers in two parts (skip, upsampled), others whole.
        const int parts = L.skip ? 2 : 1;
        for (int k = 0; k < parts; k++) {
            const int ci0 = k == 0 ? 0 : L.skip, n = L.skip ? (k == 0 ? L.skip : L.cin - L.skip) : L.cin;
            if (!net->wb[i][k].ensure((size_t)n * 9 * L.cout * 2)) return fail(ART_ERR_CUDA, "weight packs: cudaMalloc failed");
            rc = art_cnn_pack_weights(w + net->w_off[i], L.cout, L.cin, 1, ci0, n, ck_for(L.cout), net->wb[i][k].p, s);
            if (rc) return rc;
        }
    }
    net->packed = true;
    return ART_OK;
}

// Forward convolution of `layer`: bf16 output into channels [coff, coff + cout)
// of `out` (cstride channels; 2H x 2W, each pixel stored to its 2x2 cell,
// when up2), optionally also the fp32 output and the 2x2-pooled output.
int32_t conv(ArtNet *net, int layer, const void *x, int B, int H, int W, void *out, int cstride, int coff,
             float *out_f32, cudaStream_t s, void *pool_out = nullptr, int up2 = 0, int f32_channels = RSTRIDE)
{
    const LayerDef &L = LAYERS[layer];
    ArtCnnConv d{};
    d.B = B;
    d.H = H;
    d.W = W;
    d.cin = L.cin;
    d.ck = ck_for(L.cin);
    d.n = L.cout;
    d.n_store = L.cout;
    d.x = x;
    d.wpack = net->wf[layer].p;
    d.bias = net->params.as<float>() + net->b_off[layer];
    d.out = out;
    d.out_cstride = cstride;
    d.out_coff = coff;
    d.out_f32 = out_f32;
    // The fp32 output is the head's: only its first 4 channels (the 2x2 cell
    // residuals; 12 for the joint 4:2:0 network, three components' cells) are
    // used, stored densely.
    d.f32_cstride = f32_channels;
    d.f32_channels = f32_channels;
    d.relu = L.relu;
    d.err = net->errflag.as<int>();
    d.pool_out = pool_out;
    d.up2 = up2;
    return conv3x3(&d, s);
}

// Backward-data of `layer` (part k) from the gradient g of its
// pre-activation output; writes n channels dense into out.
int32_t dgrad(ArtNet *net, int layer, int k, const void *g, int B, int H, int W, void *out, const void *mask,
              int mask_cstride, cudaStream_t s)
{
    const LayerDef &L = LAYERS[layer];
    const int n = L.skip ? (k == 0 ? L.skip : L.cin - L.skip) : L.cin;
    ArtCnnConv d{};
    d.B = B;
    d.H = H;
    d.W = W;
    d.cin = L.cout;
    d.ck = ck_for(L.cout);
    d.n = n;
    d.n_store = n;
    d.x = g;
    d.wpack = net->wb[layer][k].p;
    d.out = out;
    d.out_cstride = n;
    d.out_coff = 0;
    d.mask = mask;
    d.mask_cstride = mask_cstride;
    d.err = net->errflag.as<int>();
    return conv3x3(&d, s);
}

int32_t wgrad(ArtNet *net, int layer, const void *x, const void *g, int B, int H, int W, cudaStream_t s)
{
    const LayerDef &L = LAYERS[layer];
    ArtCnnWgrad d{};
    d.B = B;
    d.H = H;
    d.W = W;
    d.cout = L.cout;
    d.cin = L.cin;
    d.dy = g;
    d.x = x;
    d.dw = net->grads.as<float>() + net->w_off[layer];
    d.workspace = net->workspace.p;
    d.workspace_bytes = (int64_t)net->workspace.n;
    d.err = net->errflag.as<int>();
    int32_t rc = wgrad3x3(&d, s);
    if (rc) return rc;
    return art_cnn_bias_grad(g, (int64_t)B * H * W, L.cout, net->workspace.as<float>(), (int64_t)net->workspace.n,
                             net->grads.as<float>() + net->b_off[layer], 0, s);
}

#define NET_TRY(x)                \
    do {                          \
        const int32_t rc_ = (x);  \
        if (rc_) return rc_;      \
    } while (0)

// Forward pass on level-0 size H x W. The encoder convolutions also write
// their pooled outputs. For inference the e4/d3/d2 convolutions store their
// outputs upsampled straight into the next concatenation; training keeps
// them whole (the backward pass reads them as ReLU masks) and upsamples after.
int32_t net_forward(ArtNet *net, NetActs &A, int B, int H, int W, cudaStream_t s, bool train, int rch = RSTRIDE)
{
    const int H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
    NET_TRY(conv(net, E1, A.feat.p, B, H, W, A.cat1.p, 96, 0, nullptr, s, A.p1.p));
    NET_TRY(conv(net, E2, A.p1.p, B, H1, W1, A.cat2.p, 160, 0, nullptr, s, A.p2.p));
    NET_TRY(conv(net, E3, A.p2.p, B, H2, W2, A.cat3.p, 224, 0, nullptr, s, A.p3.p));
    if (train) {
        NET_TRY(conv(net, E4, A.p3.p, B, H3, W3, A.e4.p, 128, 0, nullptr, s));
        NET_TRY(art_cnn_upsample2(A.e4.p, B, H2, W2, 128, A.cat3.p, 224, 96, s));
        NET_TRY(conv(net, D3, A.cat3.p, B, H2, W2, A.d3.p, 96, 0, nullptr, s));
        NET_TRY(art_cnn_upsample2(A.d3.p, B, H1, W1, 96, A.cat2.p, 160, 64, s));
        NET_TRY(conv(net, D2, A.cat2.p, B, H1, W1, A.d2.p, 64, 0, nullptr, s));
        NET_TRY(art_cnn_upsample2(A.d2.p, B, H, W, 64, A.cat1.p, 96, 32, s));
    } else {
        NET_TRY(conv(net, E4, A.p3.p, B, H3, W3, A.cat3.p, 224, 96, nullptr, s, nullptr, 1));
        NET_TRY(conv(net, D3, A.cat3.p, B, H2, W2, A.cat2.p, 160, 64, nullptr, s, nullptr, 1));
        NET_TRY(conv(net, D2, A.cat2.p, B, H1, W1, A.cat1.p, 96, 32, nullptr, s, nullptr, 1));
    }
    NET_TRY(conv(net, D1, A.cat1.p, B, H, W, A.d1.p, 32, 0, nullptr, s));
    NET_TRY(conv(net, HEAD, A.d1.p, B, H, W, nullptr, 0, 0, A.r.as<float>(), s, nullptr, 0, rch));
    return ART_OK;
}

int32_t net_backward(ArtNet *net, int B, int H, int W, cudaStream_t s)
{
    NetActs &A = net->act[0];
    const int H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
    // head
    NET_TRY(wgrad(net, HEAD, A.d1.p, net->dr.p, B, H, W, s));
    NET_TRY(dgrad(net, HEAD, 0, net->dr.p, B, H, W, net->gd1.p, A.d1.p, 32, s));
    // d1 (level 0): input cat1 = [e1 | up(d2)]
    NET_TRY(wgrad(net, D1, A.cat1.p, net->gd1.p, B, H, W, s));
    NET_TRY(dgrad(net, D1, 0, net->gd1.p, B, H, W, net->ge1.p, nullptr, 0, s));
    NET_TRY(dgrad(net, D1, 1, net->gd1.p, B, H, W, net->gup1.p, nullptr, 0, s));
    NET_TRY(art_cnn_downsum2_mask(net->gup1.p, B, H, W, 64, A.d2.p, net->gd2.p, s));
    // d2 (level 1): input cat2 = [e2 | up(d3)]
    NET_TRY(wgrad(net, D2, A.cat2.p, net->gd2.p, B, H1, W1, s));
    NET_TRY(dgrad(net, D2, 0, net->gd2.p, B, H1, W1, net->ge2.p, nullptr, 0, s));
    NET_TRY(dgrad(net, D2, 1, net->gd2.p, B, H1, W1, net->gup2.p, nullptr, 0, s));
    NET_TRY(art_cnn_downsum2_mask(net->gup2.p, B, H1, W1, 96, A.d3.p, net->gd3.p, s));
    // d3 (level 2): input cat3 = [e3 | up(e4)]
    NET_TRY(wgrad(net, D3, A.cat3.p, net->gd3.p, B, H2, W2, s));
    NET_TRY(dgrad(net, D3, 0, net->gd3.p, B, H2, W2, net->ge3.p, nullptr, 0, s));
    NET_TRY(dgrad(net, D3, 1, net->gd3.p, B, H2, W2, net->gup3.p, nullptr, 0, s));
    NET_TRY(art_cnn_downsum2_mask(net->gup3.p, B, H2, W2, 128, A.e4.p, net->ge4.p, s));
    // e4 (level 3)
    NET_TRY(wgrad(net, E4, A.p3.p, net->ge4.p, B, H3, W3, s));
    NET_TRY(dgrad(net, E4, 0, net->ge4.p, B, H3, W3, net->gp3.p, nullptr, 0, s));
    NET_TRY(art_cnn_unpool_add_mask(net->ge3.p, net->gp3.p, B, H2, W2, 96, A.cat3.p, 224, 0, s));
    // e3 (level 2)
    NET_TRY(wgrad(net, E3, A.p2.p, net->ge3.p, B, H2, W2, s));
    NET_TRY(dgrad(net, E3, 0, net->ge3.p, B, H2, W2, net->gp2.p, nullptr, 0, s));
    NET_TRY(art_cnn_unpool_add_mask(net->ge2.p, net->gp2.p, B, H1, W1, 64, A.cat2.p, 160, 0, s));
    // e2 (level 1)
    NET_TRY(wgrad(net, E2, A.p1.p, net->ge2.p, B, H1, W1, s));
    NET_TRY(dgrad(net, E2, 0, net->ge2.p, B, H1, W1, net->gp1.p, nullptr, 0, s));
    NET_TRY(art_cnn_unpool_add_mask(net->ge1.p, net->gp1.p, B, H, W, 32, A.cat1.p, 96, 0, s));
    // e1 (level 0)
    NET_TRY(wgrad(net, E1, A.feat.p, net->ge1.p, B, H, W, s));
    return ART_OK;
}

// Side of the network's first (half-resolution) level for a component side n:
// n padded to a multiple of 16, halved, so that three 2x2 poolings divide it.
int level0(int n) { return (n + 15) / 16 * 8; }

int32_t check_geometry(int B, int H, int W)
{
    if (B < 1 || H < 8 || W < 8 || H % 8 || W % 8)
        return fail(ART_ERR_INVALID_ARGUMENT, "network input must be at least 8x8 and a multiple of 8 on each side");
    if ((long long)B * H * W > (1LL << 28)) return fail(ART_ERR_INVALID_ARGUMENT, "network input too large");
    return ART_OK;
}

int32_t read_err(ArtNet *net, cudaStream_t s)
{
    int h = 0;
    if (cudaMemcpyAsync(&h, net->errflag.p, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return fail(ART_ERR_CUDA, std::string("network: ") + cudaGetErrorString(cudaGetLastError()));
    if (h) return fail(ART_ERR_CUDA, "network: a tensor-core pipeline wait timed out");
    return ART_OK;
}

// Features + forward for B coefficient images; prediction into pred (or the
// net's own buffer when pred is null).
int32_t net_predict(ArtNet *net, int slot, const int16_t *coef, int cpitch, long long img_stride, const float *q, int B,
                    int H, int W, float *pred, cudaStream_t s)
{
    NET_TRY(check_geometry(B, H, W));
    const int H0 = level0(H), W0 = level0(W);
    NET_TRY(net_alloc(net, slot, (long long)B * H0 * W0, (long long)B * H * W, false));
    if (!net->packed) NET_TRY(net_pack(net, false, s));
    NetActs &A = net->act[slot];
    NET_TRY(art_cnn_features(coef, cpitch, img_stride, q, B, H, W, A.dec.as<float>(), A.feat.p, s));
    NET_TRY(net_forward(net, A, B, H0, W0, s, false));
    return art_cnn_residual(A.r.as<float>(), RSTRIDE, A.dec.as<float>(), nullptr, B, H, W,
                            pred ? pred : A.pred.as<float>(), nullptr, nullptr, 8 * num_sms(), s);
}

int32_t net_predict_async(ArtNet *net, int slot, const int16_t *coef, int cpitch, long long img_stride, const float *q,
                          int B, int H, int W, float *pred, void *stream)
{
    return net_predict(net, slot, coef, cpitch, img_stride, q, B, H, W, pred, static_cast<cudaStream_t>(stream));
}

int32_t net_prepare(ArtNet *net, int slot, int B, int H, int W, void *stream)
{
    NET_TRY(check_geometry(B, H, W));
    NET_TRY(net_alloc(net, slot, (long long)B * level0(H) * level0(W), (long long)B * H * W, false));
    if (!net->packed) NET_TRY(net_pack(net, false, static_cast<cudaStream_t>(stream)));
    return ART_OK;
}

// Joint 4:2:0 geometry: H x W luma (multiples of 16), chroma H/2 x W/2.
int32_t check_joint_geometry(int B, int H, int W)
{
    if (B < 1 || H < 16 || W < 16 || H % 16 || W % 16)
        return fail(ART_ERR_INVALID_ARGUMENT, "joint network input must be at least 16x16 and a multiple of 16 on each side");
    if ((long long)B * H * W * 4 > (1LL << 28)) return fail(ART_ERR_INVALID_ARGUMENT, "network input too large");
    return ART_OK;
}

// Level-0 pixels and full-resolution floats (bases [3][B][H][W] plus the
// decoded chroma at component resolution) of a joint pass.
inline long long joint_px(int B, int H, int W) { return (long long)B * (H / 2) * (W / 2); }
inline long long joint_full(int B, int H, int W) { return 4LL * B * H * W; }

// Features of B joint 4:2:0 images into A.feat and the bases into A.dec
// ([3][B][H][W], then the decoded chroma [B][2][H/2][W/2]).
int32_t joint_features(NetActs &A, const int16_t *cy, int py, long long sy, const int16_t *cc, int pc, long long sc,
                       const float *qy, const float *qc, int B, int H, int W, cudaStream_t s)
{
    float *dec = A.dec.as<float>();
    float *decC = dec + 3 * (size_t)B * H * W;
    NET_TRY(art_cnn_features(cy, py, sy, qy, B, H, W, dec, A.feat.p, s));
    NET_TRY(art_cnn_features(cc, pc, sc, qc, 2 * B, H / 2, W / 2, decC, nullptr, s));
    k_features_joint<<<blocks_for(joint_px(B, H, W), 256), 256, 0, s>>>(decC, qc, B, H, W, dec,
                                                                        static_cast<bf16 *>(A.feat.p));
    return check_launch("k_features_joint");
}

// Prediction of B joint images: sample (c, b, Y, X) to pred[c ocs + (b H + Y)
// opitch + X] and, when pred2 is given, to the same place of pred2.
int32_t net_predict_joint(ArtNet *net, int slot, const int16_t *cy, int py, long long sy, const int16_t *cc, int pc,
                          long long sc, const float *qy, const float *qc, int B, int H, int W, float *pred,
                          float *pred2, long long ocs, int opitch, cudaStream_t s)
{
    NET_TRY(check_joint_geometry(B, H, W));
    NET_TRY(net_alloc(net, slot, joint_px(B, H, W), joint_full(B, H, W), false));
    if (!net->packed) NET_TRY(net_pack(net, false, s));
    NetActs &A = net->act[slot];
    NET_TRY(joint_features(A, cy, py, sy, cc, pc, sc, qy, qc, B, H, W, s));
    NET_TRY(net_forward(net, A, B, H / 2, W / 2, s, false, JOINT_RSTRIDE));
    k_residual_joint<<<8 * num_sms(), 256, 0, s>>>(A.r.as<float>(), JOINT_RSTRIDE, A.dec.as<float>(), nullptr, B, H,
                                                  W, 0.f, 1.f, pred, pred2, ocs, opitch, nullptr, nullptr);
    return check_launch("k_residual_joint");
}

int32_t net_predict_joint_async(ArtNet *net, int slot, const int16_t *cy, int py, long long sy, const int16_t *cc,
                                int pc, long long sc, const float *qy, const float *qc, int H, int W, float *x,
                                float *y, long long cstride, int pitch, void *stream)
{
    return net_predict_joint(net, slot, cy, py, sy, cc, pc, sc, qy, qc, 1, H, W, x, y, cstride, pitch,
                             static_cast<cudaStream_t>(stream));
}

int32_t net_prepare_joint(ArtNet *net, int slot, int H, int W, void *stream)
{
    NET_TRY(check_joint_geometry(1, H, W));
    NET_TRY(net_alloc(net, slot, joint_px(1, H, W), joint_full(1, H, W), false));
    if (!net->packed) NET_TRY(net_pack(net, false, static_cast<cudaStream_t>(stream)));
    return ART_OK;
}

unsigned long long net_generation(const ArtNet *net, int slot) { return net->act[slot].gen; }

int net_device(const ArtNet *net) { return net->device; }

int32_t net_error(ArtNet *net)
{
    int h = 0;
    if (cudaMemcpy(&h, net->errflag.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(ART_ERR_CUDA, std::string("network: ") + cudaGetErrorString(cudaGetLastError()));
    if (h) return fail(ART_ERR_CUDA, "network: a tensor-core pipeline wait timed out");
    return ART_OK;
}

}  // namespace cnn
}  // namespace art

extern "C" {

int64_t art_net_num_params(void) { return art::cnn::param_count(); }

int32_t art_net_create(int32_t device, const float *params, int64_t nparams, ArtNet **out)
{
    using namespace art::cnn;
    if (!out || !params) return fail(ART_ERR_INVALID_ARGUMENT, "net_create: null pointer");
    *out = nullptr;
    if (nparams != param_count()) return fail(ART_ERR_INVALID_ARGUMENT, "net_create: wrong parameter count");
    for (int64_t i = 0; i < nparams; i++)
        if (!std::isfinite(params[i])) return fail(ART_ERR_INVALID_DATA, "net_create: non-finite parameter");
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(ART_ERR_CUDA, "net_create: no device");
    if (cudaSetDevice(device) != cudaSuccess) return fail(ART_ERR_CUDA, "net_create: cudaSetDevice failed");
    ArtNet *net = new ArtNet();
    net->device = device;
    net->nparam = nparams;
    size_t off = 0;
    for (int i = 0; i < NLAYER; i++) {
        net->w_off[i] = off;
        off += (size_t)LAYERS[i].cout * 9 * LAYERS[i].cin;
        net->b_off[i] = off;
        off += LAYERS[i].cout;
    }
    const size_t pb = (size_t)nparams * 4;
    if (!net->params.ensure(pb) || !net->errflag.ensure(64) || !net->workspace.ensure(WORKSPACE_BYTES) ||
        !net->loss_partial.ensure(3 * LOSS_BLOCKS * 4) ||
        cudaMemcpy(net->params.p, params, pb, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(net->errflag.p, 0, 64) != cudaSuccess) {
        art_net_destroy(net);
        return fail(ART_ERR_CUDA, "net_create: device allocation failed");
    }
    *out = net;
    return ART_OK;
}

void art_net_destroy(ArtNet *net)
{
    if (!net) return;
    cudaSetDevice(net->device);
    art::cnn::Buf *all[] = {&net->params, &net->grads, &net->adam_m, &net->adam_v, &net->errflag, &net->workspace,
                            &net->loss_partial, &net->dr, &net->gd1, &net->ge1, &net->gup1, &net->gd2, &net->ge2,
                            &net->gup2, &net->gd3, &net->ge3, &net->gup3, &net->ge4, &net->gp3, &net->gp2, &net->gp1,
                            &net->obj};
    for (auto *b : all) b->release();
    for (auto &A : net->act) {
        art::cnn::Buf *acts[] = {&A.feat, &A.dec, &A.cat1, &A.cat2, &A.cat3, &A.p1, &A.p2,
                                 &A.p3,   &A.e4,  &A.d3,   &A.d2,   &A.d1,   &A.r,  &A.pred};
        for (auto *b : acts) b->release();
    }
    for (int i = 0; i < art::cnn::NLAYER; i++) {
        net->wf[i].release();
        net->wb[i][0].release();
        net->wb[i][1].release();
    }
    delete net;
}

int32_t art_net_params(ArtNet *net, float *host, int64_t n)
{
    if (!net || !host || n != net->nparam) return fail(ART_ERR_INVALID_ARGUMENT, "net_params: bad arguments");
    cudaSetDevice(net->device);
    if (cudaMemcpy(host, net->params.p, (size_t)n * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(ART_ERR_CUDA, "net_params: copy failed");
    return ART_OK;
}

int32_t art_net_gradients(ArtNet *net, float *host, int64_t n)
{
    if (!net || !host || n != net->nparam || !net->grads.p)
        return fail(ART_ERR_INVALID_ARGUMENT, "net_gradients: no gradients yet");
    cudaSetDevice(net->device);
    if (cudaMemcpy(host, net->grads.p, (size_t)n * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(ART_ERR_CUDA, "net_gradients: copy failed");
    return ART_OK;
}

int32_t art_net_predict(ArtNet *net, const int16_t *coef, int32_t cpitch, int64_t img_stride, const float *q,
                        int32_t B, int32_t H, int32_t W, float *pred, void *stream)
{
    using namespace art::cnn;
    if (!net || !coef || !q || !pred) return fail(ART_ERR_INVALID_ARGUMENT, "net_predict: null pointer");
    cudaSetDevice(net->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    NET_TRY(net_predict(net, 0, coef, cpitch, img_stride, q, B, H, W, pred, s));
    return read_err(net, s);
}

int32_t art_net_predict_joint(ArtNet *net, const int16_t *coef_y, int32_t cpitch_y, int64_t stride_y,
                              const int16_t *coef_c, int32_t cpitch_c, int64_t stride_c, const float *q_y,
                              const float *q_c, int32_t B, int32_t H, int32_t W, float *pred, void *stream)
{
    using namespace art::cnn;
    if (!net || !coef_y || !coef_c || !q_y || !q_c || !pred)
        return fail(ART_ERR_INVALID_ARGUMENT, "net_predict_joint: null pointer");
    cudaSetDevice(net->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    NET_TRY(net_predict_joint(net, 0, coef_y, cpitch_y, stride_y, coef_c, cpitch_c, stride_c, q_y, q_c, B, H, W, pred,
                              nullptr, (long long)B * H * W, W, s));
    return read_err(net, s);
}

int32_t art_net_train_step_joint(ArtNet *net, const int16_t *coef_y, int32_t cpitch_y, int64_t stride_y,
                                 const int16_t *coef_c, int32_t cpitch_c, int64_t stride_c, const float *q_y,
                                 const float *q_c, const float *target, int32_t B, int32_t H, int32_t W, float lr,
                                 float *loss, void *stream)
{
    using namespace art::cnn;
    if (!net || !coef_y || !coef_c || !q_y || !q_c || !target)
        return fail(ART_ERR_INVALID_ARGUMENT, "net_train_step_joint: null pointer");
    cudaSetDevice(net->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    NET_TRY(check_joint_geometry(B, H, W));
    const int H0 = H / 2, W0 = W / 2;
    NET_TRY(net_alloc(net, 0, joint_px(B, H, W), joint_full(B, H, W), true));
    NetActs &A = net->act[0];
    const size_t pb = (size_t)net->nparam * 4;
    if (!net->grads.p) {
        if (!net->grads.ensure(pb) || !net->adam_m.ensure(pb) || !net->adam_v.ensure(pb) ||
            cudaMemsetAsync(net->adam_m.p, 0, pb, s) != cudaSuccess || cudaMemsetAsync(net->adam_v.p, 0, pb, s) != cudaSuccess)
            return fail(ART_ERR_CUDA, "net_train_step_joint: allocation failed");
    }
    NET_TRY(net_pack(net, true, s));
    NET_TRY(joint_features(A, coef_y, cpitch_y, stride_y, coef_c, cpitch_c, stride_c, q_y, q_c, B, H, W, s));
    NET_TRY(net_forward(net, A, B, H0, W0, s, true, JOINT_RSTRIDE));
    const long long n = 3LL * B * H * W;
    k_residual_joint<<<LOSS_BLOCKS, 256, 0, s>>>(A.r.as<float>(), JOINT_RSTRIDE, A.dec.as<float>(), target, B, H, W,
                                                 1.f / (float)n, net->joint_luma_w, A.pred.as<float>(), nullptr,
                                                 (long long)B * H * W, W,
                                                 static_cast<bf16 *>(net->dr.p), net->loss_partial.as<float>());
    NET_TRY(check_launch("k_residual_joint"));
    NET_TRY(net_backward(net, B, H0, W0, s));
    if (lr > 0.f) {
        net->step++;
        NET_TRY(art_cnn_adam(net->params.as<float>(), net->grads.as<float>(), net->adam_m.as<float>(),
                             net->adam_v.as<float>(), net->nparam, lr, 0.9f, 0.999f, 1e-8f, net->step, s));
        net->packed = false;
    }
    if (loss) {
        float h[LOSS_BLOCKS];
        if (cudaMemcpyAsync(h, net->loss_partial.p, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return fail(ART_ERR_CUDA, "net_train_step_joint: loss copy failed");
        NET_TRY(read_err(net, s));
        double t = 0;
        for (float v : h) t += v;
        *loss = (float)(t / (double)n);
        return ART_OK;
    }
    return read_err(net, s);
}

int32_t art_net_set_joint_loss(ArtNet *net, float luma_weight)
{
    if (!net || !(luma_weight > 0.f) || !std::isfinite(luma_weight))
        return fail(ART_ERR_INVALID_ARGUMENT, "net_set_joint_loss: the luma weight must be finite and > 0");
    net->joint_luma_w = luma_weight;
    return ART_OK;
}

int32_t art_net_set_loss(ArtNet *net, float smooth_weight)
{
    if (!net || !(smooth_weight >= 0.f) || !std::isfinite(smooth_weight))
        return fail(ART_ERR_INVALID_ARGUMENT, "net_set_loss: weight must be finite and >= 0");
    net->smooth_weight = smooth_weight;
    return ART_OK;
}

int32_t art_net_set_objective(ArtNet *net, float lambda, float weight, float pweight, int32_t nch)
{
    if (!net || !(lambda >= 0.f) || !std::isfinite(lambda) || !(weight >= 0.f) || !std::isfinite(weight) ||
        !(pweight >= 0.f) || !std::isfinite(pweight) || nch < 1 || nch > 3)
        return fail(ART_ERR_INVALID_ARGUMENT, "net_set_objective: weights must be finite and >= 0, nch 1..3");
    // The solver's term weights for an nch-channel image (compute_step.rs:8-72).
    const double r = 1.0 / std::sqrt((double)nch);
    net->obj_lambda = lambda;
    net->obj_tv = (float)r;
    net->obj_tgv = (float)(weight * r);
    net->obj_p = (float)(pweight * 2.0 * 255.0 * std::sqrt(2.0));
    return ART_OK;
}

int32_t art_net_train_step(ArtNet *net, const int16_t *coef, int32_t cpitch, int64_t img_stride, const float *q,
                           const float *target, int32_t B, int32_t H, int32_t W, float lr, float *loss, void *stream)
{
    using namespace art::cnn;
    if (!net || !coef || !q || !target) return fail(ART_ERR_INVALID_ARGUMENT, "net_train_step: null pointer");
    cudaSetDevice(net->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    NET_TRY(check_geometry(B, H, W));
    const int H0 = level0(H), W0 = level0(W);
    NET_TRY(net_alloc(net, 0, (long long)B * H0 * W0, (long long)B * H * W, true));
    NetActs &A = net->act[0];
    const size_t pb = (size_t)net->nparam * 4;
    if (!net->grads.p) {
        if (!net->grads.ensure(pb) || !net->adam_m.ensure(pb) || !net->adam_v.ensure(pb) ||
            cudaMemsetAsync(net->adam_m.p, 0, pb, s) != cudaSuccess || cudaMemsetAsync(net->adam_v.p, 0, pb, s) != cudaSuccess)
            return fail(ART_ERR_CUDA, "net_train_step: allocation failed");
    }
    NET_TRY(net_pack(net, true, s));
    NET_TRY(art_cnn_features(coef, cpitch, img_stride, q, B, H, W, A.dec.as<float>(), A.feat.p, s));
    NET_TRY(net_forward(net, A, B, H0, W0, s, true));
    const long long npix = (long long)B * H * W;
    NET_TRY(art_cnn_residual(A.r.as<float>(), RSTRIDE, A.dec.as<float>(), target, B, H, W, A.pred.as<float>(),
                             net->dr.p, net->loss_partial.as<float>(), LOSS_BLOCKS, s));
    const bool objective = net->obj_lambda > 0.f;
    if (objective) {
        const size_t n = (size_t)npix, nblk = n / 64;
        if (!net->obj.ensure(n * 7 * 4 + nblk * 8)) return fail(ART_ERR_CUDA, "net_train_step: allocation failed");
        float *x = net->obj.as<float>(), *P = x + n, *T = P + n;
        auto *mask = reinterpret_cast<unsigned long long *>(T + 5 * n);
        float *lp = net->loss_partial.as<float>();
        k_obj_project<<<LOSS_BLOCKS, 256, 0, s>>>(A.pred.as<float>(), coef, cpitch, img_stride, q, B, H, W,
                                                  net->obj_p, x, P, mask, lp + LOSS_BLOCKS);
        NET_TRY(check_launch("k_obj_project"));
        k_obj_terms<<<LOSS_BLOCKS, 256, 0, s>>>(x, B, H, W, net->obj_tv, net->obj_tgv, T, lp + 2 * LOSS_BLOCKS);
        NET_TRY(check_launch("k_obj_terms"));
        k_obj_back<<<LOSS_BLOCKS, 256, 0, s>>>(T, P, mask, A.pred.as<float>(), target, B, H, W, net->obj_lambda,
                                               1.f / (float)npix, static_cast<bf16 *>(net->dr.p));
        NET_TRY(check_launch("k_obj_back"));
    } else if (net->smooth_weight > 0.f) {
        k_residual_smooth_grad<<<LOSS_BLOCKS, 256, 0, s>>>(A.pred.as<float>(), target, B, H, W, net->smooth_weight,
                                                           1.f / (float)npix, static_cast<bf16 *>(net->dr.p),
                                                           net->loss_partial.as<float>() + LOSS_BLOCKS);
        NET_TRY(check_launch("k_residual_smooth_grad"));
    }
    NET_TRY(net_backward(net, B, H0, W0, s));
    if (lr > 0.f) {
        net->step++;
        NET_TRY(art_cnn_adam(net->params.as<float>(), net->grads.as<float>(), net->adam_m.as<float>(),
                             net->adam_v.as<float>(), net->nparam, lr, 0.9f, 0.999f, 1e-8f, net->step, s));
        net->packed = false;
    }
    if (loss) {
        float h[3 * LOSS_BLOCKS];
        const int nparts = objective ? 3 * LOSS_BLOCKS : net->smooth_weight > 0.f ? 2 * LOSS_BLOCKS : LOSS_BLOCKS;
        if (cudaMemcpyAsync(h, net->loss_partial.p, nparts * sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return fail(ART_ERR_CUDA, "net_train_step: loss copy failed");
        NET_TRY(read_err(net, s));
        double t = 0;
        for (int i = 0; i < nparts; i++) t += (objective && i >= LOSS_BLOCKS ? (double)net->obj_lambda : 1.0) * h[i];
        *loss = (float)(t / (double)npix);
        return ART_OK;
    }
    return read_err(net, s);
}

}  // extern "C"
