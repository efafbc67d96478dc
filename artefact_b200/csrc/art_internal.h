// Internal declarations shared by the host-side translation units.
#pragma once

#include <cstdint>
#include <memory>
#include <new>
#include <string>
#include <utility>
#include <vector>

struct ArtNet;

namespace art {

// Allocator whose value-less construct leaves elements uninitialised, so
// resize() of a coefficient plane that every block decode fills anyway does
// not write the whole plane first.
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U> &) noexcept
    {
    }
    template <class U>
    void construct(U *p) noexcept
    {
        ::new (static_cast<void *>(p)) U;
    }
    template <class U, class... A>
    void construct(U *p, A &&...a)
    {
        ::new (static_cast<void *>(p)) U(std::forward<A>(a)...);
    }
};
using CoefVec = std::vector<int16_t, NoInitAlloc<int16_t>>;

struct JpegChannel {
    uint32_t rounded_px_w = 0, rounded_px_h = 0, block_w = 0, block_h = 0;
    uint32_t samp_h = 1, samp_v = 1;
    float quant[64];
    CoefVec coefs;  // block raster, natural order inside a block
};

struct JpegImage {
    uint32_t real_w = 0, real_h = 0;
    std::vector<JpegChannel> channels;
};

bool decode_jpeg(const uint8_t *data, size_t len, JpegImage &out, std::string &err);

// Thread-local error message for art_last_error().
void set_error(const std::string &msg);

namespace cnn {
// Warm-start prediction for the solver: features + forward + residual of B
// coefficient images into pred (dense [B][H][W] floats), queued on `stream`
// (a cudaStream_t) without waiting for it. `slot` (0 or 1) picks one of the
// network's two activation sets: predictions on different sets may run on
// two streams at once.
int32_t net_predict_async(ArtNet *net, int slot, const int16_t *coef, int cpitch, long long img_stride, const float *q,
                          int B, int H, int W, float *pred, void *stream);
// Joint 4:2:0 prediction of one image (art_net_predict_joint with B = 1):
// luma H x W, chroma H/2 x W/2 (Cb at cc, Cr sc elements after it), tables
// qy[64] and qc[2][64]; full-resolution sample (c, Y, X) written to
// x[c cstride + Y pitch + X] and to the same place of y (the solver's two
// state buffers). Queued on `stream` on activation set `slot`, as
// net_predict_async.
int32_t net_predict_joint_async(ArtNet *net, int slot, const int16_t *cy, int py, long long sy, const int16_t *cc,
                                int pc, long long sc, const float *qy, const float *qc, int H, int W, float *x,
                                float *y, long long cstride, int pitch, void *stream);
// What net_predict_joint_async of one H x W image would allocate and pack.
int32_t net_prepare_joint(ArtNet *net, int slot, int H, int W, void *stream);
// Allocation and weight packing that a prediction of B x H x W on activation
// set `slot` would do, done now (so that a later net_predict_async only
// launches kernels and can be captured into a CUDA graph).
int32_t net_prepare(ArtNet *net, int slot, int B, int H, int W, void *stream);
// Process-wide serial of activation set `slot`: renewed whenever its buffers
// are (re)allocated, never shared by two networks (a graph holding their
// addresses is stale once it changes).
unsigned long long net_generation(const ArtNet *net, int slot);
int net_device(const ArtNet *net);
// Reads the network's device error flag (synchronous): ART_OK, or an error if
// one of its bounded tensor-core waits gave up.
int32_t net_error(ArtNet *net);
}  // namespace cnn

}  // namespace art
