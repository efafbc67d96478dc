// C ABI of the host-side pieces: the JPEG coefficient front end.
#include <cstring>
#include <new>
#include <string>

#include "../../include/artefact_b200.h"
#include "art_internal.h"

struct ArtJpeg {
    art::JpegImage img;
};

extern "C" {

int32_t art_jpeg_decode(const uint8_t *data, size_t len, ArtJpeg **out)
{
    if (!out) {
        art::set_error("null output pointer");
        return ART_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (!data && len) {
        art::set_error("null input buffer");
        return ART_ERR_INVALID_ARGUMENT;
    }
    ArtJpeg *j = new (std::nothrow) ArtJpeg();
    if (!j) {
        art::set_error("out of host memory");
        return ART_ERR_INVALID_ARGUMENT;
    }
    std::string err;
    if (!art::decode_jpeg(data, len, j->img, err)) {
        delete j;
        art::set_error("Failed to decode JPEG: " + err);
        return err.find("not supported") != std::string::npos || err.find("Unsupported") != std::string::npos
                   ? ART_ERR_UNSUPPORTED
                   : ART_ERR_DECODE;
    }
    *out = j;
    return ART_OK;
}

void art_jpeg_free(ArtJpeg *jpeg) { delete jpeg; }

int32_t art_jpeg_info(const ArtJpeg *jpeg, uint32_t *nchannel, uint32_t *real_px_w, uint32_t *real_px_h)
{
    if (!jpeg) {
        art::set_error("null jpeg handle");
        return ART_ERR_INVALID_ARGUMENT;
    }
    if (nchannel) *nchannel = (uint32_t)jpeg->img.channels.size();
    if (real_px_w) *real_px_w = jpeg->img.real_w;
    if (real_px_h) *real_px_h = jpeg->img.real_h;
    return ART_OK;
}

int32_t art_jpeg_channel(const ArtJpeg *jpeg, uint32_t c, ArtChannel *out)
{
    if (!jpeg || !out || c >= jpeg->img.channels.size()) {
        art::set_error("bad jpeg handle, channel index or output pointer");
        return ART_ERR_INVALID_ARGUMENT;
    }
    const art::JpegChannel &jc = jpeg->img.channels[c];
    memset(out, 0, sizeof(*out));
    out->rounded_px_w = jc.rounded_px_w;
    out->rounded_px_h = jc.rounded_px_h;
    out->block_w = jc.block_w;
    out->block_h = jc.block_h;
    out->samp_h = jc.samp_h;
    out->samp_v = jc.samp_v;
    out->coef_type = ART_COEF_I16;
    out->dct_coefs = jc.coefs.data();
    out->quant_table = jc.quant;
    return ART_OK;
}

}  // extern "C"
