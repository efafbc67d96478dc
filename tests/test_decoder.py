"""Host JPEG coefficient decoder (CPU only): check (a), bit-exact coefficients
and quantisation tables, plus the reference decoder's error cases."""
import io
import json
from pathlib import Path

import numpy as np
import pytest

import jpeg_encoder as E
import oracle_lib as O
from artefact_b200 import synth
from artefact_b200.api import ArtefactError, Jpeg, JpegSource

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("case", json.loads((GOLDEN / "decoder_malformed.json").read_text()),
                         ids=lambda c: c["name"])
def test_malformed_streams_are_rejected(case):
    """backend/zune-jpeg/tests/invalid_images.rs:12-66."""
    with pytest.raises(ArtefactError) as ei:
        Jpeg.from_source(JpegSource.Buffer(bytes(case["bytes"])))
    if case["message"]:
        assert case["message"] in str(ei.value)


@pytest.mark.parametrize("name", ["gray_37x21", "420_100x70_rst3", "422_50x30", "444_24x40_rst5"])
def test_golden_roundtrip_bit_exact(name):
    j = Jpeg.from_source(JpegSource.File(str(GOLDEN / f"roundtrip_{name}.jpg")))
    ref = np.load(GOLDEN / f"roundtrip_{name}.npz")
    assert j.nchannel == len([k for k in ref.files if k.startswith("coefs")])
    for i, c in enumerate(j.coefs):
        bw, bh, sh, sv = ref[f"meta{i}"].tolist()
        assert (c.block_w, c.block_h, c.horizontal_samp_factor, c.vertical_samp_factor) == (bw, bh, sh, sv)
        assert (c.rounded_px_w, c.rounded_px_h) == (bw * 8, bh * 8)
        assert c.dct_coefs.dtype == np.int16
        assert np.array_equal(c.dct_coefs.reshape(-1, 64), ref[f"coefs{i}"])
        assert np.array_equal(c.quant_table, ref[f"qt{i}"])


@pytest.mark.parametrize("seed", range(6))
def test_random_roundtrip_bit_exact(seed):
    rng = np.random.default_rng(100 + seed)
    samplings = [[(1, 1)], [(2, 2), (1, 1), (1, 1)], [(2, 1), (1, 1), (1, 1)], [(1, 1)] * 3]
    samp = samplings[seed % len(samplings)]
    w, h = int(rng.integers(1, 90)), int(rng.integers(1, 90))
    comps, expect, (rw, rh) = E.random_image(rng, w, h, samp, qt_max=255 if seed % 2 else 1000)
    data = E.encode(w, h, comps, restart_interval=int(rng.integers(0, 4)))
    j = Jpeg.from_source(JpegSource.Buffer(data))
    assert (j.real_px_w, j.real_px_h) == (w, h)
    assert j.max_rounded()[:2] == (rw, rh)
    for c, (coefs, qt, bw, bh, sh, sv) in zip(j.coefs, expect):
        assert (c.block_w, c.block_h, c.horizontal_samp_factor, c.vertical_samp_factor) == (bw, bh, sh, sv)
        assert np.array_equal(c.dct_coefs.reshape(-1, 64), coefs)
        assert np.array_equal(c.quant_table, qt)


@pytest.mark.parametrize("seed,w,h,samp,restart", [
    (0, 33, 17, [(2, 2), (1, 1), (1, 1)], 0),   # luma: an uncoded block column and row
    (1, 41, 23, [(2, 2), (1, 1), (1, 1)], 3),   # luma: an uncoded block row
    (2, 17, 11, [(2, 1), (1, 1), (1, 1)], 0),   # 4:2:2 luma: an uncoded block column
    (3, 27, 30, [(1, 1), (1, 1), (1, 1)], 2),   # 4:4:4: every block coded
    (4, 97, 9, [(2, 2), (1, 1), (1, 1)], 5),    # luma: an uncoded block column
])
def test_separate_component_scans(seed, w, h, samp, restart):
    """A sequential stream with one non-interleaved scan per component: each
    scan codes only the blocks covering its component's samples (T.81 A.2.2),
    and the blocks of the rounded plane past them decode as zeros."""
    rng = np.random.default_rng(900 + seed)
    comps, expect, _ = E.random_image(rng, w, h, samp)
    hmax, vmax = max(c.h for c in comps), max(c.v for c in comps)
    for c, (coefs, _, bw, bh, _, _) in zip(comps, expect):
        coded_w, coded_h = -(-(-(-w * c.h // hmax)) // 8), -(-(-(-h * c.v // vmax)) // 8)
        for grid in (c.coefs.reshape(bh, bw, 64), coefs.reshape(bh, bw, 64)):
            grid[:, coded_w:] = 0
            grid[coded_h:, :] = 0
    data = E.encode(w, h, comps, restart_interval=restart, separate_scans=True)
    assert data.count(b"\xff\xda") == len(comps)
    j = Jpeg.from_source(JpegSource.Buffer(data))
    for c, (coefs, qt, bw, bh, sh, sv) in zip(j.coefs, expect):
        assert (c.block_w, c.block_h, c.horizontal_samp_factor, c.vertical_samp_factor) == (bw, bh, sh, sv)
        assert np.array_equal(c.dct_coefs.reshape(-1, 64), coefs)
        assert np.array_equal(c.quant_table, qt)


def test_component_without_a_scan_is_zero():
    """A stream whose last component has no scan: that component's plane
    decodes as zeros, the others as coded."""
    rng = np.random.default_rng(77)
    comps, expect, _ = E.random_image(rng, 48, 32, [(2, 2), (1, 1), (1, 1)])  # every block coded
    data = E.encode(48, 32, comps, separate_scans=True, omit_scans=(2,))
    j = Jpeg.from_source(JpegSource.Buffer(data))
    assert np.array_equal(j.coefs[0].dct_coefs.reshape(-1, 64), expect[0][0])
    assert np.array_equal(j.coefs[1].dct_coefs.reshape(-1, 64), expect[1][0])
    assert not np.any(j.coefs[2].dct_coefs)


def _pixels(c):
    blocks = c.dct_coefs.reshape(-1, 64).astype(np.float64) * c.quant_table[None, :]
    img = np.zeros((c.rounded_px_h, c.rounded_px_w))
    for i, b in enumerate(blocks):
        by, bx = divmod(i, c.block_w)
        img[by * 8:by * 8 + 8, bx * 8:bx * 8 + 8] = O.idct8x8(b.reshape(8, 8), fp64=True)
    return np.clip(img + 128, 0, 255)


@pytest.mark.parametrize("w,h,sub,gray", [(64, 48, "4:4:4", True), (100, 70, "4:2:0", False),
                                          (96, 64, "4:4:4", False), (33, 17, "4:2:0", False)])
def test_pillow_pixels_agree(w, h, sub, gray):
    """Dequantised IDCT of the decoded coefficients equals libjpeg's decode to rounding."""
    from PIL import Image

    data = synth.make_jpeg(w, h, 75, sub, gray, seed=3)
    j = Jpeg.from_source(JpegSource.Buffer(data))
    im = Image.open(io.BytesIO(data))
    if not gray:
        im.draft("YCbCr", im.size)
    ref = np.asarray(im).astype(np.float64)
    if gray:
        ref = ref[..., None]
    for ci, c in enumerate(j.coefs):
        if c.horizontal_samp_factor != 1 or c.vertical_samp_factor != 1:
            continue  # libjpeg upsamples chroma with its own filter
        assert np.abs(_pixels(c)[:h, :w] - ref[..., ci]).max() <= 1.0


def test_rounded_sizes_follow_max_sampling():
    data = synth.make_jpeg(1920, 1080, 75, "4:2:0", False, seed=1)
    j = Jpeg.from_source(JpegSource.Buffer(data))
    assert [(c.rounded_px_w, c.rounded_px_h, c.horizontal_samp_factor) for c in j.coefs] == [
        (1920, 1088, 1), (960, 544, 2), (960, 544, 2)]


def _pillow(img, quality, subsampling, progressive, optimize=False, **kw):
    from PIL import Image

    buf = io.BytesIO()
    opts = dict(format="JPEG", quality=quality, optimize=optimize, progressive=progressive, **kw)
    if img.ndim == 3:
        opts["subsampling"] = subsampling
    Image.fromarray(img).save(buf, **opts)
    return buf.getvalue()


@pytest.mark.parametrize("w,h,q,sub,gray,restart", [
    (72, 40, 75, 2, False, {}), (131, 67, 30, 0, False, {}), (64, 48, 50, 0, True, {}),
    (200, 136, 90, 2, False, {}), (33, 17, 20, 1, False, {}), (130, 70, 60, 2, False, {"restart_marker_blocks": 3}),
    (96, 80, 40, 0, False, {"restart_marker_rows": 1}), (57, 91, 85, 0, True, {"restart_marker_blocks": 5}),
])
def test_progressive_equals_sequential(w, h, q, sub, gray, restart):
    """A progressive stream (libjpeg's default script: spectral selection and
    successive approximation for DC and AC, EOB runs) of the same image carries
    the same quantised coefficients as the sequential one: the decoder must
    return them bit for bit, with the same tables and sizes."""
    img = synth.channel_image(h, w, 7) if gray else synth.rgb_image(h, w, 7)
    a = Jpeg.from_source(JpegSource.Buffer(_pillow(img, q, sub, False, **restart)))
    pdata = _pillow(img, q, sub, True, **restart)
    assert pdata[:2] == b"\xff\xd8" and b"\xff\xc2" in pdata  # really progressive (SOF2)
    b = Jpeg.from_source(JpegSource.Buffer(pdata))
    assert (a.nchannel, a.real_px_w, a.real_px_h) == (b.nchannel, b.real_px_w, b.real_px_h)
    for x, y in zip(a.coefs, b.coefs):
        assert (x.rounded_px_w, x.rounded_px_h, x.horizontal_samp_factor, x.vertical_samp_factor) == (
            y.rounded_px_w, y.rounded_px_h, y.horizontal_samp_factor, y.vertical_samp_factor)
        np.testing.assert_array_equal(x.quant_table, y.quant_table)
        np.testing.assert_array_equal(x.dct_coefs, y.dct_coefs)


@pytest.mark.parametrize("seed,w,h,q,sub,restart", [
    (0, 320, 200, 95, 0, {}), (1, 257, 131, 60, 2, {"restart_marker_blocks": 2}), (2, 96, 512, 15, 1, {}),
    (3, 641, 97, 100, 2, {"restart_marker_rows": 1}), (4, 33, 47, 80, 0, {}),
])
def test_optimised_tables_sequential_equals_progressive(seed, w, h, q, sub, restart):
    """Streams with image-specific (optimised) Huffman tables -- long codes and,
    on a noisy image, large magnitudes: the sequential path (its combined
    code-and-magnitude lookup) and the progressive path decode the same
    coefficients."""
    rng = np.random.default_rng(seed)
    img = synth.rgb_image(h, w, 11 + seed).astype(np.int16) + rng.integers(-70, 71, size=(h, w, 3))
    img = np.clip(img, 0, 255).astype(np.uint8)
    a = Jpeg.from_source(JpegSource.Buffer(_pillow(img, q, sub, False, optimize=True, **restart)))
    b = Jpeg.from_source(JpegSource.Buffer(_pillow(img, q, sub, True, **restart)))
    for x, y in zip(a.coefs, b.coefs):
        np.testing.assert_array_equal(x.quant_table, y.quant_table)
        np.testing.assert_array_equal(x.dct_coefs, y.dct_coefs)


def test_truncated_progressive_stream_is_an_error_or_partial():
    """A progressive stream cut inside its scans decodes what it holds or fails
    with a decode error; it never crashes."""
    data = _pillow(synth.rgb_image(64, 64, 3), 75, 2, True)
    for cut in (len(data) // 4, len(data) // 2, len(data) - 10):
        try:
            Jpeg.from_source(JpegSource.Buffer(data[:cut]))
        except ArtefactError:
            pass


def test_truncated_stream_is_an_error():
    data = synth.make_jpeg(64, 64, 75, "4:2:0", False, seed=2)
    with pytest.raises(ArtefactError):
        Jpeg.from_source(JpegSource.Buffer(data[:200]))


@pytest.mark.parametrize("progressive", [False, True])
def test_corrupted_streams_never_crash(progressive):
    """Seeded byte flips in the entropy-coded data: each decode returns
    coefficients or a decode error (the decoder reads only inside the buffer
    and writes only inside its planes)."""
    rng = np.random.default_rng(17 + progressive)
    data = _pillow(synth.rgb_image(48, 80, 5), 70, 2, progressive, restart_marker_blocks=4)
    start = data.index(b"\xff\xda")
    for _ in range(150):
        d = bytearray(data)
        for _ in range(int(rng.integers(1, 6))):
            d[int(rng.integers(start + 10, len(d) - 2))] = int(rng.integers(0, 256))
        try:
            j = Jpeg.from_source(JpegSource.Buffer(bytes(d)))
            assert all(c.dct_coefs.size == c.block_w * c.block_h * 64 for c in j.coefs)
        except ArtefactError:
            pass


def test_decoded_coefficients_are_read_only_views():
    """Coefficient arrays of a decoded JPEG view the decoder's planes without a
    copy and are read-only: editing needs an explicit copy()."""
    j = Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(40, 24, 50, "4:4:4", True, seed=3)))
    a = j.coefs[0].dct_coefs
    assert not a.flags.writeable
    with pytest.raises(ValueError):
        a[0] = 1
    b = a.copy()
    b[0] += 1
    assert b[0] == a[0] + 1
