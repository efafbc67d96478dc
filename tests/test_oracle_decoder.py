"""The oracle's plain-Python JPEG decoder (CPU only).

Pinned against the known coefficients the test encoder writes (the golden
round-trip fixtures and seeded random streams, with restart markers and
separate scans), then used as a second, independent check (a) of the
product's decoder on Pillow-encoded synthetic JPEGs: coefficients, tables and
sizes must agree exactly.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

import jpeg_encoder as E
from artefact_b200 import synth
from artefact_b200.api import Jpeg, JpegSource

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
import jpeg_oracle as JO  # noqa: E402

GOLDEN = Path(__file__).resolve().parent / "golden"


def _same(o, expect):
    for c, (coefs, qt, bw, bh, sh, sv) in zip(o.coefs, expect):
        assert (c.block_w, c.block_h, c.horizontal_samp_factor, c.vertical_samp_factor) == (bw, bh, sh, sv)
        assert (c.rounded_px_w, c.rounded_px_h) == (bw * 8, bh * 8)
        assert np.array_equal(c.dct_coefs.reshape(-1, 64), coefs)
        assert np.array_equal(c.quant_table, qt)


@pytest.mark.parametrize("name", ["gray_37x21", "420_100x70_rst3", "422_50x30", "444_24x40_rst5"])
def test_golden_roundtrip(name):
    o = JO.decode((GOLDEN / f"roundtrip_{name}.jpg").read_bytes())
    ref = np.load(GOLDEN / f"roundtrip_{name}.npz")
    n = len([k for k in ref.files if k.startswith("coefs")])
    assert o.nchannel == n
    _same(o, [(ref[f"coefs{i}"], ref[f"qt{i}"], *ref[f"meta{i}"].tolist()) for i in range(n)])


@pytest.mark.parametrize("seed", range(8))
def test_random_roundtrip(seed):
    rng = np.random.default_rng(300 + seed)
    samplings = [[(1, 1)], [(2, 2), (1, 1), (1, 1)], [(2, 1), (1, 1), (1, 1)], [(1, 1)] * 3]
    samp = samplings[seed % len(samplings)]
    w, h = int(rng.integers(1, 90)), int(rng.integers(1, 90))
    comps, expect, (rw, rh) = E.random_image(rng, w, h, samp, qt_max=255 if seed % 2 else 1000)
    data = E.encode(w, h, comps, restart_interval=int(rng.integers(0, 4)))
    o = JO.decode(data)
    assert (o.real_px_w, o.real_px_h) == (w, h)
    assert o.max_rounded()[:2] == (rw, rh)
    _same(o, expect)


@pytest.mark.parametrize("seed,w,h,samp,restart", [
    (0, 33, 17, [(2, 2), (1, 1), (1, 1)], 0),
    (2, 17, 11, [(2, 1), (1, 1), (1, 1)], 2),
    (4, 97, 9, [(2, 2), (1, 1), (1, 1)], 5),
])
def test_separate_component_scans(seed, w, h, samp, restart):
    """One non-interleaved scan per component (T.81 A.2.2): blocks past the
    coded ones stay zero."""
    rng = np.random.default_rng(900 + seed)
    comps, expect, _ = E.random_image(rng, w, h, samp)
    hmax, vmax = max(c.h for c in comps), max(c.v for c in comps)
    for c, (coefs, _, bw, bh, _, _) in zip(comps, expect):
        coded_w, coded_h = -(-(-(-w * c.h // hmax)) // 8), -(-(-(-h * c.v // vmax)) // 8)
        for grid in (c.coefs.reshape(bh, bw, 64), coefs.reshape(bh, bw, 64)):
            grid[:, coded_w:] = 0
            grid[coded_h:, :] = 0
    _same(JO.decode(E.encode(w, h, comps, restart_interval=restart, separate_scans=True)), expect)


@pytest.mark.parametrize("w,h,q,sub,gray", [(72, 40, 75, "4:2:0", False), (37, 21, 50, "4:4:4", True),
                                            (50, 30, 75, "4:2:2", False), (130, 70, 20, "4:4:4", False),
                                            (333, 211, 90, "4:2:0", False)])
def test_product_decoder_agrees(w, h, q, sub, gray):
    """Check (a) twice over: the product's decoder and the oracle's give the
    same coefficients, tables and sizes on Pillow-encoded JPEGs."""
    data = synth.make_jpeg(w, h, q, sub, gray, seed=41)
    o = JO.decode(data)
    p = Jpeg.from_source(JpegSource.Buffer(data))
    assert (o.nchannel, o.real_px_w, o.real_px_h) == (p.nchannel, p.real_px_w, p.real_px_h)
    for a, b in zip(o.coefs, p.coefs):
        assert (a.rounded_px_w, a.rounded_px_h, a.block_w, a.block_h, a.horizontal_samp_factor,
                a.vertical_samp_factor) == (b.rounded_px_w, b.rounded_px_h, b.block_w, b.block_h,
                                            b.horizontal_samp_factor, b.vertical_samp_factor)
        assert np.array_equal(a.dct_coefs, np.asarray(b.dct_coefs))
        assert np.array_equal(a.quant_table, np.asarray(b.quant_table, np.float32))


def test_progressive_is_rejected():
    from PIL import Image
    import io

    buf = io.BytesIO()
    Image.fromarray(synth.channel_image(32, 32, 1), "L").save(buf, format="JPEG", quality=70, progressive=True)
    with pytest.raises(JO.OracleDecodeError):
        JO.decode(buf.getvalue())
