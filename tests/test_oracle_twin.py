"""Two independent restatements of pipeline_scalar agree bit for bit (CPU).

The C oracle (oracle/oracle_body.inc) and the numpy fp32 transliteration
(oracle/pipeline_numpy.py) were written separately from the reference's Rust
(backend/artefact-lib/pipeline_scalar/*.rs, utils/dct.rs, utils/boxing.rs).
Every plane they return must be identical to the last bit, on the small
parity shapes (gray, 4:2:0, 4:2:2, 4:4:4, edge-cropped sizes), with the
DCT-distance term on, off and per channel, and on the 512x512 gray q50
benchmark configuration at a few iterations.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as O
from artefact_b200 import synth
from artefact_b200.api import Jpeg, JpegSource

sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "oracle"))
import pipeline_numpy as PN  # noqa: E402

SHAPES = [
    (40, 24, 50, "4:4:4", True),
    (8, 8, 50, "4:4:4", True),
    (72, 40, 75, "4:2:0", False),
    (16, 16, 60, "4:2:0", False),
    (48, 32, 30, "4:4:4", False),
    (33, 17, 90, "4:2:0", False),
    (130, 70, 20, "4:4:4", False),
    (50, 30, 75, "4:2:2", False),
]


def _jpeg(w, h, q, sub, gray, seed):
    return Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(w, h, q, sub, gray, seed)))


def _bits_equal(a, b):
    return all(np.array_equal(np.asarray(x, np.float32).view(np.uint32), np.asarray(y, np.float32).view(np.uint32))
               for x, y in zip(a, b))


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[0]}x{s[1]}_q{s[2]}_{s[3]}{'_gray' if s[4] else ''}")
@pytest.mark.parametrize("iterations", [0, 1, 3, 8])
def test_numpy_and_c_oracles_are_bit_identical(shape, iterations):
    j = _jpeg(*shape, seed=11)
    W, H, _ = j.max_rounded()
    a = O.compute(j.nchannel, j.coefs, 0.3, [0.001] * 3, iterations, W, H)
    b = PN.compute(j.nchannel, j.coefs, 0.3, [0.001] * 3, iterations, W, H)
    assert _bits_equal(a, b)


@pytest.mark.parametrize("weight,pweight", [(0.0, (0.001,) * 3), (0.3, (0.0,) * 3), (1.5, (0.01, 0.0, 0.02))])
def test_weights_bit_identical(weight, pweight):
    j = _jpeg(72, 40, 75, "4:2:0", False, seed=12)
    W, H, _ = j.max_rounded()
    a = O.compute(3, j.coefs, weight, pweight, 6, W, H)
    b = PN.compute(3, j.coefs, weight, pweight, 6, W, H)
    assert _bits_equal(a, b)


def test_config1_512_gray_q50_bit_identical():
    j = _jpeg(512, 512, 50, "4:4:4", True, seed=1000)
    W, H, _ = j.max_rounded()
    a = O.compute(1, j.coefs, 0.3, [0.001] * 3, 3, W, H)
    b = PN.compute(1, j.coefs, 0.3, [0.001] * 3, 3, W, H)
    assert _bits_equal(a, b)


def test_transforms_bit_identical():
    rng = np.random.default_rng(5)
    for _ in range(20):
        blk = (rng.standard_normal((8, 8)) * 100).astype(np.float32)
        assert np.array_equal(O.dct8x8(blk).view(np.uint32), PN.dct8x8(blk).view(np.uint32))
        assert np.array_equal(O.idct8x8(blk).view(np.uint32), PN.idct8x8(blk).view(np.uint32))
