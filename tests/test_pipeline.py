"""Overlapped decode + solve of many JPEGs (artefact_b200.pipeline).

CPU: order, depth and error propagation with a stand-in solver (the host
decoder is real). GPU: the images equal process_jpeg's, one by one.
"""
import numpy as np
import pytest

from artefact_b200 import Jpeg, JpegSource, process_jpeg, synth
from artefact_b200.pipeline import process_stream

SHAPES = [(40, 24, 50, "4:2:0"), (72, 40, 75, "4:4:4"), (16, 16, 30, "4:2:0"), (100, 56, 90, "4:2:0"),
          (48, 32, 60, "4:4:4"), (24, 40, 20, "4:2:0")]


def _datas():
    return [synth.make_jpeg(w, h, q, sub, False, seed=31 + i) for i, (w, h, q, sub) in enumerate(SHAPES)]


def test_order_and_depth_with_stand_in_solver():
    seen = []

    def fake(j):
        seen.append((j.real_px_w, j.real_px_h))
        return np.full((j.real_px_h, j.real_px_w, 3), len(seen), np.uint8)

    for depth in (1, 2, 5, 16):
        seen.clear()
        outs = list(process_stream(_datas(), decoders=3, solvers=2, depth=depth, solve=fake))
        assert [(o.shape[1], o.shape[0]) for o in outs] == [(w, h) for w, h, _, _ in SHAPES]
        assert sorted(seen) == sorted((w, h) for w, h, _, _ in SHAPES)


def test_decode_errors_surface_in_order():
    datas = _datas()
    datas[2] = datas[2][:40]  # truncated stream

    def fake(j):
        return np.zeros((j.real_px_h, j.real_px_w, 3), np.uint8)

    gen = process_stream(datas, decoders=2, solvers=1, depth=4, solve=fake)
    assert next(gen).shape == (24, 40, 3)
    assert next(gen).shape == (40, 72, 3)
    with pytest.raises(Exception):
        next(gen)


def test_rejects_bad_arguments():
    with pytest.raises(ValueError):
        list(process_stream(_datas(), depth=0))


@pytest.mark.gpu
def test_stream_equals_process_jpeg(gpu):
    datas = _datas()
    outs = list(process_stream(datas, (0.3,) * 3, (0.001,) * 3, (20,) * 3, decoders=3, solvers=2, depth=4,
                               device=0))
    for d, o in zip(datas, outs):
        j = Jpeg.from_source(JpegSource.Buffer(d))
        ref = process_jpeg(j, [0.3] * 3, [0.001] * 3, [20] * 3, False, device=0)
        np.testing.assert_array_equal(o, ref)
