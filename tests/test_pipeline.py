"""Overlapped decode + solve of many JPEGs (artefact_b200.pipeline).

CPU: order, depth, batch budgets and error propagation with a stand-in solver
(the host decoder is real). GPU: the images equal process_jpeg's, one by one,
whether solved in batches (art_context_process_batch) or image by image, in
joint and separate mode.
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

    for depth in (0, 1, 2, 5, 16):
        for batch_images, batch_pixels in ((1, 1 << 30), (2, 1 << 30), (32, 3000), (32, 1 << 30)):
            seen.clear()
            outs = list(process_stream(_datas(), decoders=3, solvers=2, depth=depth, batch_images=batch_images,
                                       batch_pixels=batch_pixels, solve=fake))
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
    for kw in (dict(depth=-1), dict(batch_images=0), dict(batch_pixels=0), dict(solvers=0), dict(decoders=0),
               dict(solvers=2, contexts=[object()])):
        with pytest.raises(ValueError):
            list(process_stream(_datas(), **kw))


@pytest.mark.gpu
@pytest.mark.parametrize("batch_images", [1, 3, 32])
@pytest.mark.parametrize("separate,iterations", [(False, (20, 20, 20)), (True, (12, 12, 12)), (True, (15, 8, 4))])
def test_stream_equals_process_jpeg(gpu, batch_images, separate, iterations):
    datas = _datas() + [synth.make_jpeg(37, 21, 50, "4:4:4", True, seed=44)]
    weight, pweight = (0.3, 0.5, 0.2), (0.001, 0.002, 0.003)
    outs = list(process_stream(datas, weight, pweight, iterations, separate, decoders=3, solvers=2,
                               batch_images=batch_images, device=0))
    assert len(outs) == len(datas)
    for d, o in zip(datas, outs):
        j = Jpeg.from_source(JpegSource.Buffer(d))
        ref = process_jpeg(j, list(weight), list(pweight), list(iterations), separate, device=0)
        np.testing.assert_array_equal(o, ref)


@pytest.mark.gpu
def test_caller_contexts_serve_two_streams(gpu):
    """Contexts passed in stay open after the stream and give the same images
    on the next one (buffers and graphs reused, shapes changing between
    batches)."""
    from artefact_b200.api import Context

    datas = _datas()
    weight, pweight, iterations = (0.3, 0.3, 0.3), (0.001, 0.001, 0.001), (16, 16, 16)
    ctxs = [Context(0), Context(0)]
    try:
        first = list(process_stream(datas, weight, pweight, iterations, decoders=2, solvers=2, batch_images=2,
                                    contexts=ctxs))
        second = list(process_stream(datas[::-1], weight, pweight, iterations, decoders=2, solvers=2,
                                     batch_images=3, contexts=ctxs))
    finally:
        for c in ctxs:
            c.close()
    for a, b in zip(first, second[::-1]):
        np.testing.assert_array_equal(a, b)
    for d, o in zip(datas, first):
        ref = process_jpeg(Jpeg.from_source(JpegSource.Buffer(d)), list(weight), list(pweight), list(iterations),
                           False, device=0)
        np.testing.assert_array_equal(o, ref)
