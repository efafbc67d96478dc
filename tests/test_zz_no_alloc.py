"""The allocation-free entry point art_solve_noalloc (GPU).

Some callers cannot allocate device memory: their GPU memory belongs to
another allocator (a framework's caching allocator, or a server that splits
each GPU up front), or they cannot afford the device-wide synchronisation that
cudaMalloc and cudaFree may cause. For them the library runs the solver out of
one fixed device array. This test calls that entry point through the C ABI
on consecutive calls and checks each result against the regular
device-resident entry point with the parity
tolerance the other GPU tests use: 4:2:0, grayscale, 4:4:4 and 4:2:2 images
one after the other, then the first again. It lives in its own file, collected last,
and works alone in a fresh process as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from artefact_b200 import _native as N
from artefact_b200 import synth
from artefact_b200.api import Jpeg, JpegSource

pytestmark = pytest.mark.gpu

MAX_ABS = 1.0  # the float-plane tolerance of the parity tests (0..255 units)


def _device_channels(j, torch):
    keep = []
    chans = (N.ArtChannel * j.nchannel)()
    for i, c in enumerate(j.coefs):
        d = torch.from_numpy(c.dct_coefs.copy()).cuda()
        q = np.ascontiguousarray(c.quant_table, np.float32)
        keep += [d, q]
        ch = chans[i]
        ch.rounded_px_w, ch.rounded_px_h, ch.block_w, ch.block_h = c.rounded_px_w, c.rounded_px_h, c.block_w, c.block_h
        ch.samp_h, ch.samp_v, ch.coef_type = c.horizontal_samp_factor, c.vertical_samp_factor, N.ART_COEF_I16
        ch.dct_coefs = d.data_ptr()
        ch.quant_table = q.ctypes.data_as(C.POINTER(C.c_float))
    return chans, keep


def _solve(entry, j, iterations, torch, ctx=None):
    lib = N.lib()
    W, H, _ = j.max_rounded()
    chans, keep = _device_channels(j, torch)
    pitch = W + 16
    outs = [torch.full((H, pitch), float("nan"), device="cuda") for _ in range(j.nchannel)]
    ptrs = (C.c_void_p * j.nchannel)(*[o.data_ptr() for o in outs])
    pw = (C.c_float * 3)(0.001, 0.001, 0.001)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if entry == "noalloc":
        N.check(lib.art_solve_noalloc(j.nchannel, chans, 0.3, pw, iterations, W, H, ptrs, pitch, stream))
    else:
        N.check(lib.art_context_compute_device(ctx, j.nchannel, chans, 0.3, pw, iterations, W, H, ptrs, pitch,
                                               None, stream))
        N.check(lib.art_context_synchronize(ctx))
    torch.cuda.synchronize()
    return [o[:, :W].cpu().numpy() for o in outs]


def test_noalloc_matches_regular_entry_point_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    lib = N.lib()
    ctx = C.c_void_p()
    N.check(lib.art_context_create(0, C.byref(ctx)))
    try:
        first = Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(200, 136, 75, "4:2:0", False, seed=41)))
        second = Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(96, 80, 50, "4:4:4", True, seed=42)))
        third = Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(130, 70, 30, "4:4:4", False, seed=43)))
        fourth = Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(64, 48, 60, "4:2:2", False, seed=44)))
        assert second.nchannel == 1 and fourth.coefs[1].horizontal_samp_factor == 2
        for j, iters in ((first, 20), (second, 12), (third, 15), (fourth, 10), (first, 20)):
            got = _solve("noalloc", j, iters, torch)
            ref = _solve("regular", j, iters, torch, ctx)
            for a, b in zip(got, ref):
                assert np.isfinite(a).all()
                assert np.abs(a - b).max() <= MAX_ABS
    finally:
        lib.art_context_destroy(ctx)


def test_noalloc_rejects_images_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    lib = N.lib()
    W, H = 4096, 4096  # 16.7 M pixels x 3 channels: far beyond 64 MiB of scratch
    q = np.ones(64, np.float32)
    chans = (N.ArtChannel * 3)()
    dummy = torch.zeros(1, dtype=torch.int16, device="cuda")
    for i in range(3):
        ch = chans[i]
        ch.rounded_px_w, ch.rounded_px_h, ch.block_w, ch.block_h = W, H, W // 8, H // 8
        ch.samp_h = ch.samp_v = 1
        ch.coef_type = N.ART_COEF_I16
        ch.dct_coefs = dummy.data_ptr()  # never read: the size check comes first
        ch.quant_table = q.ctypes.data_as(C.POINTER(C.c_float))
    out = (C.c_void_p * 3)(dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr())
    pw = (C.c_float * 3)(0.001, 0.001, 0.001)
    rc = lib.art_solve_noalloc(3, chans, 0.3, pw, 10, W, H, out, W, None)
    assert rc == N.ART_ERR_INVALID_ARGUMENT
    assert b"MiB of scratch" in lib.art_last_error()
