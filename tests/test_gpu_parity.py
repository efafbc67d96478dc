"""Parity of the CUDA solver with the CPU oracle, through the C ABI (GPU).

Bar (floating point, 0..255 pixel units): max |GPU - oracle fp32| <= 1.0 per
pixel of the float planes (1/255 of the 8-bit range), final objective within
1e-4 relative, every output block inside its quantisation box to 1e-3
coefficient units (fp64 DCT), and RGB8 within 1 LSB.

The error of both against the oracle's fp64 twin is measured on every case.
Where the input itself is ill-conditioned -- the oracle's own fp32 result is
more than 0.5 away from its fp64 twin, or its objective more than 2.5e-5
relative (tiny images at their first iterations, or the 24-megapixel image
whose fp32 gradient norm the reference folds sequentially) -- no fp32
implementation with another rounding order can meet a fixed bar. The bar then
becomes the spread of the oracle's own numerical variants around its fp64
result: fp32, and fp32/fp64 with the lagged DCT coefficients recomputed from
x_k (equal in exact arithmetic, and what the CUDA kernels do). The GPU must lie
within 2x that spread + 0.5 pixel units, and its objective within 2x + 1e-4.
"""
import ctypes as C
import threading

import numpy as np
import pytest

import oracle_lib as O
from artefact_b200 import Artefact, ArtError, JpegSource, ValueCollection, compute, process_jpeg, synth
from artefact_b200 import _native as N
from artefact_b200.api import Coefficient, Jpeg

pytestmark = pytest.mark.gpu

MAX_ABS = 1.0
OBJ_REL = 1e-4
FEAS = 1e-3

_cache = {}


def jpeg_of(w, h, q, sub, gray, seed):
    key = (w, h, q, sub, gray, seed)
    if key not in _cache:
        _cache[key] = Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(w, h, q, sub, gray, seed)))
    return _cache[key]


from parity import check_parity  # noqa: E402


SMALL = [
    (40, 24, 50, "4:4:4", True),
    (8, 8, 50, "4:4:4", True),
    (72, 40, 75, "4:2:0", False),
    (16, 16, 60, "4:2:0", False),
    (48, 32, 30, "4:4:4", False),
    (200, 136, 75, "4:2:0", False),
    (33, 17, 90, "4:2:0", False),
    (130, 70, 20, "4:4:4", False),
    (50, 30, 75, "4:2:2", False),
]


@pytest.mark.parametrize("shape", SMALL, ids=lambda s: f"{s[0]}x{s[1]}_q{s[2]}_{s[3]}{'_gray' if s[4] else ''}")
@pytest.mark.parametrize("iterations", [0, 1, 2, 10, 50])
def test_small_images(gpu, shape, iterations):
    j = jpeg_of(*shape, seed=11)
    check_parity(j, iterations, label=str(shape))


def test_config1_512_gray_q50(gpu):
    j = jpeg_of(512, 512, 50, "4:4:4", True, seed=1000)
    check_parity(j, 50, label="512x512 gray q50")


def test_config2_1080p_420_q75(gpu):
    j = jpeg_of(1920, 1080, 75, "4:2:0", False, seed=2000)
    check_parity(j, 50, label="1920x1080 4:2:0 q75")


def test_config3_24mp_444_q30_short(gpu):
    """Full-size 6000x4000 4:4:4 at 2 iterations against the oracle."""
    j = jpeg_of(6000, 4000, 30, "4:4:4", False, seed=3000)
    check_parity(j, 2, label="6000x4000 4:4:4 q30")


def test_config3_24mp_properties(gpu):
    """100 iterations at full size: feasible, deterministic, objective below x0."""
    j = jpeg_of(6000, 4000, 30, "4:4:4", False, seed=3000)
    W, H, N_ = j.max_rounded()
    a = compute(3, j.coefs, 0.3, [0.001] * 3, 100, W, H, N_)
    b = compute(3, j.coefs, 0.3, [0.001] * 3, 100, W, H, N_)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert O.feasibility(3, j.coefs, W, H, a) <= FEAS
    x0 = compute(3, j.coefs, 0.3, [0.001] * 3, 0, W, H, N_)
    assert O.objective(3, j.coefs, 0.3, [0.001] * 3, W, H, a) < O.objective(3, j.coefs, 0.3, [0.001] * 3, W, H, x0)


@pytest.mark.parametrize("weight,pweight", [(0.0, (0.001,) * 3), (0.3, (0.0,) * 3), (1.5, (0.01, 0.0, 0.02))])
def test_weights(gpu, weight, pweight):
    j = jpeg_of(72, 40, 75, "4:2:0", False, seed=12)
    check_parity(j, 20, weight=weight, pweight=pweight, label=f"w={weight} pw={pweight}")


def test_deterministic(gpu):
    j = jpeg_of(200, 136, 75, "4:2:0", False, seed=13)
    W, H, N_ = j.max_rounded()
    a = compute(3, j.coefs, 0.3, [0.001] * 3, 30, W, H, N_)
    b = compute(3, j.coefs, 0.3, [0.001] * 3, 30, W, H, N_)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_scalar_compat_init(gpu):
    j = jpeg_of(40, 24, 50, "4:4:4", True, seed=14)
    W, H, N_ = j.max_rounded()
    for it in (0, 5):
        gpu_out = compute(1, j.coefs, 0.3, [0.001] * 3, it, W, H, N_, init_mode=N.ART_INIT_SCALAR_COMPAT)[0]
        ref = O.compute(1, j.coefs, 0.3, [0.001] * 3, it, W, H, init_mode=1)[0]
        assert np.abs(gpu_out - ref).max() <= MAX_ABS


def test_f32_and_i16_coefficients_agree(gpu):
    j = jpeg_of(72, 40, 75, "4:2:0", False, seed=15)
    W, H, N_ = j.max_rounded()
    as_f32 = [Coefficient(c.rounded_px_w, c.rounded_px_h, c.block_w, c.block_h, c.horizontal_samp_factor,
                          c.vertical_samp_factor, c.dct_coefs.astype(np.float32), c.quant_table) for c in j.coefs]
    a = compute(3, j.coefs, 0.3, [0.001] * 3, 10, W, H, N_)
    b = compute(3, as_f32, 0.3, [0.001] * 3, 10, W, H, N_)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("separate", [False, True])
@pytest.mark.parametrize("shape", [(72, 40, 75, "4:2:0", False), (37, 21, 50, "4:4:4", True),
                                   (61, 45, 40, "4:4:4", False)])
def test_process_rgb_matches_oracle(gpu, shape, separate):
    j = jpeg_of(*shape, seed=16)
    weight, pweight, iters = [0.3, 0.5, 0.2], [0.001, 0.002, 0.003], [20, 10, 5]
    rgb = process_jpeg(j, weight, pweight, iters, separate)
    ref = O.process(j, weight, pweight, iters, separate)
    assert rgb.shape == ref.shape == (j.real_px_h, j.real_px_w, 3)
    diff = np.abs(rgb.astype(int) - ref.astype(int))
    assert diff.max() <= 1, diff.max()
    assert (diff > 0).mean() < 0.05


def test_artefact_builder_end_to_end(gpu, tmp_path):
    data = synth.make_jpeg(64, 48, 60, "4:2:0", False, seed=17)
    p = tmp_path / "in.jpg"
    p.write_bytes(data)
    out = (Artefact.default().source(JpegSource.File(str(p))).weight(ValueCollection.ForAll(0.3))
           .iterations(ValueCollection.ForAll(10)).process())
    assert out.shape == (48, 64, 3) and out.dtype == np.uint8
    with pytest.raises(Exception, match="BENCHMARK"):
        Artefact.default().source(JpegSource.Buffer(data)).benchmark(True).process()


def test_invalid_inputs_report_errors(gpu):
    j = jpeg_of(16, 16, 60, "4:4:4", True, seed=18)
    W, H, N_ = j.max_rounded()
    c = j.coefs[0]
    frac = Coefficient(c.rounded_px_w, c.rounded_px_h, c.block_w, c.block_h, 1, 1,
                       c.dct_coefs.astype(np.float32) + 0.25, c.quant_table)
    with pytest.raises(ArtError) as e:
        compute(1, [frac], 0.3, [0.001] * 3, 2, W, H, N_)
    assert e.value.code == N.ART_ERR_INVALID_DATA
    zero_q = Coefficient(c.rounded_px_w, c.rounded_px_h, c.block_w, c.block_h, 1, 1, c.dct_coefs,
                         np.zeros(64, np.float32))
    with pytest.raises(ArtError) as e:
        compute(1, [zero_q], 0.3, [0.001] * 3, 2, W, H, N_)
    assert e.value.code == N.ART_ERR_INVALID_DATA
    with pytest.raises(ArtError) as e:
        compute(1, [c], 0.3, [0.001] * 3, 2, W + 8, H, (W + 8) * H)
    assert e.value.code == N.ART_ERR_INVALID_ARGUMENT
    nan = Coefficient(c.rounded_px_w, c.rounded_px_h, c.block_w, c.block_h, 1, 1,
                      np.full(c.dct_coefs.shape, np.nan, np.float32), c.quant_table)
    with pytest.raises(ArtError):
        compute(1, [nan], 0.3, [0.001] * 3, 2, W, H, N_)
    # The context stays usable after errors.
    check_parity(j, 3)


def test_concurrent_threads(gpu):
    """Re-entrant like the reference's rayon callers (lib.rs:133-153)."""
    jobs = [jpeg_of(72, 40, 75, "4:2:0", False, seed=20 + i) for i in range(4)]
    results = [None] * 4

    def run(i):
        j = jobs[i]
        W, H, N_ = j.max_rounded()
        results[i] = compute(3, j.coefs, 0.3, [0.001] * 3, 15, W, H, N_)

    ts = [threading.Thread(target=run, args=(i,)) for i in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for i, j in enumerate(jobs):
        W, H, N_ = j.max_rounded()
        single = compute(3, j.coefs, 0.3, [0.001] * 3, 15, W, H, N_)
        assert all(np.array_equal(a, b) for a, b in zip(results[i], single))


def test_device_resident_entry_point(gpu):
    import torch

    j = jpeg_of(200, 136, 75, "4:2:0", False, seed=21)
    W, H, N_ = j.max_rounded()
    lib = N.lib()
    ctx = C.c_void_p()
    N.check(lib.art_context_create(0, C.byref(ctx)))
    try:
        dev_coefs = [torch.from_numpy(c.dct_coefs.copy()).cuda() for c in j.coefs]
        qs = [np.ascontiguousarray(c.quant_table, np.float32) for c in j.coefs]
        chans = (N.ArtChannel * 3)()
        for i, c in enumerate(j.coefs):
            ch = chans[i]
            ch.rounded_px_w, ch.rounded_px_h, ch.block_w, ch.block_h = c.rounded_px_w, c.rounded_px_h, c.block_w, c.block_h
            ch.samp_h, ch.samp_v, ch.coef_type = c.horizontal_samp_factor, c.vertical_samp_factor, N.ART_COEF_I16
            ch.dct_coefs = dev_coefs[i].data_ptr()
            ch.quant_table = qs[i].ctypes.data_as(C.POINTER(C.c_float))
        pitch = W + 32
        outs = [torch.empty(H, pitch, device="cuda") for _ in range(3)]
        ptrs = (C.c_void_p * 3)(*[o.data_ptr() for o in outs])
        pw = (C.c_float * 3)(0.001, 0.001, 0.001)
        stream = torch.cuda.current_stream().cuda_stream
        N.check(lib.art_context_compute_device(ctx, 3, chans, 0.3, pw, 25, W, H, ptrs, pitch, None, C.c_void_p(stream)))
        N.check(lib.art_context_synchronize(ctx))
        got = [o[:, :W].cpu().numpy().ravel() for o in outs]
        ref = compute(3, j.coefs, 0.3, [0.001] * 3, 25, W, H, N_)
        assert all(np.array_equal(a, b) for a, b in zip(got, ref))
    finally:
        lib.art_context_destroy(ctx)
