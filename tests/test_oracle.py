"""Pins of the CPU oracle (CPU only).

The reference has no solver tests or golden vectors (it is Rust and cannot be
run here), so parity of the oracle with the reference is unpinned; these tests
pin it instead by known answers of the transforms, by finite differences of
the objective, by its fp64 twin and by committed golden outputs.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as O
from artefact_b200.api import Jpeg, JpegSource

GOLDEN = Path(__file__).resolve().parent / "golden"


def dct_matrix() -> np.ndarray:
    k = np.arange(8)[:, None]
    n = np.arange(8)[None, :]
    m = np.sqrt(2 / 8) * np.cos(np.pi * (2 * n + 1) * k / 16)
    m[0] /= np.sqrt(2)
    return m


def test_dct_matches_orthonormal_dct_ii():
    rng = np.random.default_rng(0)
    m = dct_matrix()
    for _ in range(20):
        a = rng.uniform(-255, 255, (8, 8))
        ref = m @ a @ m.T
        np.testing.assert_allclose(O.dct8x8(a, fp64=True), ref, atol=1e-9)
        np.testing.assert_allclose(O.dct8x8(a), ref, atol=2e-4)
        np.testing.assert_allclose(O.idct8x8(ref, fp64=True), a, atol=1e-9)


def test_dct_constant_block_and_roundtrip():
    a = np.full((8, 8), 100.0)
    d = O.dct8x8(a, fp64=True)
    assert abs(d[0, 0] - 800.0) < 1e-9
    assert np.abs(d.ravel()[1:]).max() < 1e-9
    rng = np.random.default_rng(1)
    for _ in range(20):
        x = rng.uniform(-128, 128, (8, 8)).astype(np.float32)
        np.testing.assert_allclose(O.idct8x8(O.dct8x8(x)), x, atol=1e-4)


def _load(name):
    return Jpeg.from_source(JpegSource.File(str(GOLDEN / f"synth_{name}.jpg")))


@pytest.mark.parametrize("name", ["gray_40x24_q50", "420_72x40_q75", "444_48x32_q30"])
def test_oracle_reproduces_golden(name):
    j = _load(name)
    g = np.load(GOLDEN / f"synth_{name}.npz")
    W, H, _ = j.max_rounded()
    it = int(g["iterations"])
    out32 = np.stack(O.compute(j.nchannel, j.coefs, 0.3, [0.001] * 3, it, W, H))
    out64 = np.stack(O.compute(j.nchannel, j.coefs, 0.3, [0.001] * 3, it, W, H, fp64=True))
    assert np.array_equal(out32, g["f32"])
    np.testing.assert_allclose(out64, g["f64"], rtol=0, atol=1e-9)
    # fp32 restatement stays close to its fp64 twin.
    assert np.abs(out32 - out64).max() < 0.5


@pytest.mark.parametrize("name", ["gray_40x24_q50", "420_72x40_q75", "444_48x32_q30"])
def test_gradient_matches_finite_differences(name):
    """Interior TV/TGV/prob gradient equals the derivative of the objective."""
    j = _load(name)
    W, H, _ = j.max_rounded()
    x = [p.astype(np.float64) for p in O.compute(j.nchannel, j.coefs, 0.3, [0.001] * 3, 3, W, H, fp64=True)]
    rng = np.random.default_rng(5)
    x = [p + rng.normal(0, 2.0, p.shape) for p in x]  # move off the box to exercise the prob term
    g = O.gradient(j.nchannel, j.coefs, 0.3, [0.001] * 3, W, H, x)
    h = 1e-5
    errs = []
    for _ in range(60):
        c = int(rng.integers(j.nchannel))
        yy, xx = int(rng.integers(3, H - 3)), int(rng.integers(3, W - 3))
        p = yy * W + xx
        xp = [a.copy() for a in x]
        xm = [a.copy() for a in x]
        xp[c][p] += h
        xm[c][p] -= h
        fd = (O.objective(j.nchannel, j.coefs, 0.3, [0.001] * 3, W, H, xp) -
              O.objective(j.nchannel, j.coefs, 0.3, [0.001] * 3, W, H, xm)) / (2 * h)
        errs.append(abs(fd - g[c][p]) / max(1.0, abs(fd)))
    assert np.median(errs) < 1e-5
    assert np.percentile(errs, 90) < 1e-3


def test_objective_decreases_and_output_feasible():
    j = _load("420_72x40_q75")
    W, H, _ = j.max_rounded()
    e0 = O.objective(3, j.coefs, 0.3, [0.001] * 3, W, H, O.compute(3, j.coefs, 0.3, [0.001] * 3, 0, W, H))
    out = O.compute(3, j.coefs, 0.3, [0.001] * 3, 50, W, H)
    e50 = O.objective(3, j.coefs, 0.3, [0.001] * 3, W, H, out)
    assert e50 < 0.9 * e0
    assert O.feasibility(3, j.coefs, W, H, out) < 1e-3


def test_scalar_compat_init_differs_and_is_deterministic():
    j = _load("gray_40x24_q50")
    W, H, _ = j.max_rounded()
    a = O.compute(1, j.coefs, 0.3, [0.001] * 3, 0, W, H, init_mode=1)[0]
    b = O.compute(1, j.coefs, 0.3, [0.001] * 3, 0, W, H, init_mode=1)[0]
    d = O.compute(1, j.coefs, 0.3, [0.001] * 3, 0, W, H, init_mode=0)[0]
    assert np.array_equal(a, b)
    assert not np.array_equal(a, d)


def test_rgb_output_stage_truncates():
    planes = [np.array([-128.0, 127.9, 10.6, 500.0], np.float32), np.zeros(4, np.float32),
              np.array([0.0, 0.0, 1.0, 0.0], np.float32)]
    out = O.rgb(3, 4, 4, 1, planes)
    assert out[0, 0].tolist() == [0, 0, 0]
    assert out[0, 1].tolist() == [255, 255, 255]
    # 138.6 + 1.402 = 140.002 -> 140; G = 138.6 - 0.71414 = 137.88 -> 137; B = 138.6 -> 138
    assert out[0, 2].tolist() == [140, 137, 138]
    gray = O.rgb(1, 4, 4, 1, planes[:1])
    assert gray[0, 2].tolist() == [138, 138, 138]


def test_compute_from_step_decay():
    """A step decay of 1 is the constant schedule; a smaller one changes the
    result and keeps the planes feasible."""
    from artefact_b200 import synth
    from artefact_b200.api import Jpeg, JpegSource

    j = Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(48, 32, 60, "4:2:0", False, seed=9)))
    W, H, _ = j.max_rounded()
    start = O.compute(3, j.coefs, 0.3, [0.001] * 3, 0, W, H)
    a = O.compute_from(3, j.coefs, 0.3, [0.001] * 3, 6, W, H, start, 2, tail_iterations=2, tail_step_iterations=50)
    b = O.compute_from(3, j.coefs, 0.3, [0.001] * 3, 6, W, H, start, 2, tail_iterations=2, tail_step_iterations=50,
                       step_decay=1.0)
    c = O.compute_from(3, j.coefs, 0.3, [0.001] * 3, 6, W, H, start, 2, tail_iterations=2, tail_step_iterations=50,
                       step_decay=0.5)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert any(not np.array_equal(x, y) for x, y in zip(a, c))
    assert O.feasibility(3, j.coefs, W, H, c) <= 1e-3


def test_rows_first_idct_variant_is_a_rounding_variant():
    """Mode bit 2 (the projection's IDCTs rows first, as the GPU runs them) is
    the same iteration up to fp32 rounding: its result stays within the
    reference-order fp32 result's own distance from fp64, and in fp64 the two
    orders agree to rounding."""
    from artefact_b200 import synth

    j = Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(64, 48, 75, "4:2:0", False, seed=11)))
    W, H, _ = j.max_rounded()
    args = (3, j.coefs, 0.3, [0.001] * 3, 6, W, H)
    ref = O.compute(*args)
    rows = O.compute(*args, init_mode=4)
    r64 = O.compute(*args, fp64=True)
    r64_rows = O.compute(*args, init_mode=4, fp64=True)
    d = max(float(np.abs(a.astype(np.float64) - b).max()) for a, b in zip(ref, rows))
    spread = max(float(np.abs(a.astype(np.float64) - b).max()) for a, b in zip(ref, r64))
    assert 0 < d <= max(4 * spread, 1e-3)
    assert max(float(np.abs(a - b).max()) for a, b in zip(r64, r64_rows)) < 1e-9
