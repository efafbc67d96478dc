"""The warm-start network's CPU FP64 oracle against finite differences (CPU)."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "oracle"))
import cnn_oracle as O  # noqa: E402


def _case(seed, B=1, H=16, W=16):
    rng = np.random.default_rng(seed)
    _, total = O.offsets()
    params = np.zeros(total)
    offs, _ = O.offsets()
    for name, cin, cout, _, _ in O.LAYERS:
        wo, bo = offs[name]
        params[wo:wo + cout * 9 * cin] = rng.standard_normal(cout * 9 * cin) * np.sqrt(2.0 / (9 * cin))
        params[bo:bo + cout] = rng.standard_normal(cout) * 0.05
    coef = rng.integers(-20, 20, size=(B, H, W)).astype(np.int16)
    q = rng.integers(2, 40, size=(B, 64)).astype(np.float64)
    dec, F = O.features(coef, q)
    target = dec + rng.standard_normal(dec.shape) * 4.0
    return params, F, dec, target


def test_features_decode_dc_block():
    coef = np.zeros((1, 8, 8), np.int16)
    coef[0, 0, 0] = 4
    q = np.full((1, 64), 2.0)
    dec, F = O.features(coef, q)
    np.testing.assert_allclose(dec, 1.0, atol=1e-12)  # DC 8 / 8 (orthonormal 2-D DCT)
    assert F.shape == (1, 8, 8, 16)  # level 0 of an 8x8 component: padded to 16x16, halved
    np.testing.assert_allclose(F[0, :4, :4, 0:4], 1.0 / 128.0, atol=1e-12)
    np.testing.assert_allclose(F[0, :4, :4, 4:8], 2.0 / 64.0)
    assert np.all(F[0, 4:] == 0) and np.all(F[0, :, 4:] == 0)  # padding
    assert np.all(F[..., 8:] == 0)


def test_space_to_depth_round_trip():
    rng = np.random.default_rng(4)
    a = rng.standard_normal((2, 24, 40))
    H0, W0 = O.level0(24, 40)
    assert (H0, W0) == (16, 24)
    s = O.space_to_depth(a, H0, W0)
    assert s[1, 3, 5, 2] == a[1, 7, 10] and s[1, 3, 5, 1] == a[1, 6, 11]
    np.testing.assert_array_equal(O.depth_to_space(s, 24, 40), a)


def test_gradients_match_finite_differences():
    """Central differences with a step small enough that no ReLU changes side."""
    params, F, dec, target = _case(1)
    loss, g = O.gradients(params, F, dec, target, bf=False)
    rng = np.random.default_rng(7)
    for _ in range(3):
        v = rng.standard_normal(params.size)
        eps = 1e-8
        lp = O.forward(params + eps * v, F, dec, target, bf=False)[2]
        lm = O.forward(params - eps * v, F, dec, target, bf=False)[2]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g @ v) <= 1e-5 * max(1.0, abs(fd)), (fd, g @ v)


def test_layer_gradients_match_finite_differences():
    """Per layer, so that a wrong slice (skip vs upsampled channels) cannot hide."""
    params, F, dec, target = _case(2, H=24, W=40)
    _, g = O.gradients(params, F, dec, target, bf=False)
    offs, _ = O.offsets()
    rng = np.random.default_rng(3)
    for name, cin, cout, _, _ in O.LAYERS:
        wo, bo = offs[name]
        for lo, hi in ((wo, wo + cout * 9 * cin), (bo, bo + cout)):
            v = np.zeros(params.size)
            v[lo:hi] = rng.standard_normal(hi - lo)
            eps = 1e-8
            fd = (O.forward(params + eps * v, F, dec, target, bf=False)[2] -
                  O.forward(params - eps * v, F, dec, target, bf=False)[2]) / (2 * eps)
            assert abs(fd - g @ v) <= 1e-5 * max(1e-3, abs(fd)), (name, fd, g @ v)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0], np.float64)
    r = O.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5 and r[4] == 0.0


def test_smooth_loss_gradient_matches_finite_differences():
    """The smoothness term of the training loss, checked on the whole network."""
    params, F, dec, target = _case(5, H=16, W=24)
    loss, g = O.gradients(params, F, dec, target, bf=False, smooth=2.0)
    assert loss > O.forward(params, F, dec, target, bf=False)[2]
    rng = np.random.default_rng(8)
    for _ in range(3):
        v = rng.standard_normal(params.size)
        eps = 1e-8
        lp = O.forward(params + eps * v, F, dec, target, bf=False, smooth=2.0)[2]
        lm = O.forward(params - eps * v, F, dec, target, bf=False, smooth=2.0)[2]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g @ v) <= 1e-5 * max(1.0, abs(fd)), (fd, g @ v)


def _interior(shape, ring, rng):
    d = np.zeros(shape)
    d[:, ring:-ring, ring:-ring] = rng.standard_normal((shape[0], shape[1] - 2 * ring, shape[2] - 2 * ring))
    return d


def test_objective_gradient_matches_finite_differences():
    """The training loss's objective term: the gradient the reference's scatter
    gives (TV, TGV) against central differences of the objective, for
    perturbations off the first and last rows and columns (where the
    reference's second-order edge rule is not the derivative of its value)."""
    rng = np.random.default_rng(11)
    B, H, W = 2, 24, 32
    x = rng.standard_normal((B, H, W)) * 10
    a_tv, a_tgv, _ = O.solver_weights()
    zero = np.zeros((B, H // 8, W // 8, 8, 8))
    val, T = O.objective_value(x, zero, zero, a_tv, a_tgv, 0.0)
    g = O.objective_gradient(T)
    for _ in range(3):
        d = _interior(x.shape, 1, rng)
        eps = 1e-6
        fp = O.objective_value(x + eps * d, zero, zero, a_tv, a_tgv, 0.0)[0]
        fm = O.objective_value(x - eps * d, zero, zero, a_tv, a_tgv, 0.0)[0]
        fd = (fp - fm) / (2 * eps)
        assert abs(fd - float(np.sum(g * d))) <= 1e-6 * max(1.0, abs(fd)), (fd, float(np.sum(g * d)))


def test_objective_through_projection_matches_finite_differences():
    """E(proj(pred)) and its gradient through the projection (J = IDCT diag(m)
    DCT, symmetric), DCT-distance term included, with some coefficients
    clamped: perturbations confined to blocks off the image border."""
    rng = np.random.default_rng(12)
    B, H, W = 1, 32, 32
    coef = rng.integers(-6, 6, size=(B, H, W)).astype(np.int16)
    q = rng.integers(4, 30, size=(B, 64)).astype(np.float64)
    dec, _ = O.features(coef, q)
    pred = dec + rng.standard_normal(dec.shape) * 6
    a_tv, a_tgv, a_p = O.solver_weights()
    _, _, mask, _ = O.project(pred, coef, q)
    assert 0.05 < mask.mean() < 0.95  # some coefficients clamped, some free
    val, grad = O.objective_and_back(pred, coef, q, a_tv, a_tgv, a_p)
    assert val > 0
    for _ in range(3):
        d = np.zeros_like(pred)
        d[:, 8:24, 8:24] = rng.standard_normal((B, 16, 16))
        eps = 1e-6
        fp = O.objective_and_back(pred + eps * d, coef, q, a_tv, a_tgv, a_p)[0]
        fm = O.objective_and_back(pred - eps * d, coef, q, a_tv, a_tgv, a_p)[0]
        fd = (fp - fm) / (2 * eps)
        assert abs(fd - float(np.sum(grad * d))) <= 1e-5 * max(1.0, abs(fd)), (fd, float(np.sum(grad * d)))


def test_objective_loss_gradient_matches_finite_differences():
    """The objective term of the training loss on the whole network. The
    perturbed parameters move every sample, edges included, where the
    reference's second-order edge rule differs from the derivative of the
    value (a few 1e-4 here), so the bar is 2e-3; a wrong scale of the term
    would miss it by orders of magnitude."""
    params, F, dec, target = _case(6, H=16, W=24)
    rng = np.random.default_rng(9)
    coef = rng.integers(-20, 20, size=(1, 16, 24)).astype(np.int16)
    q = rng.integers(2, 40, size=(1, 64)).astype(np.float64)
    dec, F = O.features(coef, q)
    obj = (0.05, coef, q) + O.solver_weights()
    loss, g = O.gradients(params, F, dec, target, bf=False, objective=obj)
    assert loss > O.forward(params, F, dec, target, bf=False)[2]
    for _ in range(3):
        v = rng.standard_normal(params.size)
        eps = 1e-8
        lp = O.forward(params + eps * v, F, dec, target, bf=False, objective=obj)[2]
        lm = O.forward(params - eps * v, F, dec, target, bf=False, objective=obj)[2]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g @ v) <= 2e-3 * max(1.0, abs(fd)), (fd, g @ v)


def _joint_case(seed, B=1, H=32, W=48):
    rng = np.random.default_rng(seed)
    params, _, _, _ = _case(seed)
    cy = rng.integers(-20, 20, size=(B, H, W)).astype(np.int16)
    cc = rng.integers(-20, 20, size=(B, 2, H // 2, W // 2)).astype(np.int16)
    qy = rng.integers(2, 40, size=(B, 64)).astype(np.float64)
    qc = rng.integers(2, 40, size=(B, 2, 64)).astype(np.float64)
    dec, F = O.features_joint(cy, qy, cc, qc)
    target = dec + rng.standard_normal(dec.shape) * 4.0
    return params, F, dec, target, (cy, qy, cc, qc)


def test_joint_features_layout():
    """Channels 8-11 carry the chroma samples and steps at the luma's level 0;
    the chroma bases are the decoded chroma upsampled as the learned start
    upsamples (warmstart.upsample_component, float32)."""
    from artefact_b200.warmstart import upsample_component

    _, F, dec, _, (cy, qy, cc, qc) = _joint_case(3)
    B, H, W = cy.shape
    decC, _ = O.features(cc.reshape(2 * B, H // 2, W // 2), qc.reshape(2 * B, 64))
    np.testing.assert_allclose(F[0, :, :, 8], decC[0] / 128.0)
    np.testing.assert_allclose(F[0, 5, 11, 11], qc[0, 1, 5 * 8 + 3] / 64.0)
    assert np.all(F[..., 12:] == 0)
    up = upsample_component(decC[1].astype(np.float32), 2, 2, H, W)
    np.testing.assert_allclose(dec[2, 0], up, atol=1e-3)


def test_joint_loss_gradient_matches_finite_differences():
    params, F, dec, target, _ = _joint_case(4)
    loss, g = O.gradients(params, F, dec, target, bf=False, joint=True)
    rng = np.random.default_rng(10)
    for _ in range(3):
        v = rng.standard_normal(params.size)
        eps = 1e-8
        lp = O.forward(params + eps * v, F, dec, target, bf=False, joint=True)[2]
        lm = O.forward(params - eps * v, F, dec, target, bf=False, joint=True)[2]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g @ v) <= 1e-5 * max(1.0, abs(fd)), (fd, g @ v)
