"""Tensor-core kernels of the warm-start network against the CPU FP64 oracle (GPU).

The oracle rounds to bf16 wherever the GPU stores bf16, so forward values
agree up to the GPU's fp32 accumulation order (a rare flip of one bf16 ulp,
2^-8 relative); weight gradients are fp32 sums of exact bf16 products.
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "oracle"))
import cnn_oracle as O  # noqa: E402

from artefact_b200 import _native as N  # noqa: E402
from artefact_b200 import warmstart as WS  # noqa: E402

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _bf(a):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).cuda()


def _f32(a):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def _np(t):
    return t.float().cpu().numpy().astype(np.float64)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _pack(w, transpose=0, ci0=0, n=None, ck=32):
    torch = _torch()
    cout, _, cin = w.shape
    n = n if n is not None else (cin if transpose else cout)
    K = cout if transpose else cin
    out = torch.empty(n * 9 * K, dtype=torch.bfloat16, device="cuda")
    wt = _f32(w)
    N.check(N.lib().art_cnn_pack_weights(_ptr(wt), cout, cin, transpose, ci0, n, ck, _ptr(out), None))
    return out


def _conv(x, wpack, cin, ck, n, bias=None, relu=0, mask=None, out=None, out_cstride=None, out_coff=0, f32=None,
          accumulate=0, pool_out=None, up2=0, tile_rows=0, f32_channels=0):
    torch = _torch()
    B, H, W, _ = x.shape
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    if out is None and f32 is None:
        out = torch.zeros((B, H, W, n), dtype=torch.bfloat16, device="cuda")
    d = N.ArtCnnConv()
    d.B, d.H, d.W, d.cin, d.ck, d.n, d.n_store = B, H, W, cin, ck, n, n
    d.x, d.wpack = x.data_ptr(), wpack.data_ptr()
    d.bias = bias.data_ptr() if bias is not None else None
    d.out = out.data_ptr() if out is not None else None
    d.out_cstride = out_cstride if out_cstride is not None else n
    d.out_coff = out_coff
    d.out_f32 = f32.data_ptr() if f32 is not None else None
    d.f32_cstride = f32_channels or n
    d.f32_channels = f32_channels
    d.mask = mask.data_ptr() if mask is not None else None
    d.mask_cstride = mask.shape[-1] if mask is not None else 0
    d.relu, d.accumulate = relu, accumulate
    d.err = err.data_ptr()
    d.pool_out = pool_out.data_ptr() if pool_out is not None else None
    d.up2 = up2
    d.tile_rows = tile_rows
    N.check(N.lib().art_cnn_conv3x3(C.byref(d), None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0, "a pipeline wait timed out"
    return out


def _close(got, ref, rel=1.2e-2):
    scale = max(float(np.abs(ref).max()), 1e-6)
    err = float(np.abs(got - ref).max())
    assert err <= rel * scale, f"max err {err:.3g} vs scale {scale:.3g}"
    # Mean error well below one bf16 ulp: only rare rounding flips.
    assert float(np.abs(got - ref).mean()) <= 1e-3 * scale


CONV_SHAPES = [(1, 8, 128, 16, 16), (2, 10, 200, 32, 64), (1, 6, 40, 64, 96), (1, 4, 260, 224, 96),
               (2, 16, 96, 96, 128), (1, 3, 130, 160, 32), (1, 7, 1100, 64, 64)]


@pytest.mark.parametrize("tile_rows", [0, 1, 2, 4, 8])
@pytest.mark.parametrize("B,H,W,cin,cout", CONV_SHAPES)
def test_conv_forward(gpu, B, H, W, cin, cout, tile_rows):
    """Every tile height (0: the automatic choice) on ragged heights and widths."""
    if tile_rows * cout > 256:
        pytest.skip("two tiles' accumulators hold 2 x tile_rows x n TMEM columns: at most 512")
    rng = np.random.default_rng(cin * 7 + cout)
    x = O.bf16(rng.standard_normal((B, H, W, cin)))
    w = O.bf16(rng.standard_normal((cout, 9, cin)) * np.sqrt(2 / (9 * cin)))
    b = rng.standard_normal(cout) * 0.1
    ck = 32 if cin % 32 == 0 else 16
    got = _np(_conv(_bf(x), _pack(w, ck=ck), cin, ck, cout, bias=_f32(b), relu=1, tile_rows=tile_rows))
    ref = O.bf16(np.maximum(O.conv(x, w, b), 0))
    _close(got, ref)


def test_conv_rejects_bad_tile_rows(gpu):
    torch = _torch()
    x = torch.zeros((1, 4, 16, 16), dtype=torch.bfloat16, device="cuda")
    wp = torch.zeros(9 * 16 * 96, dtype=torch.bfloat16, device="cuda")
    pooled = torch.zeros((1, 2, 8, 96), dtype=torch.bfloat16, device="cuda")
    for kw in ({"tile_rows": 3}, {"tile_rows": 4}, {"tile_rows": 16}, {"tile_rows": 1, "pool_out": pooled}):
        with pytest.raises(N.ArtError):
            _conv(x, wp, 16, 16, 96, **kw)


def test_conv_channel_offset_accumulate_and_f32(gpu):
    torch = _torch()
    rng = np.random.default_rng(5)
    B, H, W, cin, cout = 1, 6, 150, 32, 32
    x = O.bf16(rng.standard_normal((B, H, W, cin)))
    w = O.bf16(rng.standard_normal((cout, 9, cin)) * 0.1)
    wp = _pack(w)
    base = O.bf16(rng.standard_normal((B, H, W, 96)))
    out = _bf(base)
    _conv(_bf(x), wp, cin, 32, cout, out=out, out_cstride=96, out_coff=32, accumulate=1)
    got = _np(out)
    ref = base.copy()
    ref[..., 32:64] = O.bf16(base[..., 32:64] + O.conv(x, w))
    assert np.array_equal(got[..., :32], base[..., :32]) and np.array_equal(got[..., 64:], base[..., 64:])
    _close(got[..., 32:64], ref[..., 32:64])
    f = torch.zeros((B, H, W, cout), dtype=torch.float32, device="cuda")
    _conv(_bf(x), wp, cin, 32, cout, f32=f)
    np.testing.assert_allclose(_np(f), O.conv(x, w), rtol=1e-4, atol=1e-4 * float(np.abs(O.conv(x, w)).max()))
    # Only the first f32_channels channels, densely (stride f32_channels); the
    # buffer's tail past B H W x 4 floats stays untouched.
    f4 = torch.full((B * H * W * 4 + 64,), 5.0, dtype=torch.float32, device="cuda")
    for tr in (0, 1, 2, 4, 8):
        _conv(_bf(x), wp, cin, 32, cout, f32=f4, f32_channels=4, tile_rows=tr)
        got4 = f4[:B * H * W * 4].reshape(B, H, W, 4).cpu().numpy().astype(np.float64)
        np.testing.assert_allclose(got4, O.conv(x, w)[..., :4], rtol=1e-4,
                                   atol=1e-4 * float(np.abs(O.conv(x, w)).max()))
        assert np.all(f4[B * H * W * 4:].cpu().numpy() == 5.0)
    for bad in (6, 48, -4):
        with pytest.raises(N.ArtError):
            _conv(_bf(x), wp, cin, 32, cout, f32=f4, f32_channels=bad)


@pytest.mark.parametrize("tile_rows", [0, 2, 4, 8])
@pytest.mark.parametrize("B,H,W,cin,cout", [(1, 8, 130, 16, 32), (2, 6, 64, 64, 96), (1, 4, 40, 96, 128),
                                            (1, 10, 260, 32, 64)])
def test_conv_fused_pool_and_upsample(gpu, B, H, W, cin, cout, tile_rows):
    """The epilogue's 2x2-pooled output equals pooling the stored activation,
    and the upsampled store equals nearest upsampling of the plain store (the
    upsampled store also with 1-row tiles)."""
    if tile_rows * cout > 256:
        pytest.skip("two tiles' accumulators hold 2 x tile_rows x n TMEM columns: at most 512")
    torch = _torch()
    rng = np.random.default_rng(cin + cout + H)
    x = O.bf16(rng.standard_normal((B, H, W, cin)))
    w = O.bf16(rng.standard_normal((cout, 9, cin)) * np.sqrt(2 / (9 * cin)))
    b = rng.standard_normal(cout) * 0.1
    ck = 32 if cin % 32 == 0 else 16
    wp, xt, bt = _pack(w, ck=ck), _bf(x), _f32(b)
    pooled = torch.zeros((B, H // 2, W // 2, cout), dtype=torch.bfloat16, device="cuda")
    plain = _conv(xt, wp, cin, ck, cout, bias=bt, relu=1, pool_out=pooled, tile_rows=tile_rows)
    ref = O.bf16(np.maximum(O.conv(x, w, b), 0))
    _close(_np(plain), ref)
    np.testing.assert_array_equal(_np(pooled), O.bf16(O.pool(_np(plain))))
    for up_rows in ((tile_rows, 1) if tile_rows == 2 else (tile_rows,)):
        big = torch.zeros((B, 2 * H, 2 * W, cout + 16), dtype=torch.bfloat16, device="cuda")
        _conv(xt, wp, cin, ck, cout, bias=bt, relu=1, out=big, out_cstride=cout + 16, out_coff=16, up2=1,
              tile_rows=up_rows)
        got = _np(big)
        np.testing.assert_array_equal(got[..., 16:], O.up(_np(plain)))
        assert np.all(got[..., :16] == 0)


def test_conv_backward_data_with_mask(gpu):
    rng = np.random.default_rng(9)
    B, H, W, cin, cout = 2, 8, 136, 96, 64
    g = O.bf16(rng.standard_normal((B, H, W, cout)))
    w = O.bf16(rng.standard_normal((cout, 9, cin)) * 0.1)
    act = O.bf16(rng.standard_normal((B, H, W, 32)))
    # Input channels 64..95 only, masked by act > 0.
    got = _np(_conv(_bf(g), _pack(w, transpose=1, ci0=64, n=32), cout, 32, 32, mask=_bf(act)))
    ref = O.bf16(O.conv_dgrad(g, w)[..., 64:96] * (act > 0))
    _close(got, ref)


@pytest.mark.parametrize("B,H,W,cin,cout", [(1, 8, 128, 16, 32), (2, 6, 70, 224, 96), (1, 10, 300, 32, 128),
                                            (3, 4, 40, 64, 16)])
def test_conv_weight_gradient(gpu, B, H, W, cin, cout):
    torch = _torch()
    rng = np.random.default_rng(cin + 3 * cout)
    x = O.bf16(rng.standard_normal((B, H, W, cin)))
    g = O.bf16(rng.standard_normal((B, H, W, cout)))
    dw = torch.zeros(cout * 9 * cin, dtype=torch.float32, device="cuda")
    ws = torch.empty(64 << 20, dtype=torch.uint8, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    d = N.ArtCnnWgrad()
    d.B, d.H, d.W, d.cout, d.cin = B, H, W, cout, cin
    xt, gt = _bf(x), _bf(g)
    d.dy, d.x, d.dw, d.accumulate = gt.data_ptr(), xt.data_ptr(), dw.data_ptr(), 0
    d.workspace, d.workspace_bytes, d.err = ws.data_ptr(), ws.numel(), err.data_ptr()
    N.check(N.lib().art_cnn_wgrad3x3(C.byref(d), None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = O.conv_wgrad(x, g)
    got = dw.cpu().numpy().astype(np.float64).reshape(cout, 9, cin)
    np.testing.assert_allclose(got, ref, rtol=0, atol=2e-5 * float(np.abs(ref).max()) + 1e-5)


def test_memory_kernels(gpu):
    torch = _torch()
    rng = np.random.default_rng(11)
    B, H, W, C = 2, 8, 12, 16
    # Every device input is held in a variable for the duration of its call:
    # a temporary would go back to torch's caching allocator as soon as its
    # pointer is taken, and the next input could be placed in the same memory.
    a = O.bf16(rng.standard_normal((B, H, W, 48)))
    a_d = _bf(a)
    out = torch.empty((B, H // 2, W // 2, C), dtype=torch.bfloat16, device="cuda")
    N.check(N.lib().art_cnn_pool2(_ptr(a_d), B, H, W, C, 48, 16, _ptr(out), None))
    np.testing.assert_array_equal(_np(out), O.bf16(O.pool(a[..., 16:32])))
    lo = O.bf16(rng.standard_normal((B, H // 2, W // 2, C)))
    lo_d = _bf(lo)
    cat = _bf(np.zeros((B, H, W, 32)))
    N.check(N.lib().art_cnn_upsample2(_ptr(lo_d), B, H, W, C, _ptr(cat), 32, 16, None))
    np.testing.assert_array_equal(_np(cat)[..., 16:], O.up(lo))
    g = O.bf16(rng.standard_normal((B, H, W, C)))
    act = O.bf16(rng.standard_normal((B, H // 2, W // 2, C)))
    g_d, act_d = _bf(g), _bf(act)
    ds = torch.empty((B, H // 2, W // 2, C), dtype=torch.bfloat16, device="cuda")
    N.check(N.lib().art_cnn_downsum2_mask(_ptr(g_d), B, H, W, C, _ptr(act_d), _ptr(ds), None))
    np.testing.assert_array_equal(_np(ds), O.bf16(O.downsum(g) * (act > 0)))
    gs = O.bf16(rng.standard_normal((B, H, W, C)))
    gp = O.bf16(rng.standard_normal((B, H // 2, W // 2, C)))
    act2 = O.bf16(rng.standard_normal((B, H, W, 48)))
    gt, gp_d, act2_d = _bf(gs), _bf(gp), _bf(act2)
    N.check(N.lib().art_cnn_unpool_add_mask(_ptr(gt), _ptr(gp_d), B, H, W, C, _ptr(act2_d), 48, 32, None))
    np.testing.assert_array_equal(_np(gt), O.bf16((gs + 0.25 * O.up(gp)) * (act2[..., 32:48] > 0)))


def _batch(seed, B=2, H=64, W=48):
    rng = np.random.default_rng(seed)
    coef = np.zeros((B, H, W), np.int16)
    for b in range(B):  # sparse low-frequency coefficients like a real JPEG
        blk = coef[b].reshape(H // 8, 8, W // 8, 8)
        blk[:, 0, :, 0] = rng.integers(-60, 60, size=(H // 8, W // 8))
        blk[:, :3, :, :3] += rng.integers(-3, 4, size=(H // 8, 3, W // 8, 3)).astype(np.int16)
    q = rng.integers(4, 40, size=(B, 64)).astype(np.float32)
    dec, _ = O.features(coef, q)
    target = (dec + rng.standard_normal(dec.shape) * 3.0).astype(np.float32)
    return coef, q, target


@pytest.mark.parametrize("B,H,W", [(1, 8, 8), (2, 40, 56), (1, 64, 48), (3, 24, 136), (1, 136, 72)])
def test_features_match_oracle(gpu, B, H, W):
    """art_cnn_features on ragged component sizes (padded block grids whose
    rows are not a multiple of the 4 blocks one warp takes): the decoded image
    to fp32 rounding, the quantisation-step channels exactly, zeros in channels
    8-15 and in cells outside the component (the output starts as garbage)."""
    torch = _torch()
    rng = np.random.default_rng(B * 1000 + H * 10 + W)
    coef = np.zeros((B, H, W), np.int16)
    for b in range(B):
        blk = coef[b].reshape(H // 8, 8, W // 8, 8)
        blk[:, 0, :, 0] = rng.integers(-60, 60, size=(H // 8, W // 8))
        blk[:, :4, :, :4] += rng.integers(-5, 6, size=(H // 8, 4, W // 8, 4)).astype(np.int16)
    q = rng.integers(1, 80, size=(B, 64)).astype(np.float32)
    H0, W0 = O.level0(H, W)
    coef_d = torch.from_numpy(coef).cuda()
    q_d = _f32(q)
    dec_d = torch.full((B, H, W), 7.0, dtype=torch.float32, device="cuda")
    feat_d = torch.full((B, H0, W0, 16), 3.0, dtype=torch.bfloat16, device="cuda")
    N.check(N.lib().art_cnn_features(_ptr(coef_d), W, H * W, _ptr(q_d), B, H, W, _ptr(dec_d), _ptr(feat_d), None))
    torch.cuda.synchronize()
    dec_ref, F_ref = O.features(coef, q)
    dec = dec_d.cpu().numpy().astype(np.float64)
    np.testing.assert_allclose(dec, dec_ref, rtol=0, atol=2e-3)
    F = _np(feat_d)
    np.testing.assert_array_equal(F[..., 0:4], O.bf16(O.space_to_depth(dec, H0, W0) / 128.0))
    np.testing.assert_array_equal(F[..., 4:8], O.bf16(F_ref[..., 4:8]))
    assert np.all(F[..., 8:] == 0)


def test_features_and_prediction(gpu):
    torch = _torch()
    coef, q, _ = _batch(1)
    params = WS.init_params(3)
    net = WS.WarmStartNet(params)
    pred = net.predict(torch.from_numpy(coef).cuda(), _f32(q)).cpu().numpy().astype(np.float64)
    dec, F = O.features(coef, q)
    a, ref, _, _ = O.forward(params.astype(np.float64), F, dec)
    np.testing.assert_allclose(pred, ref, rtol=0, atol=2e-3 * max(1.0, float(np.abs(ref - dec).max())) + 1e-3)


def _joint_batch(seed, B=2, H=64, W=96):
    rng = np.random.default_rng(seed)

    def coefs(b, h, w):
        c = np.zeros((b, h, w), np.int16)
        for i in range(b):
            blk = c[i].reshape(h // 8, 8, w // 8, 8)
            blk[:, 0, :, 0] = rng.integers(-60, 60, size=(h // 8, w // 8))
            blk[:, :3, :, :3] += rng.integers(-3, 4, size=(h // 8, 3, w // 8, 3)).astype(np.int16)
        return c

    cy = coefs(B, H, W)
    cc = coefs(2 * B, H // 2, W // 2).reshape(B, 2, H // 2, W // 2)
    qy = rng.integers(4, 40, size=(B, 64)).astype(np.float32)
    qc = rng.integers(4, 40, size=(B, 2, 64)).astype(np.float32)
    dec, _ = O.features_joint(cy, qy, cc, qc)
    target = (dec + rng.standard_normal(dec.shape) * 3.0).astype(np.float32)
    return cy, cc, qy, qc, target


def _joint_params(seed):
    params = WS.init_params(seed)
    rng = np.random.default_rng(seed)
    offs, _ = O.offsets()
    wo, bo = offs["head"]
    params[wo:bo] = (rng.standard_normal(bo - wo) * 0.05).astype(np.float32)
    params[wo + 12 * 32 * 9:bo] = 0.0  # outputs 12-15 are unused by the joint network
    return params


def test_joint_prediction_matches_oracle(gpu):
    """art_net_predict_joint: luma and full-resolution chroma planes against the
    oracle's joint forward pass (bf16 storage emulated)."""
    torch = _torch()
    cy, cc, qy, qc, _ = _joint_batch(6)
    params = _joint_params(6)
    net = WS.WarmStartNet(params)
    pred = net.predict_joint(torch.from_numpy(cy).cuda(), torch.from_numpy(cc).cuda(), _f32(qy), _f32(qc))
    pred = pred.cpu().numpy().astype(np.float64)
    dec, F = O.features_joint(cy, qy, cc, qc)
    _, ref, _, _ = O.forward(params.astype(np.float64), F, dec, joint=True)
    assert pred.shape == ref.shape
    np.testing.assert_allclose(pred, ref, rtol=0, atol=2e-3 * max(1.0, float(np.abs(ref - dec).max())) + 1e-3)


def test_joint_gradients_match_oracle(gpu):
    """art_net_train_step_joint's backward pass against the oracle's FP64
    gradient of the joint loss: per layer cosine >= 0.999, relative <= 3e-2."""
    torch = _torch()
    cy, cc, qy, qc, target = _joint_batch(7)
    params = _joint_params(7)
    net = WS.WarmStartNet(params)
    loss = net.train_step_joint(torch.from_numpy(cy).cuda(), torch.from_numpy(cc).cuda(), _f32(qy), _f32(qc),
                                _f32(target), lr=0.0)
    g = net.gradients().astype(np.float64)
    dec, F = O.features_joint(cy, qy, cc, qc)
    ref_loss, ref = O.gradients(params.astype(np.float64), F, dec, target.astype(np.float64), joint=True)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss, (loss, ref_loss)
    offs, _ = O.offsets()
    for name, cin, cout, _, _ in O.LAYERS:
        for lo, hi in ((offs[name][0], offs[name][1]), (offs[name][1], offs[name][1] + cout)):
            a, b = g[lo:hi], ref[lo:hi]
            nb = float(np.linalg.norm(b))
            if nb == 0:
                assert float(np.abs(a).max()) == 0
                continue
            cos = float(a @ b) / (float(np.linalg.norm(a)) * nb)
            rel = float(np.linalg.norm(a - b)) / nb
            assert cos >= 0.999 and rel <= 3e-2, (name, cos, rel)


def test_joint_geometry_is_checked(gpu):
    torch = _torch()
    net = WS.WarmStartNet(WS.init_params(1))
    cy = torch.zeros((1, 40, 48), dtype=torch.int16, device="cuda")
    cc = torch.zeros((1, 2, 20, 24), dtype=torch.int16, device="cuda")
    q = torch.ones((1, 64), device="cuda")
    with pytest.raises(Exception, match="multiple of 16"):
        net.predict_joint(cy, cc, q, torch.ones((1, 2, 64), device="cuda"))


@pytest.mark.parametrize("smooth", [0.0, 2.0])
def test_network_gradients_match_oracle(gpu, smooth):
    """The full forward + backward on the GPU against the oracle's FP64 backward
    (bf16 storage emulated), with and without the loss's smoothness term: per
    layer, cosine >= 0.999 and relative error <= 3e-2."""
    torch = _torch()
    coef, q, target = _batch(2)
    params = WS.init_params(4)
    rng = np.random.default_rng(4)
    offs, _ = O.offsets()
    wo, bo = offs["head"]
    params[wo:bo] = (rng.standard_normal(bo - wo) * 0.05).astype(np.float32)  # a head that passes gradient
    params[wo + 4 * 32 * 9:bo] = 0.0  # outputs 4-15 are unused (outputs 0-3: the 2x2 cell)
    net = WS.WarmStartNet(params)
    net.set_loss(smooth)
    loss = net.train_step(torch.from_numpy(coef).cuda(), _f32(q), _f32(target), lr=0.0)
    g = net.gradients().astype(np.float64)
    dec, F = O.features(coef, q)
    ref_loss, ref = O.gradients(params.astype(np.float64), F, dec, target.astype(np.float64), smooth=smooth)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss, (loss, ref_loss)
    for name, cin, cout, _, _ in O.LAYERS:
        for lo, hi in ((offs[name][0], offs[name][1]), (offs[name][1], offs[name][1] + cout)):
            a, b = g[lo:hi], ref[lo:hi]
            nb = float(np.linalg.norm(b))
            if nb == 0:
                assert float(np.abs(a).max()) == 0
                continue
            cos = float(a @ b) / (float(np.linalg.norm(a)) * nb)
            rel = float(np.linalg.norm(a - b)) / nb
            assert cos >= 0.999 and rel <= 3e-2, (name, cos, rel)


@pytest.mark.parametrize("lam", [0.02, 0.2])
def test_objective_loss_gradients_match_oracle(gpu, lam):
    """The loss's objective term (art_net_set_objective: the solver's objective
    of the projected prediction) through the whole backward pass, against the
    oracle's FP64 gradient of the same loss: loss within 1e-3, per layer cosine
    >= 0.999 and relative error <= 3e-2."""
    torch = _torch()
    coef, q, target = _batch(5)
    params = WS.init_params(5)
    rng = np.random.default_rng(5)
    offs, _ = O.offsets()
    wo, bo = offs["head"]
    params[wo:bo] = (rng.standard_normal(bo - wo) * 0.05).astype(np.float32)
    params[wo + 4 * 32 * 9:bo] = 0.0
    net = WS.WarmStartNet(params)
    net.set_objective(lam, 0.3, 0.001, 3)
    loss = net.train_step(torch.from_numpy(coef).cuda(), _f32(q), _f32(target), lr=0.0)
    g = net.gradients().astype(np.float64)
    dec, F = O.features(coef, q)
    obj = (lam, coef, q.astype(np.float64)) + O.solver_weights(0.3, 0.001, 3)
    ref_loss, ref = O.gradients(params.astype(np.float64), F, dec, target.astype(np.float64), objective=obj)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss, (loss, ref_loss)
    for name, cin, cout, _, _ in O.LAYERS:
        for lo, hi in ((offs[name][0], offs[name][1]), (offs[name][1], offs[name][1] + cout)):
            a, b = g[lo:hi], ref[lo:hi]
            nb = float(np.linalg.norm(b))
            if nb == 0:
                assert float(np.abs(a).max()) == 0
                continue
            cos = float(a @ b) / (float(np.linalg.norm(a)) * nb)
            rel = float(np.linalg.norm(a - b)) / nb
            assert cos >= 0.999 and rel <= 3e-2, (name, cos, rel)
    net.set_objective(0.0)
    plain = net.train_step(torch.from_numpy(coef).cuda(), _f32(q), _f32(target), lr=0.0)
    assert plain < loss


def test_training_reduces_loss(gpu):
    """A residual the network can represent -- the decoded image smoothed by a
    3x3 box filter, minus itself -- is learned: the loss falls well below its
    starting value (where the prediction is about the decoded image)."""
    torch = _torch()
    coef, q, _ = _batch(3, B=4, H=64, W=64)
    dec, _ = O.features(coef, q)
    pad = np.pad(dec, ((0, 0), (1, 1), (1, 1)), mode="edge")
    target = sum(pad[:, 1 + dy:1 + dy + 64, 1 + dx:1 + dx + 64] for dy in (-1, 0, 1) for dx in (-1, 0, 1)) / 9.0
    net = WS.WarmStartNet(WS.init_params(5))
    c, qq, t = torch.from_numpy(coef).cuda(), _f32(q), _f32(target.astype(np.float32))
    losses = [net.train_step(c, qq, t, lr=2e-3) for _ in range(100)]
    assert all(np.isfinite(losses))
    assert losses[-1] < 0.5 * losses[0], losses[::10]


def test_bounded_wait_gives_up_and_reports(gpu):
    """A pipeline wait on a phase that never completes gives up after its
    limit and reports through the error flag; the context stays usable (a
    convolution right after it is still correct)."""
    import time

    torch = _torch()
    err = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    t0 = time.perf_counter()
    N.check(N.lib().art_cnn_wait_selftest(_ptr(err), 20_000_000, None))
    torch.cuda.synchronize()
    assert int(err.item()) == 1
    assert time.perf_counter() - t0 < 10.0
    rng = np.random.default_rng(12)
    x = O.bf16(rng.standard_normal((1, 4, 64, 16)))
    w = O.bf16(rng.standard_normal((16, 9, 16)) * 0.2)
    got = _np(_conv(_bf(x), _pack(w, ck=16), 16, 16, 16))
    _close(got, O.bf16(O.conv(x, w)))
