"""CPU FP64 oracle of the warm-start network (test infrastructure only).

The network has no counterpart in the reference (it only chooses where the
solver starts); this module is the checker for the project's tensor-core
forward and backward kernels. Only tests import it.

It restates the network independently of the CUDA code. The network runs on
a half-resolution grid ("level 0", H0 x W0 = ceil(H / 16) * 8 x ceil(W / 16) * 8):
each level-0 pixel carries a 2x2 cell of the component (space to depth).

  e1 = relu(conv(F, 16 -> 32))                       level 0
  e2 = relu(conv(pool(e1), 32 -> 64))                level 1
  e3 = relu(conv(pool(e2), 64 -> 96))                level 2
  e4 = relu(conv(pool(e3), 96 -> 128))               level 3
  d3 = relu(conv([e3 | up(e4)], 224 -> 96))         level 2
  d2 = relu(conv([e2 | up(d3)], 160 -> 64))         level 1
  d1 = relu(conv([e1 | up(d2)], 96 -> 32))          level 0
  r  = depth_to_space(conv(d1, 32 -> 16)[..., 0:4]) cropped to H x W
  prediction = decoded + 16 r, e = r - (target - decoded) / 16,
  loss = (sum e^2 + smooth * sum over adjacent sample pairs (e_p - e_q)^2) / n
         [+ lam * E(proj(prediction)) / n, the objective term, see objective_value]

conv = 3x3, stride 1, zero padding 1, weights W[cout][tap = 3 (dy+1) + (dx+1)][cin];
pool = 2x2 mean; up = nearest 2x. F = (space_to_depth(decoded) / 128,
space_to_depth(q) / 64, 0 x 8) with q the quantisation step of each sample's
frequency position; channel 2 dy + dx of a level-0 pixel (y, x) is sample
(2y + dy, 2x + dx), zero outside the component.

With ``bf16=True`` every tensor the GPU stores in bf16 is rounded to bf16
(round to nearest even) at the same point, so the only remaining difference
from the GPU is the order of its fp32 accumulations.
"""
from __future__ import annotations

import numpy as np

LAYERS = [  # name, cin, cout, relu, skip channels
    ("e1", 16, 32, True, 0), ("e2", 32, 64, True, 0), ("e3", 64, 96, True, 0), ("e4", 96, 128, True, 0),
    ("d3", 224, 96, True, 96), ("d2", 160, 64, True, 64), ("d1", 96, 32, True, 32), ("head", 32, 16, False, 0),
]


def offsets():
    """(name -> (weight offset, bias offset)) in the flat parameter array."""
    off, out = 0, {}
    for name, cin, cout, _, _ in LAYERS:
        out[name] = (off, off + cout * 9 * cin)
        off += cout * 9 * cin + cout
    return out, off


def unpack(params):
    offs, total = offsets()
    assert params.size == total
    res = {}
    for name, cin, cout, _, _ in LAYERS:
        wo, bo = offs[name]
        res[name] = (params[wo:wo + cout * 9 * cin].reshape(cout, 9, cin).astype(np.float64),
                     params[bo:bo + cout].astype(np.float64))
    return res


def bf16(x):
    """Round to bfloat16 (nearest even) and return as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + ((u >> 16) & 1) + 0x7FFF) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _shifted(x, dy, dx):
    """x[b, y + dy, x + dx, c] with zeros outside."""
    B, H, W, C = x.shape
    p = np.zeros((B, H + 2, W + 2, C), np.float64)
    p[:, 1:H + 1, 1:W + 1] = x
    return p[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W]


def conv(x, w, b=None):
    out = 0.0
    for tap in range(9):
        out = out + np.einsum("bhwc,oc->bhwo", _shifted(x, tap // 3 - 1, tap % 3 - 1), w[:, tap, :], optimize=True)
    return out if b is None else out + b


def conv_dgrad(g, w):
    """Gradient with respect to the input of conv(x, w) given the output gradient g."""
    wt = np.transpose(w[:, ::-1, :], (2, 1, 0))  # [cin][tap'][cout] = w[cout][8 - tap'][cin]
    return conv(g, wt)


def conv_wgrad(x, g):
    cout, cin = g.shape[-1], x.shape[-1]
    dw = np.zeros((cout, 9, cin))
    for tap in range(9):
        dw[:, tap, :] = np.einsum("bhwo,bhwc->oc", g, _shifted(x, tap // 3 - 1, tap % 3 - 1), optimize=True)
    return dw


def pool(x):
    B, H, W, C = x.shape
    return x.reshape(B, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2)


def downsum(g):
    B, H, W, C = g.shape
    return g.reshape(B, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


def _dct_matrix():
    k = np.arange(8)
    m = np.sqrt(2 / 8) * np.cos(np.pi * (2 * k[None, :] + 1) * k[:, None] / 16)
    m[0] /= np.sqrt(2)
    return m  # m[u][x]


def level0(H, W):
    """Size of the network's first level for an H x W component."""
    return (H + 15) // 16 * 8, (W + 15) // 16 * 8


def space_to_depth(a, H0, W0):
    """[B][H][W] -> [B][H0][W0][4], zero-padded to 2 H0 x 2 W0; channel 2 dy + dx."""
    B, H, W = a.shape
    p = np.zeros((B, 2 * H0, 2 * W0))
    p[:, :H, :W] = a
    return p.reshape(B, H0, 2, W0, 2).transpose(0, 1, 3, 2, 4).reshape(B, H0, W0, 4)


def depth_to_space(r, H, W):
    """[B][H0][W0][4] -> [B][H][W] (inverse of space_to_depth, cropped)."""
    B, H0, W0, _ = r.shape
    return r.reshape(B, H0, W0, 2, 2).transpose(0, 1, 3, 2, 4).reshape(B, 2 * H0, 2 * W0)[:, :H, :W]


def features(coef_img, q):
    """coef_img [B][H][W] (coefficient (v,u) of block (bx,by) at (8by+v, 8bx+u)), q [B][64].
    Returns decoded [B][H][W] (fp64) and F [B][H0][W0][16]."""
    m = _dct_matrix()
    B, H, W = coef_img.shape
    c = coef_img.reshape(B, H // 8, 8, W // 8, 8).transpose(0, 1, 3, 2, 4).astype(np.float64)
    qq = q.reshape(B, 1, 1, 8, 8).astype(np.float64)
    blocks = np.einsum("vy,bijvu,ux->bijyx", m, c * qq, m)
    dec = blocks.transpose(0, 1, 3, 2, 4).reshape(B, H, W)
    qt = np.tile(q.reshape(B, 8, 8), (1, H // 8, W // 8)).astype(np.float64)
    H0, W0 = level0(H, W)
    F = np.zeros((B, H0, W0, 16))
    F[..., 0:4] = space_to_depth(dec, H0, W0) / 128.0
    F[..., 4:8] = space_to_depth(qt, H0, W0) / 64.0
    return dec, F


def smooth_up2(c):
    """[..., h, w] -> [..., 2h, 2w]: along each axis sample 2 i + d = 3/4 of
    cell i + 1/4 of cell i - 1 (d = 0) or i + 1 (d = 1), clamped at the edges,
    horizontal first (the learned start's chroma upsampling)."""
    h, w = c.shape[-2:]
    i = np.arange(2 * w)
    cx = i // 2
    nx = np.where(i & 1, np.minimum(cx + 1, w - 1), np.maximum(cx - 1, 0))
    r = 0.75 * c[..., :, cx] + 0.25 * c[..., :, nx]
    j = np.arange(2 * h)
    cy = j // 2
    ny = np.where(j & 1, np.minimum(cy + 1, h - 1), np.maximum(cy - 1, 0))
    return 0.75 * r[..., cy, :] + 0.25 * r[..., ny, :]


def features_joint(coef_y, q_y, coef_c, q_c):
    """Joint 4:2:0 input: coef_y [B][H][W], q_y [B][64], coef_c [B][2][H/2][W/2],
    q_c [B][2][64] (H, W multiples of 16). Returns dec [3][B][H][W] (the decoded
    luma, then the decoded chroma upsampled by smooth_up2: the bases the
    residuals are added to) and F [B][H/2][W/2][16]: the luma's features plus
    channels 8 / 10 = decoded Cb / Cr sample / 128 and 9 / 11 = its step / 64."""
    B, H, W = coef_y.shape
    decY, F = features(coef_y, q_y)
    decC, _ = features(coef_c.reshape(2 * B, H // 2, W // 2), np.asarray(q_c).reshape(2 * B, 64))
    decC = decC.reshape(B, 2, H // 2, W // 2)
    for k in range(2):
        qt = np.tile(np.asarray(q_c)[:, k].reshape(B, 8, 8), (1, H // 16, W // 16)).astype(np.float64)
        F[..., 8 + 2 * k] = decC[:, k] / 128.0
        F[..., 9 + 2 * k] = qt / 64.0
    dec = np.stack([decY, smooth_up2(decC[:, 0]), smooth_up2(decC[:, 1])])
    return dec, F


def project(pred, coef_img, q):
    """Per 8x8 block of pred [B][H][W]: orthonormal DCT, clamp to
    [(c - 1/2) q, (c + 1/2) q], inverse DCT (pipeline_scalar/compute_projection.rs:8-122
    on one component at its own resolution). Returns x, the clamped
    coefficients minus c q over q^2 (block layout [B][by][bx][v][u]) and the
    mask of unclamped coefficients."""
    m = _dct_matrix()
    B, H, W = pred.shape
    blk = pred.reshape(B, H // 8, 8, W // 8, 8).transpose(0, 1, 3, 2, 4)
    C = np.einsum("vy,bijyx,ux->bijvu", m, blk, m)
    c = coef_img.reshape(B, H // 8, 8, W // 8, 8).transpose(0, 1, 3, 2, 4).astype(np.float64)
    qq = q.reshape(B, 1, 1, 8, 8).astype(np.float64)
    Cc = np.clip(C, (c - 0.5) * qq, (c + 0.5) * qq)
    inv = lambda a: np.einsum("vy,bijvu,ux->bijyx", m, a, m).transpose(0, 1, 3, 2, 4).reshape(B, H, W)
    return inv(Cc), (Cc - c * qq) / (qq * qq), Cc == C, inv


def objective_value(x, d, qq_d_cq, a_tv, a_tgv, a_p):
    """The solver's objective of one channel at x: a_tv sum |grad x|
    (compute_step_tv.rs:29-93) + a_tgv sum of the second-order norm
    (compute_step_tv2.rs:32-136) + a_p sum (DCT(x) - c q)^2 / (2 q^2)
    (compute_step_prob.rs:5-60), with the reference's edge rules: forward
    differences vanish on the last column / row, backward ones on the first.
    d = (cos - c q) / q^2 and qq_d_cq = cos - c q per coefficient.
    Returns the value and the terms the gradient needs."""
    dX = np.zeros_like(x)
    dX[:, :, :-1] = x[:, :, 1:] - x[:, :, :-1]
    dY = np.zeros_like(x)
    dY[:, :-1, :] = x[:, 1:, :] - x[:, :-1, :]
    xx = np.zeros_like(x)
    xx[:, :, 1:] = dX[:, :, 1:] - dX[:, :, :-1]
    gyx = np.zeros_like(x)
    gyx[:, :, 1:] = dY[:, :, 1:] - dY[:, :, :-1]
    yy = np.zeros_like(x)
    yy[:, 1:, :] = dY[:, 1:, :] - dY[:, :-1, :]
    gxy = np.zeros_like(x)
    gxy[:, 1:, :] = dX[:, 1:, :] - dX[:, :-1, :]
    s = 0.5 * (gxy + gyx)
    n1 = np.sqrt(dX * dX + dY * dY)
    n2 = np.sqrt(yy * yy + 2 * s * s + xx * xx)
    value = float(a_tv * n1.sum() + a_tgv * n2.sum() + 0.5 * a_p * np.sum(d * qq_d_cq))
    with np.errstate(divide="ignore", invalid="ignore"):
        i1 = np.where(n1 > 0, a_tv / n1, 0.0)
        i2 = np.where(n2 > 0, a_tgv / n2, 0.0)
    return value, (i1 * dX, i1 * dY, i2 * xx, i2 * yy, i2 * s)


def objective_gradient(T):
    """d E / d x from the terms: the reference's scatter of each term centred
    on a sample to its neighbours (compute_step_tv.rs:64-88,
    compute_step_tv2.rs:106-134), without the DCT-distance part."""
    T0, T1, T2, T3, T4 = T
    g = -(T0 + T1) - 2 * (T3 + T2 + T4)
    g[:, :, 1:] += T0[:, :, :-1] + T4[:, :, :-1] + T2[:, :, :-1]
    g[:, 1:, :] += T1[:, :-1, :] + T3[:, :-1, :] + T4[:, :-1, :]
    g[:, :, :-1] += T4[:, :, 1:] + T2[:, :, 1:]
    g[:, :-1, :] += T3[:, 1:, :] + T4[:, 1:, :]
    g[:, :-1, 1:] -= T4[:, 1:, :-1]
    g[:, 1:, :-1] -= T4[:, :-1, 1:]
    return g


def objective_and_back(pred, coef_img, q, a_tv, a_tgv, a_p):
    """E(proj(pred)) and its gradient with respect to pred through the
    projection: J^T grad E with J = IDCT diag(mask) DCT (= J^T)."""
    m = _dct_matrix()
    B, H, W = pred.shape
    x, d, mask, inv = project(pred, coef_img, q)
    qq = q.reshape(B, 1, 1, 8, 8).astype(np.float64)
    value, T = objective_value(x, d, d * qq * qq, a_tv, a_tgv, a_p)
    g = objective_gradient(T) + a_p * inv(d)
    gb = g.reshape(B, H // 8, 8, W // 8, 8).transpose(0, 1, 3, 2, 4)
    G = np.einsum("vy,bijyx,ux->bijvu", m, gb, m) * mask
    return value, inv(G)


def solver_weights(weight=0.3, pweight=0.001, nch=3):
    """(a_tv, a_tgv, a_p) of the solver for an nch-channel image (compute_step.rs:8-72)."""
    r = 1.0 / np.sqrt(nch)
    return r, weight * r, pweight * 2.0 * 255.0 * np.sqrt(2.0)


def _pair_sum(e):
    """Sum over horizontally and vertically adjacent samples of (e_p - e_q)^2."""
    return float(np.sum((e[:, :, 1:] - e[:, :, :-1]) ** 2) + np.sum((e[:, 1:, :] - e[:, :-1, :]) ** 2))


def _pair_grad(e):
    """d/de_p of the pair sum: 2 sum over the neighbours q of p of (e_p - e_q)."""
    g = np.zeros_like(e)
    dx = e[:, :, 1:] - e[:, :, :-1]
    dy = e[:, 1:, :] - e[:, :-1, :]
    g[:, :, 1:] += 2 * dx
    g[:, :, :-1] -= 2 * dx
    g[:, 1:, :] += 2 * dy
    g[:, :-1, :] -= 2 * dy
    return g


def forward(params, F, dec, target=None, bf=True, smooth=0.0, objective=None, joint=False):
    """Activations (dict), prediction and, with a target, the loss.
    objective = (lam, coef_img, q, a_tv, a_tgv, a_p) adds the objective term
    (and replaces the smoothness term, as the GPU does). joint: dec and
    target are [3][B][H][W] and head outputs 4 c .. 4 c + 3 are component c's
    2x2 full-resolution cells (the joint 4:2:0 network)."""
    rnd = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    P = unpack(params)
    Wq = {k: (rnd(w), b) for k, (w, b) in P.items()}
    a = {"F": rnd(F)}
    relu = lambda v: np.maximum(v, 0.0)
    a["e1"] = rnd(relu(conv(a["F"], *Wq["e1"])))
    a["p1"] = rnd(pool(a["e1"]))
    a["e2"] = rnd(relu(conv(a["p1"], *Wq["e2"])))
    a["p2"] = rnd(pool(a["e2"]))
    a["e3"] = rnd(relu(conv(a["p2"], *Wq["e3"])))
    a["p3"] = rnd(pool(a["e3"]))
    a["e4"] = rnd(relu(conv(a["p3"], *Wq["e4"])))
    a["cat3"] = np.concatenate([a["e3"], up(a["e4"])], axis=-1)
    a["d3"] = rnd(relu(conv(a["cat3"], *Wq["d3"])))
    a["cat2"] = np.concatenate([a["e2"], up(a["d3"])], axis=-1)
    a["d2"] = rnd(relu(conv(a["cat2"], *Wq["d2"])))
    a["cat1"] = np.concatenate([a["e1"], up(a["d2"])], axis=-1)
    a["d1"] = rnd(relu(conv(a["cat1"], *Wq["d1"])))
    r = conv(a["d1"], *Wq["head"])
    if bf:
        r = r.astype(np.float32).astype(np.float64)
    a["r"] = r
    H, W = dec.shape[-2:]
    if joint:
        rf = np.stack([depth_to_space(r[..., 4 * c:4 * c + 4], H, W) for c in range(3)])
    else:
        rf = depth_to_space(r[..., 0:4], H, W)
    pred = dec + 16.0 * rf
    loss = None
    if target is not None:
        e = rf - (target - dec) / 16.0
        a["e"] = e
        if objective is not None:
            lam, coef_img, q, a_tv, a_tgv, a_p = objective
            val, dpred = objective_and_back(pred, coef_img, q, a_tv, a_tgv, a_p)
            loss = float(np.mean(e * e)) + lam * val / e.size
            a["obj_grad"] = lam * 16.0 * dpred
        else:
            loss = float(np.mean(e * e)) + smooth * _pair_sum(e) / e.size
    return a, pred, loss, Wq


def gradients(params, F, dec, target, bf=True, smooth=0.0, objective=None, joint=False):
    """Loss and d loss / d params (flat, same layout as params)."""
    rnd = bf16 if bf else (lambda v: np.asarray(v, np.float64))
    a, _, loss, Wq = forward(params, F, dec, target, bf, smooth, objective, joint)
    npix = dec.size
    mask = lambda g, act: g * (act > 0)
    dr = np.zeros(a["r"].shape)
    if joint:
        for c in range(3):
            dr[..., 4 * c:4 * c + 4] = space_to_depth(2.0 * a["e"][c] / npix, *a["r"].shape[1:3])
        if bf:
            dr[..., 0:12] = bf16(dr[..., 0:12].astype(np.float32))
    else:
        if objective is not None:
            dlde = (2.0 * a["e"] + a["obj_grad"]) / npix
        else:
            dlde = (2.0 * a["e"] + smooth * _pair_grad(a["e"])) / npix
        dr[..., 0:4] = space_to_depth(dlde, *a["r"].shape[1:3])
        if bf:
            dr[..., 0:4] = bf16(dr[..., 0:4].astype(np.float32))
    grads = {}

    def wb(name, x, g):
        grads[name] = (conv_wgrad(x, g), g.sum(axis=(0, 1, 2)))

    wb("head", a["d1"], dr)
    gd1 = rnd(mask(conv_dgrad(dr, Wq["head"][0]), a["d1"]))
    wb("d1", a["cat1"], gd1)
    w = Wq["d1"][0]
    ge1 = rnd(conv_dgrad(gd1, w[:, :, :32]))
    gd2 = rnd(mask(downsum(rnd(conv_dgrad(gd1, w[:, :, 32:]))), a["d2"]))
    wb("d2", a["cat2"], gd2)
    w = Wq["d2"][0]
    ge2 = rnd(conv_dgrad(gd2, w[:, :, :64]))
    gd3 = rnd(mask(downsum(rnd(conv_dgrad(gd2, w[:, :, 64:]))), a["d3"]))
    wb("d3", a["cat3"], gd3)
    w = Wq["d3"][0]
    ge3 = rnd(conv_dgrad(gd3, w[:, :, :96]))
    ge4 = rnd(mask(downsum(rnd(conv_dgrad(gd3, w[:, :, 96:]))), a["e4"]))
    wb("e4", a["p3"], ge4)
    gp3 = rnd(conv_dgrad(ge4, Wq["e4"][0]))
    ge3 = rnd(mask(ge3 + 0.25 * up(gp3), a["e3"]))
    wb("e3", a["p2"], ge3)
    gp2 = rnd(conv_dgrad(ge3, Wq["e3"][0]))
    ge2 = rnd(mask(ge2 + 0.25 * up(gp2), a["e2"]))
    wb("e2", a["p1"], ge2)
    gp1 = rnd(conv_dgrad(ge2, Wq["e2"][0]))
    ge1 = rnd(mask(ge1 + 0.25 * up(gp1), a["e1"]))
    wb("e1", a["F"], ge1)
    offs, total = offsets()
    flat = np.zeros(total)
    for name, cin, cout, _, _ in LAYERS:
        wo, bo = offs[name]
        flat[wo:wo + cout * 9 * cin] = grads[name][0].ravel()
        flat[bo:bo + cout] = grads[name][1]
    return loss, flat
