"""Second restatement of pipeline_scalar in numpy fp32 -- TEST INFRASTRUCTURE.

An independent transliteration of Delnegend/artefact's default solver
(backend/artefact-lib/pipeline_scalar), written from the Rust line by line
and vectorised over pixels and blocks, used only to cross-check the C oracle
(oracle/oracle_body.inc): the two must agree bit for bit in fp32. Every
operation keeps the reference's operand order and rounding:

  * mul_add!(a, b, c) is a * b + c, two roundings (utils/macros.rs:9-13, the
    default build without the "native" feature);
  * f32::midpoint(a, b) is the f64 mean rounded to f32;
  * the gradient norm is a sequential f32 fold (compute_step.rs:52-58), here
    np.add.accumulate, which adds strictly in order;
  * every gradient element receives its contributions in the reference's
    order: the DCT-distance term (compute_step_prob.rs:5-60), then the TV
    scatter of its source pixels in raster order (compute_step_tv.rs:29-93),
    then the TGV scatter likewise (compute_step_tv2.rs:32-136). A vectorised
    pass adds, for all targets at once, the contribution of one source offset,
    in the order the raster loop reaches those sources.

The start is the decoded image (block IDCT of c q, one unboxing, nearest
upsampling: pipeline_simd_adaptive/coef.rs:69-95 with
pipeline_scalar/coef.rs:69-92), the oracle's init mode 0.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np

F = np.float32
# utils/dct.rs:19-27 (Ooura's shrtdct.c constants).
C8_1R, C8_1I = F(0.49039264020161522456), F(0.09754516100806413392)
C8_2R, C8_2I = F(0.46193976625564337806), F(0.19134171618254488586)
C8_3R, C8_3I = F(0.41573480615127261854), F(0.27778511650980111237)
C8_4R = F(0.35355339059327376220)
W8_4R = F(0.70710678118654752440)


def _idct8(a):
    """One 1-D pass of idct8x8s (utils/dct.rs:30-67) on 8 arrays."""
    x1r = C8_1R * a[1] + C8_1I * a[7]
    x1i = C8_1R * a[7] + (-(C8_1I * a[1]))
    x3r = C8_3R * a[3] + C8_3I * a[5]
    x3i = C8_3R * a[5] + (-(C8_3I * a[3]))
    xr = x1r - x3r
    xi = x1i + x3i
    x1r = x1r + x3r
    x3i = x3i - x1i
    x1i = W8_4R * (xr + xi)
    x3r = W8_4R * (xr - xi)
    xr = C8_2R * a[2] + C8_2I * a[6]
    xi = C8_2R * a[6] + (-(C8_2I * a[2]))
    x0r = C8_4R * (a[0] + a[4])
    x0i = C8_4R * (a[0] - a[4])
    x2r = x0r - xr
    x2i = x0i - xi
    x0r = x0r + xr
    x0i = x0i + xi
    return [x0r + x1r, x2i + x3r, x0i + x1i, x2r + x3i, x2r - x3i, x0i - x1i, x2i - x3r, x0r - x1r]


def _dct8(a):
    """One 1-D pass of dct8x8s (utils/dct.rs:105-169) on 8 arrays."""
    x0r = a[0] + a[7]
    x1r = a[0] - a[7]
    x0i = a[2] + a[5]
    x1i = a[2] - a[5]
    x2r = a[4] + a[3]
    x3r = a[4] - a[3]
    x2i = a[6] + a[1]
    x3i = a[6] - a[1]
    xr = x0r + x2r
    xi = x0i + x2i
    o0 = C8_4R * (xr + xi)
    o4 = C8_4R * (xr - xi)
    xr = x0r - x2r
    xi = x0i - x2i
    o2 = C8_2R * xr + (-(C8_2I * xi))
    o6 = C8_2R * xi + C8_2I * xr
    xr = W8_4R * (x1i - x3i)
    x1i = W8_4R * (x1i + x3i)
    x3i = x1i - x3r
    x1i = x1i + x3r
    x3r = x1r - xr
    x1r = x1r + xr
    o1 = C8_1R * x1r + (-(C8_1I * x1i))
    o7 = C8_1R * x1i + C8_1I * x1r
    o3 = C8_3R * x3r + (-(C8_3I * x3i))
    o5 = C8_3R * x3i + C8_3I * x3r
    return [o0, o1, o2, o3, o4, o5, o6, o7]


def _separable(blocks: np.ndarray, pass_fn) -> np.ndarray:
    """Columns first (a[k * 8 + j] over k), then rows, as dct8x8s / idct8x8s."""
    cols = pass_fn([blocks[..., k, :] for k in range(8)])
    a = np.stack(cols, axis=-2)
    rows = pass_fn([a[..., :, k] for k in range(8)])
    return np.stack(rows, axis=-1)


def dct8x8(blocks: np.ndarray) -> np.ndarray:
    return _separable(np.asarray(blocks, F), _dct8)


def idct8x8(blocks: np.ndarray) -> np.ndarray:
    return _separable(np.asarray(blocks, F), _idct8)


def _box(plane: np.ndarray, bh: int, bw: int) -> np.ndarray:
    """Raster plane -> blocks (utils/boxing.rs:56-84): [bh, bw, 8, 8]."""
    return plane.reshape(bh, 8, bw, 8).transpose(0, 2, 1, 3)


def _unbox(blocks: np.ndarray) -> np.ndarray:
    """Blocks -> raster plane (utils/boxing.rs:8-47)."""
    bh, bw = blocks.shape[:2]
    return np.ascontiguousarray(blocks.transpose(0, 2, 1, 3)).reshape(bh * 8, bw * 8)


def _midpoint(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return ((a.astype(np.float64) + b.astype(np.float64)) / 2.0).astype(F)


class _Channel:
    def __init__(self, co):
        self.cw, self.ch = int(co.rounded_px_w), int(co.rounded_px_h)
        self.bw, self.bh = int(co.block_w), int(co.block_h)
        self.sh, self.sv = int(co.horizontal_samp_factor), int(co.vertical_samp_factor)
        self.q = np.asarray(co.quant_table, F).reshape(8, 8)
        self.c = np.asarray(co.dct_coefs).astype(F).reshape(self.bh, self.bw, 8, 8)
        self.cq = self.c * self.q  # coef.rs:94-104 (get_cos), the first cos
        self.lo = (self.c - F(0.5)) * self.q  # compute_projection.rs:72-79
        self.hi = (self.c + F(0.5)) * self.q


def _scatter(g: np.ndarray, contrib: np.ndarray, mask: np.ndarray, tgt, src) -> None:
    """g[tgt] += contrib[src] where mask[src] (a no-op where the norm is 0)."""
    g[tgt] = np.where(mask[src], g[tgt] + contrib[src], g[tgt])


def compute(nch: int, coefs, weight: float, pweight: Sequence[float], iterations: int, W: int, H: int
            ) -> List[np.ndarray]:
    """pipeline_scalar::compute (mod.rs:17-78) from the decoded start: nch
    fp32 planes of W * H values."""
    chans = [_Channel(c) for c in coefs[:nch]]
    weight = F(weight)
    pw = [F(p) for p in (list(pweight) + [0.0] * 3)[:3]]
    # Start (aux.rs:51-63): fdata = fista = nearest-upsampled decoded image.
    fdata = []
    for cd in chans:
        img = _unbox(idct8x8(cd.c * cd.q))
        ys = np.minimum(np.arange(H) // cd.sv, cd.ch - 1)
        xs = np.minimum(np.arange(W) // cd.sh, cd.cw - 1)
        fdata.append(np.ascontiguousarray(img[ys][:, xs]))
    fista = [f.copy() for f in fdata]
    cos = [cd.cq.copy() for cd in chans]
    radius = np.sqrt(F(W * H)) / F(2.0)
    step = radius / np.sqrt(F(1.0) + F(iterations))
    term = F(1.0)
    alpha_tv = F(1.0) / np.sqrt(F(nch))
    alpha_tgv = (weight / np.sqrt(F(2.0))) / np.sqrt(F(nch))
    for _ in range(iterations):
        # FISTA (mod.rs:49-61).
        nxt = _midpoint(np.array(1.0, F), np.sqrt(F(4.0) * (term * term) + F(1.0)))
        factor = (term - F(1.0)) / nxt
        for c in range(nch):
            fista[c] = factor * (fdata[c] - fista[c]) + fdata[c]
            fdata[c], fista[c] = fista[c], fdata[c]
        term = F(nxt)
        # DCT-distance gradient (compute_step.rs:19-35, compute_step_prob.rs:5-60).
        grads = []
        for c, cd in enumerate(chans):
            g = np.zeros((H, W), F)
            if pw[c] != 0.0:
                alpha = ((pw[c] * F(2.0)) * F(255.0)) * np.sqrt(F(2.0))
                d = (cos[c] - cd.c * cd.q) / (cd.q * cd.q)
                p = _unbox(idct8x8(d))
                for sy in range(cd.sv):
                    for sx in range(cd.sh):
                        g[sy::cd.sv, sx::cd.sh] = g[sy::cd.sv, sx::cd.sh] + alpha * p
            grads.append(g)
        # TV (compute_step_tv.rs:29-93): forward differences, coupled norm.
        gx = [np.zeros((H, W), F) for _ in range(nch)]
        gy = [np.zeros((H, W), F) for _ in range(nch)]
        n1 = np.zeros((H, W), F)
        for c in range(nch):
            gx[c][:, :-1] = fdata[c][:, 1:] - fdata[c][:, :-1]
            gy[c][:-1, :] = fdata[c][1:, :] - fdata[c][:-1, :]
        for c in range(nch):
            n1 = n1 + gx[c] * gx[c]
            n1 = n1 + gy[c] * gy[c]
        n1 = np.sqrt(n1)
        m1 = n1 != 0
        with np.errstate(divide="ignore", invalid="ignore"):
            for c in range(nch):
                cen = (alpha_tv * (-(gx[c] + gy[c]))) / n1
                right = (alpha_tv * gx[c]) / n1
                below = (alpha_tv * gy[c]) / n1
                g = grads[c]
                # Sources of target q in raster order: q - W (below), q - 1 (right), q.
                _scatter(g, below, m1, (slice(1, None), slice(None)), (slice(None, -1), slice(None)))
                _scatter(g, right, m1, (slice(None), slice(1, None)), (slice(None), slice(None, -1)))
                _scatter(g, cen, m1, (slice(None), slice(None)), (slice(None), slice(None)))
        # TGV (compute_step_tv2.rs:32-136): backward differences of the
        # forward differences, symmetrised, coupled norm.
        gxx, gyy, gs = [], [], []
        n2 = np.zeros((H, W), F)
        for c in range(nch):
            axx = np.zeros((H, W), F)
            ayx = np.zeros((H, W), F)
            ayy = np.zeros((H, W), F)
            axy = np.zeros((H, W), F)
            axx[:, 1:] = gx[c][:, 1:] - gx[c][:, :-1]
            ayx[:, 1:] = gy[c][:, 1:] - gy[c][:, :-1]
            ayy[1:, :] = gy[c][1:, :] - gy[c][:-1, :]
            axy[1:, :] = gx[c][1:, :] - gx[c][:-1, :]
            s = _midpoint(axy, ayx)
            gxx.append(axx)
            gyy.append(ayy)
            gs.append(s)
        for c in range(nch):
            n2 = n2 + (gyy[c] * gyy[c] + (F(2.0) * (gs[c] * gs[c]) + gxx[c] * gxx[c]))
        n2 = np.sqrt(n2)
        m2 = n2 != 0
        A = slice(None)
        with np.errstate(divide="ignore", invalid="ignore"):
            for c in range(nch):
                s, xx, yy = gs[c], gxx[c], gyy[c]
                cen = alpha_tgv * ((-(F(2.0) * yy + (F(2.0) * xx + F(2.0) * s))) / n2)
                lr = alpha_tgv * ((s + xx) / n2)
                ud = alpha_tgv * ((yy + s) / n2)
                dg = alpha_tgv * ((-s) / n2)
                g = grads[c]
                # Sources of target q in raster order: q - W (down term),
                # q - W + 1 (down-left), q - 1 (right), q, q + 1 (left),
                # q + W - 1 (up-right), q + W (up).
                _scatter(g, ud, m2, (slice(1, None), A), (slice(None, -1), A))
                _scatter(g, dg, m2, (slice(1, None), slice(None, -1)), (slice(None, -1), slice(1, None)))
                _scatter(g, lr, m2, (A, slice(1, None)), (A, slice(None, -1)))
                _scatter(g, cen, m2, (A, A), (A, A))
                _scatter(g, lr, m2, (A, slice(None, -1)), (A, slice(1, None)))
                _scatter(g, dg, m2, (slice(None, -1), slice(1, None)), (slice(1, None), slice(None, -1)))
                _scatter(g, ud, m2, (slice(None, -1), A), (slice(1, None), A))
        # Normalised step (compute_step.rs:52-66): sequential fp32 fold.
        for c in range(nch):
            g = grads[c].ravel()
            norm = np.sqrt(np.add.accumulate(g * g, dtype=F)[-1])
            if norm != 0.0:
                fdata[c] = (fdata[c].ravel() - step * (g / norm)).reshape(H, W)
        # Projection (compute_projection.rs:8-122).
        for c, cd in enumerate(chans):
            f = fdata[c]
            resample = cd.cw != W or cd.ch != H
            if resample:
                mean = np.zeros((cd.ch, cd.cw), F)
                for sy in range(cd.sv):
                    for sx in range(cd.sh):
                        mean = mean + f[sy::cd.sv, sx::cd.sh]
                mean = mean / F(cd.sh * cd.sv)
                for sy in range(cd.sv):
                    for sx in range(cd.sh):
                        f[sy::cd.sv, sx::cd.sh] = f[sy::cd.sv, sx::cd.sh] - mean
                src = mean
            else:
                src = f
            X = dct8x8(_box(src, cd.bh, cd.bw))
            # f32::clamp: below min -> min, then above max -> max.
            X = np.where(X < cd.lo, cd.lo, X)
            X = np.where(X > cd.hi, cd.hi, X)
            cos[c] = X.copy()
            back = _unbox(idct8x8(X))
            if resample:
                for sy in range(cd.sv):
                    for sx in range(cd.sh):
                        f[sy::cd.sv, sx::cd.sh] = f[sy::cd.sv, sx::cd.sh] + back
                fdata[c] = f
            else:
                fdata[c] = back
    return [np.ascontiguousarray(f).ravel() for f in fdata]
