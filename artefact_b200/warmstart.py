"""Learned warm start for the restoration solver.

A 4-level encoder-decoder CNN predicts, per channel, the converged solver
output from the decoded channel and its quantisation table. It runs at half
the component's resolution: each first-level pixel carries a 2x2 cell of
samples (space to depth), and the head's first four outputs are the cell's
residuals. Its forward and
backward passes are the library's own sm_100a kernels (``art_net_*`` /
``art_cnn_*`` in libartefact_b200.so: tcgen05 MMAs with TMEM accumulators,
TMA-staged tiles); PyTorch only provides device memory and streams here.

The solver uses a prediction as its starting point (``ART_INIT_LEARNED``):
the prediction is projected onto the quantisation constraint set and refined
by plain iterations, so the constraint and the objective stay the
reference's. Training pairs come from the plain solver itself (targets: long
plain runs of the same synthetic JPEGs).

Weights file: 8-byte magic ``ARTWS001``, int64 parameter count, then that
many little-endian float32 values (per layer e1, e2, e3, e4, d3, d2, d1,
head: weights [cout][9][cin], then bias [cout]).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path
from typing import Optional

import numpy as np

from . import _native as N

MAGIC = b"ARTWS001"
DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "weights" / "warmstart.bin"
# The joint 4:2:0 network (same architecture and file format, trained with
# art_net_train_step_joint): used for 4:2:0 images when present.
DEFAULT_JOINT_WEIGHTS = Path(__file__).resolve().parent / "weights" / "warmstart_joint420.bin"
LAYERS = [("e1", 16, 32), ("e2", 32, 64), ("e3", 64, 96), ("e4", 96, 128), ("d3", 224, 96), ("d2", 160, 64),
          ("d1", 96, 32), ("head", 32, 16)]


def level0(n: int) -> int:
    """Side of the network's first level for a component side n (multiple of
    8): n padded to a multiple of 16, halved; each level-0 pixel carries a 2x2
    cell of samples."""
    return (n + 15) // 16 * 8


def num_params() -> int:
    return int(N.lib().art_net_num_params())


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases; the head starts near zero (prediction =
    decoded image) and only its first four output channels (the 2x2 cell of a
    level-0 pixel) are ever non-zero."""
    rng = np.random.default_rng(seed)
    out = []
    for name, cin, cout in LAYERS:
        std = np.sqrt(2.0 / (9 * cin))
        w = rng.standard_normal((cout, 9, cin)) * std
        if name == "head":
            w[4:] = 0.0
            w[:4] *= 0.01
        out += [w.ravel(), np.zeros(cout)]
    p = np.concatenate(out).astype(np.float32)
    assert p.size == num_params()
    return p


def save_params(path, params: np.ndarray) -> None:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    p = np.ascontiguousarray(params, dtype="<f4")
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(np.int64(p.size).tobytes())
        f.write(p.tobytes())


def load_params(path=DEFAULT_WEIGHTS) -> np.ndarray:
    data = Path(path).read_bytes()
    if data[:8] != MAGIC:
        raise ValueError(f"{path}: not a warm-start weights file")
    n = int(np.frombuffer(data[8:16], "<i8")[0])
    if n != num_params() or len(data) != 16 + 4 * n:
        raise ValueError(f"{path}: expected {num_params()} parameters")
    return np.frombuffer(data[16:], "<f4").copy()


def upsample_component(plane: np.ndarray, sh: int, sv: int, H: int, W: int) -> np.ndarray:
    """A component-resolution plane [h][w] upsampled to the full H x W grid as
    the learned start places it: along each subsampled axis (factor 2), sample
    2 i + d of cell i = 3/4 of cell i + 1/4 of its neighbour on that side
    (i - 1 for d = 0, i + 1 for d = 1), clamped at the edges; horizontal first,
    every product and sum rounded to float32 (bit-equal to the solver's
    k_upsample_smooth)."""
    p = np.asarray(plane, np.float32)
    h, w = p.shape
    y, x = np.arange(H), np.arange(W)
    cy, cx = np.minimum(y // sv, h - 1), np.minimum(x // sh, w - 1)
    nx = np.where(x & 1, np.minimum(cx + 1, w - 1), np.maximum(cx - 1, 0)) if sh == 2 else cx
    ny = np.where(y & 1, np.minimum(cy + 1, h - 1), np.maximum(cy - 1, 0)) if sv == 2 else cy
    a, b = np.float32(0.75), np.float32(0.25)
    mix = lambda u, v: (a * u + b * v).astype(np.float32)
    row = lambda r: mix(p[r][:, cx], p[r][:, nx]) if sh == 2 else p[r][:, cx]
    out = row(cy)
    if sv == 2:
        out = mix(out, row(ny))
    return np.ascontiguousarray(out, np.float32)


def coef_image(coef) -> np.ndarray:
    """Block-raster coefficients of one component -> int16 coefficient image
    (coefficient (v,u) of block (bx,by) at row 8by+v, column 8bx+u)."""
    c = np.asarray(coef.dct_coefs)
    if c.dtype != np.int16:
        if not np.all(np.isfinite(c)) or np.any(c != np.rint(c)) or np.abs(c).max(initial=0) > 32767:
            raise ValueError("coefficients must be integers in [-32768, 32767]")
        c = c.astype(np.int16)
    bh, bw = coef.block_h, coef.block_w
    return np.ascontiguousarray(c.reshape(bh, bw, 8, 8).transpose(0, 2, 1, 3).reshape(bh * 8, bw * 8))


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def _stream(stream) -> C.c_void_p:
    return C.c_void_p(stream.cuda_stream if stream is not None else 0)


class WarmStartNet:
    """The network on one GPU (``art_net_*``)."""

    def __init__(self, params: Optional[np.ndarray] = None, device: int = 0):
        p = init_params() if params is None else np.ascontiguousarray(params, dtype=np.float32)
        h = C.c_void_p()
        N.check(N.lib().art_net_create(device, p.ctypes.data, p.size, C.byref(h)))
        self._h = h
        self.device = device

    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS, device: int = 0) -> "WarmStartNet":
        return cls(load_params(path), device)

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def close(self) -> None:
        if self._h:
            N.lib().art_net_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.empty(num_params(), np.float32)
        N.check(N.lib().art_net_params(self._h, out.ctypes.data, out.size))
        return out

    def gradients(self) -> np.ndarray:
        out = np.empty(num_params(), np.float32)
        N.check(N.lib().art_net_gradients(self._h, out.ctypes.data, out.size))
        return out

    def save(self, path) -> None:
        save_params(path, self.params())

    def set_loss(self, smooth_weight: float) -> None:
        """Training loss = MSE + smooth_weight * mean squared difference of the
        error between adjacent samples (art_net_set_loss; 0 = plain MSE)."""
        N.check(N.lib().art_net_set_loss(self._h, float(smooth_weight)))

    def set_joint_loss(self, luma_weight: float) -> None:
        """Weight of the luma's squared errors in the joint 4:2:0 loss
        (art_net_set_joint_loss; default 1)."""
        N.check(N.lib().art_net_set_joint_loss(self._h, float(luma_weight)))

    def set_objective(self, lam: float, weight: float = 0.3, pweight: float = 0.001, nch: int = 3) -> None:
        """Training loss += lam / n * the solver's objective of the projected
        prediction (art_net_set_objective; 0 = off)."""
        N.check(N.lib().art_net_set_objective(self._h, float(lam), float(weight), float(pweight), int(nch)))

    def train_step(self, coef, q, target, lr: float, stream=None) -> float:
        """One step on a batch: coef int16 [B][H][W], q float32 [B][64] and
        target float32 [B][H][W] CUDA tensors. Returns the mean loss."""
        B, H, W = coef.shape
        loss = C.c_float()
        N.check(N.lib().art_net_train_step(self._h, _ptr(coef), W, H * W, _ptr(q), _ptr(target), B, H, W,
                                           float(lr), C.byref(loss), _stream(stream)))
        return float(loss.value)

    def train_step_joint(self, coef_y, coef_c, q_y, q_c, target, lr: float, stream=None) -> float:
        """One joint 4:2:0 step (art_net_train_step_joint): coef_y int16
        [B][H][W], coef_c int16 [B][2][H/2][W/2], q_y [B][64], q_c [B][2][64],
        target float32 [3][B][H][W] CUDA tensors. Returns the mean loss."""
        B, H, W = coef_y.shape
        loss = C.c_float()
        N.check(N.lib().art_net_train_step_joint(self._h, _ptr(coef_y), W, H * W, _ptr(coef_c), W // 2,
                                                 (H // 2) * (W // 2), _ptr(q_y), _ptr(q_c), _ptr(target), B, H, W,
                                                 float(lr), C.byref(loss), _stream(stream)))
        return float(loss.value)

    def predict_joint(self, coef_y, coef_c, q_y, q_c, out=None, stream=None):
        """Joint 4:2:0 prediction float32 [3][B][H][W] (art_net_predict_joint)."""
        import torch

        B, H, W = coef_y.shape
        if out is None:
            out = torch.empty((3, B, H, W), dtype=torch.float32, device=coef_y.device)
        N.check(N.lib().art_net_predict_joint(self._h, _ptr(coef_y), W, H * W, _ptr(coef_c), W // 2,
                                              (H // 2) * (W // 2), _ptr(q_y), _ptr(q_c), B, H, W, _ptr(out),
                                              _stream(stream)))
        return out

    def predict(self, coef, q, out=None, stream=None):
        """Prediction float32 [B][H][W] (a CUDA tensor) for coef int16 [B][H][W]."""
        import torch

        B, H, W = coef.shape
        if out is None:
            out = torch.empty((B, H, W), dtype=torch.float32, device=coef.device)
        N.check(N.lib().art_net_predict(self._h, _ptr(coef), W, H * W, _ptr(q), B, H, W, _ptr(out),
                                        _stream(stream)))
        return out

    def predict_decoded(self, coef, q, stream=None):
        """The decoded start IDCT(c q) per block, float32 [B][H][W] (the
        network's input before its residual; what the plain solver starts from)."""
        import torch

        B, H, W = coef.shape
        dec = torch.empty((B, H, W), dtype=torch.float32, device=coef.device)
        feat = torch.empty((B, level0(H), level0(W), 16), dtype=torch.bfloat16, device=coef.device)
        N.check(N.lib().art_cnn_features(_ptr(coef), W, H * W, _ptr(q), B, H, W, _ptr(dec), _ptr(feat),
                                         _stream(stream)))
        return dec
