"""Seeded synthetic JPEG inputs for tests and benchmarks.

No public dataset is used. Each channel is the sum of
  * Gaussian-blurred white noise (sigma 4 px), scaled to std 25 around 128,
  * 20 filled rectangles/ellipses with uniform random gray levels, blended over
    the noise at 70 %,
  * 3 sinusoidal gratings of random orientation, period U[6, 40] px,
    amplitude 20,
clipped to [0, 255] and cast to uint8. RGB images use three independent seeds.
Images are encoded with Pillow (libjpeg-turbo) as baseline JPEGs with the IJG
quality scaling of the Annex K tables, standard Huffman tables and
4:4:4 / 4:2:0 subsampling; single-channel images are encoded in mode "L".
Seeds: configuration c, image i -> 1000 * c + i.
"""
from __future__ import annotations

import io
from dataclasses import dataclass
from typing import List

import numpy as np

__all__ = ["channel_image", "rgb_image", "encode_jpeg", "make_jpeg", "batch_specs", "BatchSpec"]


def _blur(img: np.ndarray, sigma: float) -> np.ndarray:
    from scipy.ndimage import gaussian_filter

    return gaussian_filter(img, sigma=sigma, mode="reflect")


def channel_image(h: int, w: int, seed: int) -> np.ndarray:
    """One seeded uint8 channel of the piecewise-smooth + texture generator."""
    rng = np.random.default_rng(seed)
    noise = _blur(rng.standard_normal((h, w)).astype(np.float32), 4.0)
    noise = noise / max(float(noise.std()), 1e-6) * 25.0 + 128.0
    img = noise.astype(np.float32)
    yy = np.arange(h, dtype=np.float32)[:, None]
    xx = np.arange(w, dtype=np.float32)[None, :]
    for _ in range(20):
        level = float(rng.uniform(0, 255))
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        rw, rh = rng.uniform(0.03, 0.3) * w, rng.uniform(0.03, 0.3) * h
        x0, x1 = int(max(cx - rw, 0)), int(min(cx + rw, w))
        y0, y1 = int(max(cy - rh, 0)), int(min(cy + rh, h))
        if x1 <= x0 or y1 <= y0:
            continue
        sub = img[y0:y1, x0:x1]
        if rng.random() < 0.5:
            sub[...] = 0.3 * sub + 0.7 * level
        else:
            m = ((xx[:, x0:x1] - cx) / rw) ** 2 + ((yy[y0:y1] - cy) / rh) ** 2 <= 1.0
            sub[m] = 0.3 * sub[m] + 0.7 * level
    for _ in range(3):
        theta = rng.uniform(0, np.pi)
        period = rng.uniform(6, 40)
        phase = rng.uniform(0, 2 * np.pi)
        img += 20.0 * np.sin(2 * np.pi * (xx * np.cos(theta) + yy * np.sin(theta)) / period + phase).astype(np.float32)
    return np.clip(np.rint(img), 0, 255).astype(np.uint8)


def rgb_image(h: int, w: int, seed: int) -> np.ndarray:
    """(h, w, 3) uint8 image with an independent seed per channel."""
    return np.stack([channel_image(h, w, seed * 3 + k) for k in range(3)], axis=-1)


def encode_jpeg(img: np.ndarray, quality: int, subsampling: str = "4:2:0") -> bytes:
    """Baseline JPEG via Pillow; subsampling "4:4:4", "4:2:2" or "4:2:0"."""
    from PIL import Image

    mode = "L" if img.ndim == 2 else "RGB"
    sub = {"4:4:4": 0, "4:2:2": 1, "4:2:0": 2}[subsampling]
    buf = io.BytesIO()
    kw = dict(format="JPEG", quality=int(quality), optimize=False, progressive=False)
    if mode == "RGB":
        kw["subsampling"] = sub
    Image.fromarray(img, mode).save(buf, **kw)
    return buf.getvalue()


def make_jpeg(w: int, h: int, quality: int, subsampling: str = "4:2:0", gray: bool = False, seed: int = 0) -> bytes:
    """Seeded synthetic image of the given size, encoded as a baseline JPEG."""
    img = channel_image(h, w, seed) if gray else rgb_image(h, w, seed)
    return encode_jpeg(img, quality, subsampling)


@dataclass
class BatchSpec:
    width: int
    height: int
    subsampling: str
    quality: int
    seed: int


def batch_specs(n: int = 256, seed: int = 4000) -> List[BatchSpec]:
    """Heterogeneous batch: W, H ~ U[256, 2048] rounded to multiples of 16,
    4:2:0 or 4:4:4 with p = 0.5, quality ~ U[20, 90]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        w = int(round(rng.uniform(256, 2048) / 16)) * 16
        h = int(round(rng.uniform(256, 2048) / 16)) * 16
        sub = "4:2:0" if rng.random() < 0.5 else "4:4:4"
        q = int(rng.integers(20, 91))
        out.append(BatchSpec(w, h, sub, q, seed + i))
    return out
