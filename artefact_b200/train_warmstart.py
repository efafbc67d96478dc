"""Training of the warm-start network on pairs the plain solver generates.

Data: ``n`` seeded 256x256 crops of the synthetic generator
(:mod:`artefact_b200.synth`), quality ~ U[20, 90], 4:2:0 or 4:4:4 with
p = 0.5, encoded as baseline JPEGs and decoded by the library's host decoder.
Targets: the plain GPU solver run to 300 iterations on each crop (joint
3-channel solve, weight 0.3, pweight 0.001); one sample per component, at the
component's own resolution (cell means of the full-resolution result for a
subsampled component), which is where the network predicts.

Training: Adam on the mean squared error of ``art_net_train_step`` (the
library's own BF16 tensor-core forward and backward kernels), optionally plus
the solver's objective of the projected prediction (``--objective``), batches
of one shape at a time, cosine learning-rate decay.

Usage::

    python -m artefact_b200.train_warmstart --crops 20000 --epochs 6 --out weights.bin
"""
from __future__ import annotations

import argparse
import math
import multiprocessing as mp
import os
import sys
import time
from concurrent.futures import ProcessPoolExecutor
from typing import Dict, List, Tuple

import numpy as np

CROP = 256
SEED0 = 100_000  # training crops; evaluation images use other seeds
WEIGHT, PWEIGHT = 0.3, 0.001
TARGET_ITERATIONS = 300


def crop_spec(i: int, seed0: int = SEED0, sub: str = "") -> Tuple[int, str, int]:
    """(quality, subsampling, seed) of training crop i; `sub` fixes the
    subsampling (the joint 4:2:0 network trains on 4:2:0 crops only)."""
    rng = np.random.default_rng(seed0 + i)
    q = int(rng.integers(20, 91))
    s = "4:2:0" if rng.random() < 0.5 else "4:4:4"
    return q, sub or s, seed0 + i


def _make_crop(args):
    i, seed0, sub = args
    from . import synth
    from .api import Jpeg, JpegSource

    q, sub, seed = crop_spec(i, seed0, sub)
    return Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(CROP, CROP, q, sub, False, seed)))


def make_crops(n: int, seed0: int = SEED0, workers: int = 0, sub: str = "") -> list:
    """Decoded JPEGs of crops 0..n-1 (a spawn-started process pool, so it is
    safe before or after CUDA is initialised)."""
    workers = workers or max(1, min(32, os.cpu_count() or 1))
    if workers == 1:
        return [_make_crop((i, seed0, sub)) for i in range(n)]
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_make_crop, [(i, seed0, sub) for i in range(n)], chunksize=64))


def cell_mean(plane: np.ndarray, sh: int, sv: int) -> np.ndarray:
    """Mean over sv x sh cells of a full-resolution plane (component resolution)."""
    H, W = plane.shape
    if sh == 1 and sv == 1:
        return plane
    return plane.reshape(H // sv, sv, W // sh, sh).mean(axis=(1, 3), dtype=np.float64).astype(np.float32)


def samples_from(jpegs: list, planes: List[List[np.ndarray]]):
    """Per component: (coefficient image int16 [h][w], q float32 [64], target float32 [h][w])."""
    from .warmstart import coef_image

    out = []
    for j, pl in zip(jpegs, planes):
        W, H, _ = j.max_rounded()
        for co, p in zip(j.coefs, pl):
            t = cell_mean(p.reshape(H, W), co.horizontal_samp_factor, co.vertical_samp_factor)
            out.append((coef_image(co), np.asarray(co.quant_table, np.float32), np.ascontiguousarray(t)))
    return out


def solve_targets(ctx, jpegs: list, iterations: int = TARGET_ITERATIONS, chunk: int = 512):
    """Plain solver results (host planes) of every crop, solved in batches."""
    res = []
    for k in range(0, len(jpegs), chunk):
        part = jpegs[k:k + chunk]
        jobs = [dict(coefs=j.coefs, weight=WEIGHT, pweight=[PWEIGHT] * 3) for j in part]
        res += ctx.compute_batch(jobs, iterations)
    return res


class Pools:
    """Training samples on the GPU, grouped by shape: {(h, w): (coef, q, target)}."""

    def __init__(self):
        self.parts: Dict[Tuple[int, int], list] = {}

    def add(self, samples) -> None:
        import torch

        by: Dict[Tuple[int, int], list] = {}
        for c, q, t in samples:
            by.setdefault(c.shape, []).append((c, q, t))
        for shp, items in by.items():
            c = torch.from_numpy(np.stack([i[0] for i in items])).cuda()
            q = torch.from_numpy(np.stack([i[1] for i in items])).cuda()
            t = torch.from_numpy(np.stack([i[2] for i in items])).cuda()
            self.parts.setdefault(shp, []).append((c, q, t))

    def tensors(self):
        import torch

        return {shp: tuple(torch.cat([p[k] for p in parts]) for k in range(3)) for shp, parts in self.parts.items()}


def build_pools(n: int, seed0: int, ctx, chunk: int = 1024, log=print):
    pools = Pools()
    t0 = time.time()
    for k in range(0, n, chunk):
        m = min(chunk, n - k)
        jpegs = make_crops(m, seed0 + k)
        t1 = time.time()
        planes = solve_targets(ctx, jpegs)
        pools.add(samples_from(jpegs, planes))
        log(f"crops {k + m}/{n}: decode {t1 - t0:.1f} s, solve {time.time() - t1:.1f} s")
        t0 = time.time()
    return pools.tensors()


def build_joint_pools(n: int, seed0: int, ctx, chunk: int = 1024, log=print):
    """Joint 4:2:0 samples on the GPU: coef_y int16 [N][H][W], coef_c int16
    [N][2][H/2][W/2], q_y [N][64], q_c [N][2][64] and the full-resolution
    300-iteration targets [N][3][H][W]."""
    import torch

    from .warmstart import coef_image

    parts = []
    t0 = time.time()
    for k in range(0, n, chunk):
        m = min(chunk, n - k)
        jpegs = make_crops(m, seed0 + k, sub="4:2:0")
        t1 = time.time()
        planes = solve_targets(ctx, jpegs)
        cy, cc, qy, qc, tg = [], [], [], [], []
        for j, pl in zip(jpegs, planes):
            W, H, _ = j.max_rounded()
            cy.append(coef_image(j.coefs[0]))
            cc.append(np.stack([coef_image(co) for co in j.coefs[1:]]))
            qy.append(np.asarray(j.coefs[0].quant_table, np.float32))
            qc.append(np.stack([np.asarray(co.quant_table, np.float32) for co in j.coefs[1:]]))
            tg.append(np.stack([p.reshape(H, W) for p in pl]))
        parts.append(tuple(torch.from_numpy(np.stack(a)).cuda() for a in (cy, cc, qy, qc, tg)))
        log(f"joint crops {k + m}/{n}: decode {t1 - t0:.1f} s, solve {time.time() - t1:.1f} s")
        t0 = time.time()
    return tuple(torch.cat([p[i] for p in parts]) for i in range(5))


def train_joint(net, data, epochs: int, lr: float = 1e-3, batch: int = 16, seed: int = 0, log=print):
    """Adam with linear warm-up and cosine decay on the joint 4:2:0 loss."""
    import torch

    g = torch.Generator(device="cpu").manual_seed(seed)
    n = data[0].shape[0]
    nb = math.ceil(n / batch)
    total = epochs * nb
    warm = min(200, total // 10 + 1)
    step, hist = 0, []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g)
        acc, t0 = 0.0, time.time()
        for b in range(nb):
            idx = perm[b * batch:(b + 1) * batch].cuda()
            cy, cc, qy, qc, tg = (t.index_select(0, idx) for t in data)
            cur = lr * min(1.0, (step + 1) / warm) * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * step / total)))
            loss = net.train_step_joint(cy.contiguous(), cc.contiguous(), qy.contiguous(), qc.contiguous(),
                                        tg.permute(1, 0, 2, 3).contiguous(), cur)
            acc += loss
            step += 1
            hist.append(loss)
        log(f"joint epoch {ep + 1}/{epochs}: mean loss {acc / nb:.5f} ({nb} steps, {time.time() - t0:.1f} s)")
    return hist


def evaluate_joint(net, data, batch: int = 16):
    """Mean squared error (levels^2) per component (luma, Cb, Cr) of the joint
    prediction against the targets."""
    import torch

    se = torch.zeros(3, dtype=torch.float64, device="cuda")
    n = data[0].shape[0]
    for b in range(0, n, batch):
        cy, cc, qy, qc, tg = (t[b:b + batch].contiguous() for t in data)
        pred = net.predict_joint(cy, cc, qy, qc)
        se += ((pred - tg.permute(1, 0, 2, 3)) ** 2).sum(dim=(1, 2, 3)).double()
    torch.cuda.synchronize()
    return (se / (n * data[0].shape[1] * data[0].shape[2])).tolist()


def batch_size(shape, pixels_per_batch: int) -> int:
    return max(1, pixels_per_batch // (shape[0] * shape[1]))


def train(net, data, epochs: int, lr: float = 1e-3, pixels_per_batch: int = 16 * CROP * CROP, seed: int = 0,
          log=print):
    """Adam with linear warm-up and cosine decay over all steps; batches are
    drawn shape by shape in a seeded random order. Returns the loss history."""
    import torch

    g = torch.Generator(device="cpu").manual_seed(seed)
    per_epoch = []
    for shp, (c, _, _) in data.items():
        per_epoch.append((shp, math.ceil(c.shape[0] / batch_size(shp, pixels_per_batch))))
    steps_epoch = sum(n for _, n in per_epoch)
    total = epochs * steps_epoch
    warm = min(200, total // 10 + 1)
    step, hist = 0, []
    for ep in range(epochs):
        order = []
        for shp, nb in per_epoch:
            n = data[shp][0].shape[0]
            perm = torch.randperm(n, generator=g)
            bs = batch_size(shp, pixels_per_batch)
            order += [(shp, perm[i * bs:(i + 1) * bs]) for i in range(nb)]
        seq = torch.randperm(len(order), generator=g).tolist()
        acc, cnt, t0 = 0.0, 0, time.time()
        for k in seq:
            shp, idx = order[k]
            c, q, t = data[shp]
            idx = idx.cuda()
            cur = lr * min(1.0, (step + 1) / warm) * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * step / total)))
            loss = net.train_step(c.index_select(0, idx).contiguous(), q.index_select(0, idx).contiguous(),
                                  t.index_select(0, idx).contiguous(), cur)
            acc += loss
            cnt += 1
            step += 1
            hist.append(loss)
        log(f"epoch {ep + 1}/{epochs}: mean loss {acc / max(cnt, 1):.5f} ({cnt} steps, {time.time() - t0:.1f} s)")
    return hist


def evaluate(net, data, pixels_per_batch: int = 16 * CROP * CROP):
    """Mean squared error (levels^2) of the prediction and of the decoded
    start against the targets, over every sample."""
    import torch

    se_pred = se_dec = 0.0
    npx = 0
    for shp, (c, q, t) in data.items():
        bs = batch_size(shp, pixels_per_batch)
        for i in range(0, c.shape[0], bs):
            cb, qb, tb = c[i:i + bs].contiguous(), q[i:i + bs].contiguous(), t[i:i + bs]
            pred = net.predict(cb, qb)
            dec = net.predict_decoded(cb, qb)
            se_pred += float(((pred - tb) ** 2).sum())
            se_dec += float(((dec - tb) ** 2).sum())
            npx += tb.numel()
    torch.cuda.synchronize()
    return se_pred / npx, se_dec / npx


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--crops", type=int, default=20000)
    ap.add_argument("--val", type=int, default=256, help="held-out crops for the final report")
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", required=True)
    ap.add_argument("--init", default=None, help="start from these weights instead of a fresh initialisation")
    ap.add_argument("--smooth", type=float, default=0.0,
                    help="weight of the loss's smoothness term (squared differences of the error between adjacent "
                         "samples); 0 = plain MSE")
    ap.add_argument("--joint", action="store_true",
                    help="train the joint 4:2:0 network (all three components in one pass, full-resolution chroma) "
                         "on 4:2:0 crops")
    ap.add_argument("--luma-weight", type=float, default=1.0,
                    help="joint network: weight of the luma's squared errors against the chroma's")
    ap.add_argument("--objective", type=float, default=0.0,
                    help="weight of the loss's objective term (the solver's objective of the projected "
                         "prediction, per sample); 0 = off")
    args = ap.parse_args(argv)

    def log(*a):
        print(*a, file=sys.stderr, flush=True)

    from . import warmstart as WS
    from .api import Context

    ctx = Context(0)
    net = WS.WarmStartNet(WS.load_params(args.init) if args.init else WS.init_params(args.seed))
    if args.joint:
        net.set_joint_loss(args.luma_weight)
        t0 = time.time()
        data = build_joint_pools(args.crops, SEED0, ctx, log=log)
        val = build_joint_pools(args.val, SEED0 + 10_000_000, ctx, log=log)
        log(f"data ready in {time.time() - t0:.1f} s: {data[0].shape[0]} crops")
        mse0 = evaluate_joint(net, val)
        t1 = time.time()
        train_joint(net, data, args.epochs, args.lr, seed=args.seed, log=log)
        log(f"training {time.time() - t1:.1f} s")
        mse = evaluate_joint(net, val)
        log(f"held-out MSE vs 300-iteration targets (levels^2, luma/Cb/Cr): untrained {mse0}, trained {mse}")
        net.save(args.out)
        print(f"{args.out}: held-out mse {mse}")
        return
    net.set_loss(args.smooth)
    net.set_objective(args.objective, WEIGHT, PWEIGHT)
    t0 = time.time()
    data = build_pools(args.crops, SEED0, ctx, log=log)
    val = build_pools(args.val, SEED0 + 10_000_000, ctx, log=log)
    log(f"data ready in {time.time() - t0:.1f} s: " + ", ".join(f"{k}: {v[0].shape[0]}" for k, v in data.items()))
    mse0, dec0 = evaluate(net, val)
    t1 = time.time()
    train(net, data, args.epochs, args.lr, seed=args.seed, log=log)
    log(f"training {time.time() - t1:.1f} s")
    mse, dec = evaluate(net, val)
    log(f"held-out MSE vs 300-iteration targets (levels^2): decoded {dec:.4f}, "
        f"untrained net {mse0:.4f}, trained net {mse:.4f}")
    net.save(args.out)
    print(f"{args.out}: held-out mse decoded {dec:.4f} trained {mse:.4f}")


if __name__ == "__main__":
    main()
