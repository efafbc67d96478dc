"""Batched solves and the autotuner (GPU)."""
import numpy as np
import pytest

import oracle_lib as O
from artefact_b200 import Context, compute, synth
from parity import check_parity
from artefact_b200.api import Jpeg, JpegSource

pytestmark = pytest.mark.gpu

MAX_ABS = 1.0


def _jpeg(w, h, q, sub, gray, seed):
    return Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(w, h, q, sub, gray, seed)))


def test_batch_matches_single_solves(gpu):
    """Heterogeneous sizes, channel counts and subsamplings in one batch."""
    shapes = [(96, 64, 75, "4:2:0", False), (40, 24, 50, "4:4:4", True), (130, 70, 30, "4:4:4", False),
              (200, 136, 90, "4:2:0", False), (64, 48, 60, "4:2:2", False), (33, 17, 75, "4:4:4", True)]
    jpegs = [_jpeg(*s, seed=500 + i) for i, s in enumerate(shapes)]
    jobs = [dict(coefs=j.coefs, weight=0.3 + 0.1 * i, pweight=[0.001, 0.002, 0.0005]) for i, j in enumerate(jpegs)]
    with Context(0) as ctx:
        batch = ctx.compute_batch(jobs, 15)
    for j, job, got in zip(jpegs, jobs, batch):
        W, H, N_ = j.max_rounded()
        single = compute(j.nchannel, j.coefs, job["weight"], job["pweight"], 15, W, H, N_)
        # Same kernels, strips and reduction order as a solve of the image alone.
        assert all(np.array_equal(a, b) for a, b in zip(got, single))
        check_parity(j, 15, job["weight"], job["pweight"], label=f"batch {j.real_px_w}x{j.real_px_h}", gpu=got)


def test_batch_is_deterministic(gpu):
    jpegs = [_jpeg(72, 40, 75, "4:2:0", False, seed=600 + i) for i in range(3)]
    jobs = [dict(coefs=j.coefs) for j in jpegs]
    with Context(0) as ctx:
        a = ctx.compute_batch(jobs, 10)
        b = ctx.compute_batch(jobs, 10)
    assert all(np.array_equal(x, y) for pa, pb in zip(a, b) for x, y in zip(pa, pb))


def test_autotune_and_cache_roundtrip(gpu, tmp_path):
    j = _jpeg(512, 384, 75, "4:2:0", False, seed=700)
    W, H, N_ = j.max_rounded()
    with Context(0) as ctx:
        kind, rows = ctx.autotune(3, [1, 2, 2], [1, 2, 2], W, H, iterations=5)
        assert kind in (0, 1) and rows in (16, 32, 64, 128)
        path = tmp_path / "tune.txt"
        ctx.save_tune_cache(path)
        assert f" {kind} {rows}\n" in path.read_text()
        tuned = ctx.compute(3, j.coefs, 0.3, [0.001] * 3, 20, W, H)
    with Context(0) as ctx2:
        ctx2.load_tune_cache(path)
        again = ctx2.compute(3, j.coefs, 0.3, [0.001] * 3, 20, W, H)
    assert all(np.array_equal(a, b) for a, b in zip(tuned, again))
    ref = O.compute(3, j.coefs, 0.3, [0.001] * 3, 20, W, H)
    assert max(float(np.abs(a - b).max()) for a, b in zip(tuned, ref)) <= MAX_ABS


@pytest.mark.parametrize("shape", [(72, 40, "4:2:0", False), (200, 136, "4:4:4", False), (128, 96, "4:2:2", False),
                                   (96, 64, "4:4:4", True)])
def test_sweep_variants_agree(gpu, monkeypatch, shape):
    """The narrow and the wide gradient sweep at every strip height match the
    oracle, and each (variant, height) is deterministic."""
    w, h, sub, gray = shape
    j = _jpeg(w, h, 80, sub, gray, seed=900 + w)
    W, H, N_ = j.max_rounded()
    for kind in (0, 1):
        for rows in (16, 32, 64, 128):
            monkeypatch.setenv("ART_SWEEP_KIND", str(kind))
            monkeypatch.setenv("ART_STRIP_ROWS", str(rows))
            with Context(0) as ctx:
                a = ctx.compute(j.nchannel, j.coefs, 0.3, [0.001] * 3, 30, W, H)
                b = ctx.compute(j.nchannel, j.coefs, 0.3, [0.001] * 3, 30, W, H)
            assert all(np.array_equal(x, y) for x, y in zip(a, b))
            check_parity(j, 30, label=f"sweep variant {kind} rows {rows}", gpu=a)


def test_learned_batch_matches_single_learned_solves(gpu):
    """The learned start in a batch (each image's components through the
    network, the chroma pair as one batch) equals the learned start of each
    image alone, with the two-phase refinement schedule."""
    from artefact_b200 import _native as N
    from artefact_b200 import warmstart as WS

    shapes = [(96, 64, 75, "4:2:0", False), (40, 24, 50, "4:4:4", True), (130, 70, 30, "4:4:4", False),
              (64, 48, 60, "4:2:2", False)]
    jpegs = [_jpeg(*s, seed=700 + i) for i, s in enumerate(shapes)]
    jobs = [dict(coefs=j.coefs, weight=0.3, pweight=[0.001] * 3) for j in jpegs]
    net = WS.WarmStartNet.load() if WS.DEFAULT_WEIGHTS.exists() else WS.WarmStartNet(WS.init_params(2))
    sched = dict(step_iterations=2, tail_iterations=2, tail_step_iterations=100)
    with Context(0) as ctx:
        ctx.set_warm_start(net)
        batch = ctx.compute_batch(jobs, 8, init_mode=N.ART_INIT_LEARNED, **sched)
        for j, got in zip(jpegs, batch):
            W, H, _ = j.max_rounded()
            single = ctx.compute(j.nchannel, j.coefs, 0.3, [0.001] * 3, 8, W, H, init_mode=N.ART_INIT_LEARNED, **sched)
            d = max(float(np.abs(a - b).max()) for a, b in zip(got, single))
            assert d <= 1e-2, (j.real_px_w, j.real_px_h, d)
            ev = O.feasibility(j.nchannel, j.coefs, W, H, got)
            assert ev <= 1e-3
        ctx.set_warm_start(None)
