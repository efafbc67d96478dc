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
        assert kind in (0, 1, 2) and rows in (16, 32, 64, 128)
        res = ctx.last_tune()
        assert (res["variant"], res["strip_rows"]) == (kind, rows) and res["proj_warps"] in (2, 4, 8)
        assert res["candidates"] >= 3 and res["best_ms"] <= res["heuristic_ms"] * 1.0001
        cands = res["candidates_ms"]
        assert len(cands) == res["candidates"] and all(m > 0 for *_, m in cands)
        assert (cands[0][0], cands[0][1]) == (res["heuristic_variant"], res["heuristic_strip_rows"])
        assert any(c[:3] == (kind, rows, res["proj_warps"]) for c in cands)
        path = tmp_path / "tune.txt"
        ctx.save_tune_cache(path)
        assert f" {kind} {rows} {res['proj_warps']}\n" in path.read_text()
        tuned = ctx.compute(3, j.coefs, 0.3, [0.001] * 3, 20, W, H)
    with Context(0) as ctx2:
        ctx2.load_tune_cache(path)
        again = ctx2.compute(3, j.coefs, 0.3, [0.001] * 3, 20, W, H)
    assert all(np.array_equal(a, b) for a, b in zip(tuned, again))
    ref = O.compute(3, j.coefs, 0.3, [0.001] * 3, 20, W, H)
    assert max(float(np.abs(a - b).max()) for a, b in zip(tuned, ref)) <= MAX_ABS
    # Three-field lines (no projection shape) still load.
    old = tmp_path / "old.txt"
    old.write_text("n3-s112222-w512-h512 0 32\n")
    with Context(0) as ctx3:
        ctx3.load_tune_cache(old)


def test_autotune_batch(gpu, tmp_path):
    """The batch tuner times the shapes on the batch itself; later batches of
    its bucket use the choice, and their results still match the oracle."""
    shapes = [(96, 64, 75, "4:2:0", False), (40, 24, 50, "4:4:4", True), (130, 70, 30, "4:4:4", False),
              (200, 136, 90, "4:2:0", False), (64, 48, 60, "4:2:2", False)]
    jpegs = [_jpeg(*s, seed=800 + i) for i, s in enumerate(shapes)]
    jobs = [dict(coefs=j.coefs) for j in jpegs]
    with Context(0) as ctx:
        res = ctx.autotune_batch(jobs, iterations=5)
        assert res["variant"] in (0, 1, 2) and res["strip_rows"] in (16, 32, 64, 128) and res["proj_warps"] in (2, 4, 8)
        assert res["best_ms"] <= res["heuristic_ms"] * 1.0001
        path = tmp_path / "tune.txt"
        ctx.save_tune_cache(path)
        assert "batch-i8-" in path.read_text()
        # 30 iterations, as the candidate test below: at a dozen, the 130x70 q30
        # image is so ill-conditioned that the oracle's own fp32 and fp64 runs
        # differ by more than a level.
        a = ctx.compute_batch(jobs, 30)
        b = ctx.compute_batch(jobs, 30)
    assert all(np.array_equal(x, y) for pa, pb in zip(a, b) for x, y in zip(pa, pb))
    for j, got in zip(jpegs, a):
        check_parity(j, 30, label=f"tuned batch {j.real_px_w}x{j.real_px_h}", gpu=got)


@pytest.mark.parametrize("shape", [(72, 40, "4:2:0", False), (200, 136, "4:4:4", False), (128, 96, "4:2:2", False),
                                   (96, 64, "4:4:4", True)])
def test_every_tuning_candidate_agrees(gpu, monkeypatch, shape):
    """Every launch shape the autotuner may choose -- narrow, wide and quad
    sweep at each strip height, and 2, 4 or 8 projection warps per block --
    matches the oracle, and each is deterministic."""
    w, h, sub, gray = shape
    j = _jpeg(w, h, 80, sub, gray, seed=900 + w)
    W, H, N_ = j.max_rounded()
    n = j.nchannel
    its = 30
    for kind in (0, 1, 2):
        for rows in (16, 32, 64, 128):
            for pw in (2, 4, 8):
                monkeypatch.setenv("ART_SWEEP_KIND", str(kind))
                monkeypatch.setenv("ART_STRIP_ROWS", str(rows))
                monkeypatch.setenv("ART_PROJ_WARPS", str(pw))
                with Context(0) as ctx:
                    a = ctx.compute(n, j.coefs, 0.3, [0.001] * 3, its, W, H)
                    b = ctx.compute(n, j.coefs, 0.3, [0.001] * 3, its, W, H)
                label = f"{shape} sweep {kind} rows {rows} projection warps {pw}"
                assert all(np.array_equal(x, y) for x, y in zip(a, b)), label
                check_parity(j, its, label=label, gpu=a)
    # The projection shape does not change the arithmetic: 2, 4 and 8 warps
    # give identical planes for one sweep shape.
    outs = []
    for pw in (2, 4, 8):
        monkeypatch.setenv("ART_SWEEP_KIND", "0")
        monkeypatch.setenv("ART_STRIP_ROWS", "32")
        monkeypatch.setenv("ART_PROJ_WARPS", str(pw))
        with Context(0) as ctx:
            outs.append(ctx.compute(n, j.coefs, 0.3, [0.001] * 3, its, W, H))
    assert all(np.array_equal(x, y) for o in outs[1:] for x, y in zip(o, outs[0]))


def test_joint_learned_batch_matches_single_learned_solves(gpu):
    """With both networks attached, a batch mixing 4:2:0 images (joint pass)
    and other samplings (per component) equals each image's learned solve
    alone."""
    from artefact_b200 import _native as N
    from artefact_b200 import warmstart as WS

    shapes = [(96, 64, 75, "4:2:0", False), (40, 24, 50, "4:4:4", True), (160, 96, 30, "4:2:0", False),
              (64, 48, 60, "4:2:2", False), (96, 64, 40, "4:2:0", False)]
    jpegs = [_jpeg(*s, seed=720 + i) for i, s in enumerate(shapes)]
    jobs = [dict(coefs=j.coefs, weight=0.3, pweight=[0.001] * 3) for j in jpegs]
    net = WS.WarmStartNet.load() if WS.DEFAULT_WEIGHTS.exists() else WS.WarmStartNet(WS.init_params(2))
    joint = (WS.WarmStartNet.load(WS.DEFAULT_JOINT_WEIGHTS) if WS.DEFAULT_JOINT_WEIGHTS.exists()
             else WS.WarmStartNet(WS.init_params(3)))
    sched = dict(step_iterations=1, step_decay=0.9, tail_iterations=2, tail_step_iterations=100)
    with Context(0) as ctx:
        ctx.set_warm_start(net)
        ctx.set_joint_warm_start(joint)
        batch = ctx.compute_batch(jobs, 8, init_mode=N.ART_INIT_LEARNED, **sched)
        for j, got in zip(jpegs, batch):
            W, H, _ = j.max_rounded()
            single = ctx.compute(j.nchannel, j.coefs, 0.3, [0.001] * 3, 8, W, H, init_mode=N.ART_INIT_LEARNED, **sched)
            # The same network passes (per image or component group), kernels and
            # strips as a solve of the image alone.
            d = max(float(np.abs(a - b).max()) for a, b in zip(got, single))
            assert all(np.array_equal(a, b) for a, b in zip(got, single)), (j.real_px_w, j.real_px_h, d)
            assert O.feasibility(j.nchannel, j.coefs, W, H, got) <= 1e-3
        ctx.set_joint_warm_start(None)
        ctx.set_warm_start(None)


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
            # The same network passes (per image or component group), kernels and
            # strips as a solve of the image alone.
            d = max(float(np.abs(a - b).max()) for a, b in zip(got, single))
            assert all(np.array_equal(a, b) for a, b in zip(got, single)), (j.real_px_w, j.real_px_h, d)
            ev = O.feasibility(j.nchannel, j.coefs, W, H, got)
            assert ev <= 1e-3
        ctx.set_warm_start(None)
