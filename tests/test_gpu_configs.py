"""Parity at the benchmark configurations' own sizes (GPU).

* 6000-wide 4:4:4 q30 at 100 iterations: a full-width 6000x512 band cut from
  the 6000x4000 benchmark image (same generator and seed), which stays
  well-conditioned, so the fixed bar applies: max |GPU - oracle fp32| <= 1.0
  in 0..255 units, objective within 1e-4 relative, feasibility <= 1e-3.
* The 256-image batch (seed 4000) solved as one batch through the public
  batch API: its 4 largest and 4 smallest images against the oracle at 50
  iterations, with the same bar.
* The learned path with the shipped trained network on 1920x1080 4:2:0 at
  q30/50/75: the GPU's ART_INIT_LEARNED solve against the oracle's iteration
  from the same (GPU-predicted) start (oracle compute_from), at 8 iterations
  and at the fewest ladder iterations that reach the plain 50-iteration
  objective within 1e-4; each must be feasible, and the objective reached
  there must hold on the oracle's planes too.

Oracle runs of different images go to host threads (the oracle releases the
interpreter lock while it computes).
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import oracle_lib as O
from artefact_b200 import _native as N
from artefact_b200 import synth
from artefact_b200 import warmstart as WS
from artefact_b200.api import Context, Jpeg, JpegSource
from parity import OracleRef, check_parity

pytestmark = pytest.mark.gpu

WEIGHT, PW = 0.3, [0.001] * 3


def _jpeg(data):
    return Jpeg.from_source(JpegSource.Buffer(data))


def test_config3_band_100_iterations(gpu):
    img = synth.rgb_image(4000, 6000, 3000)[:512]
    j = _jpeg(synth.encode_jpeg(np.ascontiguousarray(img), 30, "4:4:4"))
    assert (j.real_px_w, j.real_px_h) == (6000, 512)
    check_parity(j, 100, label="6000x512 band of the 6000x4000 4:4:4 q30 image")


def test_config2_every_sweep_variant(gpu, monkeypatch):
    """1920x1080 4:2:0 q75 at 50 iterations with each gradient-sweep variant
    the autotuner may pick (narrow, wide, quad) at 16- and 32-row strips,
    against one set of oracle runs (the conditioning-aware bar)."""
    j = _jpeg(synth.make_jpeg(1920, 1080, 75, "4:2:0", False, seed=2000))
    W, H, _ = j.max_rounded()
    ref = OracleRef(j, 50, WEIGHT, PW)
    for kind in (0, 1, 2):
        for rows in (16, 32):
            monkeypatch.setenv("ART_SWEEP_KIND", str(kind))
            monkeypatch.setenv("ART_STRIP_ROWS", str(rows))
            with Context(0) as ctx:
                got = ctx.compute(3, j.coefs, WEIGHT, PW, 50, W, H)
            ref.check(got, label=f"1080p sweep {kind} rows {rows}")


def test_config4_batch_extremes(gpu):
    specs = synth.batch_specs(256, seed=4000)
    with ThreadPoolExecutor(max_workers=16) as ex:
        datas = list(ex.map(lambda s: synth.make_jpeg(s.width, s.height, s.quality, s.subsampling, False, s.seed),
                            specs))
    jpegs = [_jpeg(d) for d in datas]
    with Context(0) as ctx:
        out = ctx.compute_batch([dict(coefs=j.coefs, weight=WEIGHT, pweight=PW) for j in jpegs], 50)
    order = sorted(range(len(jpegs)), key=lambda i: jpegs[i].real_px_w * jpegs[i].real_px_h)
    picks = order[:4] + order[-4:]

    def check(i):
        j = jpegs[i]
        check_parity(j, 50, label=f"batch image {i} {j.real_px_w}x{j.real_px_h} q{specs[i].quality} "
                                  f"{specs[i].subsampling}", gpu=out[i])
        return i

    with ThreadPoolExecutor(max_workers=len(picks)) as ex:
        assert sorted(ex.map(check, picks)) == sorted(picks)


def _refine(k):
    """The bench's refinement schedule for k iterations after a learned start."""
    return dict(step_iterations=1, step_decay=0.9, tail_iterations=min(2, k - 1) if k <= 12 else 0,
                tail_step_iterations=100)


def _prediction(net, j):
    import torch

    W, H, _ = j.max_rounded()
    out = []
    for co in j.coefs:
        ci = torch.from_numpy(WS.coef_image(co)[None]).cuda()
        q = torch.from_numpy(np.asarray(co.quant_table, np.float32)[None].copy()).cuda()
        p = net.predict(ci, q)[0].cpu().numpy()
        out.append(WS.upsample_component(p, co.horizontal_samp_factor, co.vertical_samp_factor, H, W))
    return out


def _joint_prediction(net, j):
    import torch

    W, H, _ = j.max_rounded()
    cy = torch.from_numpy(WS.coef_image(j.coefs[0])[None]).cuda()
    cc = torch.from_numpy(np.stack([WS.coef_image(co) for co in j.coefs[1:]])[None]).cuda()
    qy = torch.from_numpy(np.asarray(j.coefs[0].quant_table, np.float32)[None].copy()).cuda()
    qc = torch.from_numpy(np.stack([np.asarray(co.quant_table, np.float32) for co in j.coefs[1:]])[None]).cuda()
    pred = net.predict_joint(cy, cc, qy, qc).cpu().numpy()
    return [pred[c, 0].reshape(H, W) for c in range(3)]


@pytest.mark.skipif(not WS.DEFAULT_WEIGHTS.exists(), reason="no trained weights in the package")
@pytest.mark.parametrize("network", ["per-component", "joint"])
@pytest.mark.parametrize("quality", [30, 50, 75])
def test_config5_trained_learned_1080p(gpu, quality, network):
    """Config 5 with the shipped weights: the learned start (per-component
    network, or the joint 4:2:0 network when it ships) refined with the bench's
    schedule, against the oracle started from the same prediction, at 8
    iterations and at the fewest that reach the plain 50-iteration objective."""
    if network == "joint" and not WS.DEFAULT_JOINT_WEIGHTS.exists():
        pytest.skip("no joint 4:2:0 weights in the package")
    j = _jpeg(synth.make_jpeg(1920, 1080, quality, "4:2:0", False, seed=5000 + quality))
    W, H, _ = j.max_rounded()
    net = WS.WarmStartNet.load() if network == "per-component" else WS.WarmStartNet.load(WS.DEFAULT_JOINT_WEIGHTS)
    attach = (lambda c, n: c.set_warm_start(n)) if network == "per-component" else \
        (lambda c, n: c.set_joint_warm_start(n))
    ctx = Context(0)
    try:
        ctx.compute(3, j.coefs, WEIGHT, PW, 50, W, H)
        e50 = ctx.evaluate()["E"]
        attach(ctx, net)
        reach = None
        for k in (8, 12, 16, 20, 24, 28, 32, 40, 48):
            ctx.compute(3, j.coefs, WEIGHT, PW, k, W, H, init_mode=N.ART_INIT_LEARNED, **_refine(k))
            ev = ctx.evaluate()
            if ev["E"] <= e50 * (1 + 1e-4) and ev["infeasibility"] <= 1e-3:
                reach = k
                break
        assert reach is not None, "the learned path never reached the plain 50-iteration objective"
        runs = {}
        for k in sorted({8, reach}):
            runs[k] = ctx.compute(3, j.coefs, WEIGHT, PW, k, W, H, init_mode=N.ART_INIT_LEARNED, **_refine(k))
            runs[k] = (runs[k], ctx.evaluate())
        attach(ctx, None)
        start = _prediction(net, j) if network == "per-component" else _joint_prediction(net, j)
    finally:
        attach(ctx, None)
        ctx.close()
        net.close()

    def oracle(job):
        k, fp64 = job
        s = _refine(k)
        return job, O.compute_from(3, j.coefs, WEIGHT, PW, k, W, H, start, s["step_iterations"], fp64=fp64,
                                   tail_iterations=s["tail_iterations"], tail_step_iterations=s["tail_step_iterations"],
                                   step_decay=s["step_decay"])

    with ThreadPoolExecutor(max_workers=4) as ex:
        refs = dict(ex.map(oracle, [(k, fp64) for k in runs for fp64 in (False, True)]))
    for k, (planes, ev) in runs.items():
        ref, r64 = refs[(k, False)], refs[(k, True)]
        d = max(float(np.abs(a.astype(np.float64) - b).max()) for a, b in zip(planes, ref))
        spread = max(float(np.abs(a.astype(np.float64) - b).max()) for a, b in zip(ref, r64))
        # The fixed bar where the oracle's own fp32 and fp64 runs agree to 0.5,
        # else twice their spread + 0.5 (as tests/parity.py does).
        bar = 1.0 if spread <= 0.5 else 2 * spread + 0.5
        er = O.objective(3, j.coefs, WEIGHT, PW, W, H, ref)
        feas = O.feasibility(3, j.coefs, W, H, planes)
        print(f"q{quality} K={k}: max|gpu-oracle|={d:.3g} (oracle f32/f64 {spread:.3g}) E gpu {ev['E']:.9g} "
              f"oracle {er:.9g} rel to plain-50 {ev['E'] / e50 - 1:+.2e} feas {feas:.2g} (reaches at K={reach})")
        assert d <= bar
        assert abs(ev["E"] - er) <= 1e-4 * abs(er)
        assert feas <= 1e-3 and ev["infeasibility"] <= 1e-3
        if k == reach:
            assert er <= e50 * (1 + 2e-4)  # the oracle's planes reach it too (within the parity bar)
