"""The GPU objective evaluator and the learned (warm) start, against the oracle (GPU).

* ``art_context_evaluate`` (fp64 objective and feasibility on the GPU) against
  the oracle's fp64 objective and feasibility of the same planes.
* ``ART_INIT_LEARNED``: the solver's projection of the network's prediction
  and the plain iterations after it, against the oracle's iteration from the
  same start planes (``oracle_*_compute_from``), with the plain solver's
  parity bar (max |GPU - oracle| <= 1.0 in 0..255 units, objective within
  1e-4 relative, feasibility <= 1e-3 coefficient units).
* The trained network's gain: from its start, a few plain iterations reach a
  lower objective than the same iterations from the decoded start.
"""
import numpy as np
import pytest

import oracle_lib as O
from artefact_b200 import _native as N
from artefact_b200 import synth
from artefact_b200 import warmstart as WS
from artefact_b200.api import Context, Jpeg, JpegSource

pytestmark = pytest.mark.gpu

WEIGHT, PW = 0.3, [0.001] * 3
CASES = [(40, 24, 50, "4:4:4", True), (72, 40, 75, "4:2:0", False), (48, 32, 30, "4:4:4", False),
         (200, 136, 75, "4:2:0", False), (50, 30, 75, "4:2:2", False)]
IDS = [f"{c[0]}x{c[1]}_q{c[2]}_{c[3]}{'_gray' if c[4] else ''}" for c in CASES]


def jpeg_of(w, h, q, sub, gray, seed=21):
    return Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(w, h, q, sub, gray, seed)))


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("shape", CASES, ids=IDS)
@pytest.mark.parametrize("iterations", [0, 10])
def test_evaluate_matches_oracle(gpu, ctx, shape, iterations):
    j = jpeg_of(*shape)
    W, H, _ = j.max_rounded()
    n = j.nchannel
    planes = ctx.compute(n, j.coefs, WEIGHT, PW, iterations, W, H)
    ev = ctx.evaluate()
    e, terms = O.objective(n, j.coefs, WEIGHT, PW, W, H, planes, terms=True)
    assert abs(ev["E"] - e) <= 1e-9 * abs(e), (ev, e)
    for got, ref in zip((ev["tv"], ev["tgv"], ev["prob"]), terms):
        assert abs(got - ref) <= 1e-9 * abs(e), (ev, terms)
    feas = O.feasibility(n, j.coefs, W, H, planes)
    assert abs(ev["infeasibility"] - feas) <= 1e-6, (ev["infeasibility"], feas)
    assert ev["infeasibility"] <= 1e-3


def _strong_params(seed):
    """Untrained weights whose head is large enough that the prediction moves
    visibly away from the decoded start (the trained head is not near zero)."""
    p = WS.init_params(seed)
    rng = np.random.default_rng(seed)
    offs = {}
    o = 0
    for name, cin, cout in WS.LAYERS:
        offs[name] = (o, o + cout * 9 * cin)
        o += cout * 9 * cin + cout
    lo, hi = offs["head"]
    p[lo:lo + 4 * 9 * 32] = (rng.standard_normal(4 * 9 * 32) * 0.05).astype(np.float32)
    return p


def _upsampled_prediction(net, j):
    """Per component: the network's prediction at the component's resolution,
    upsampled to full resolution as the solver places it."""
    import torch

    W, H, _ = j.max_rounded()
    out = []
    for co in j.coefs:
        ci = torch.from_numpy(WS.coef_image(co)[None]).cuda()
        q = torch.from_numpy(np.asarray(co.quant_table, np.float32)[None].copy()).cuda()
        p = net.predict(ci, q)[0].cpu().numpy()
        out.append(WS.upsample_component(p, co.horizontal_samp_factor, co.vertical_samp_factor, H, W))
    return out


@pytest.mark.parametrize("shape", CASES, ids=IDS)
@pytest.mark.parametrize("iterations,step_iterations,tail,tail_step",
                         [(0, 0, 0, 0), (1, 0, 0, 0), (8, 0, 0, 0), (8, 50, 0, 0), (10, 8, 4, 60), (6, 0, 6, 20)])
def test_learned_start_matches_oracle(gpu, ctx, shape, iterations, step_iterations, tail, tail_step):
    j = jpeg_of(*shape)
    W, H, _ = j.max_rounded()
    n = j.nchannel
    net = WS.WarmStartNet(_strong_params(7))
    ctx.set_warm_start(net)
    try:
        gpu_planes = ctx.compute(n, j.coefs, WEIGHT, PW, iterations, W, H, init_mode=N.ART_INIT_LEARNED,
                                 step_iterations=step_iterations, tail_iterations=tail,
                                 tail_step_iterations=tail_step)
        ev = ctx.evaluate()
    finally:
        ctx.set_warm_start(None)
    start = _upsampled_prediction(net, j)
    ref = O.compute_from(n, j.coefs, WEIGHT, PW, iterations, W, H, start, step_iterations,
                         tail_iterations=tail, tail_step_iterations=tail_step)
    r64 = O.compute_from(n, j.coefs, WEIGHT, PW, iterations, W, H, start, step_iterations, fp64=True,
                         tail_iterations=tail, tail_step_iterations=tail_step)
    d = max(float(np.abs(a.astype(np.float64) - b).max()) for a, b in zip(gpu_planes, ref))
    d64 = max(float(np.abs(a.astype(np.float64) - b).max()) for a, b in zip(gpu_planes, r64))
    moved = max(float(np.abs(s.ravel() - a).max()) for s, a in zip(start, ref))
    er = O.objective(n, j.coefs, WEIGHT, PW, W, H, ref)
    print(f"{shape} it={iterations} step_it={step_iterations} max|gpu-f32|={d:.3g} max|gpu-f64|={d64:.3g} "
          f"start moved by {moved:.3g} objective gpu {ev['E']:.9g} oracle {er:.9g}")
    assert d <= 1.0
    assert abs(ev["E"] - er) <= 1e-4 * abs(er)
    assert ev["infeasibility"] <= 1e-3


@pytest.mark.parametrize("shape", CASES[1:4], ids=IDS[1:4])
@pytest.mark.parametrize("iterations,step_iterations,tail,tail_step,decay",
                         [(8, 2, 2, 100, 0.8), (10, 1, 0, 0, 0.6), (6, 4, 2, 50, 0.95)])
def test_step_decay_matches_oracle(gpu, ctx, shape, iterations, step_iterations, tail, tail_step, decay):
    """A geometric first-phase step schedule (ArtOptions.step_decay) after a
    learned start, against the oracle's iteration with the same schedule."""
    j = jpeg_of(*shape)
    W, H, _ = j.max_rounded()
    n = j.nchannel
    net = WS.WarmStartNet(_strong_params(7))
    ctx.set_warm_start(net)
    try:
        got = ctx.compute(n, j.coefs, WEIGHT, PW, iterations, W, H, init_mode=N.ART_INIT_LEARNED,
                          step_iterations=step_iterations, tail_iterations=tail, tail_step_iterations=tail_step,
                          step_decay=decay)
        ev = ctx.evaluate()
    finally:
        ctx.set_warm_start(None)
    start = _upsampled_prediction(net, j)
    ref = O.compute_from(n, j.coefs, WEIGHT, PW, iterations, W, H, start, step_iterations, tail_iterations=tail,
                         tail_step_iterations=tail_step, step_decay=decay)
    d = max(float(np.abs(a.astype(np.float64) - b).max()) for a, b in zip(got, ref))
    er = O.objective(n, j.coefs, WEIGHT, PW, W, H, ref)
    assert d <= 1.0
    assert abs(ev["E"] - er) <= 1e-4 * abs(er)
    assert ev["infeasibility"] <= 1e-3
    # The schedule changes the result: without the decay it differs.
    plain = O.compute_from(n, j.coefs, WEIGHT, PW, iterations, W, H, start, step_iterations, tail_iterations=tail,
                           tail_step_iterations=tail_step)
    assert max(float(np.abs(a - b).max()) for a, b in zip(plain, ref)) > 0


def _joint_prediction(net, j):
    """The joint network's full-resolution planes of a 4:2:0 image, as the
    solver places them."""
    import torch

    W, H, _ = j.max_rounded()
    cy = torch.from_numpy(WS.coef_image(j.coefs[0])[None]).cuda()
    cc = torch.from_numpy(np.stack([WS.coef_image(co) for co in j.coefs[1:]])[None]).cuda()
    qy = torch.from_numpy(np.asarray(j.coefs[0].quant_table, np.float32)[None].copy()).cuda()
    qc = torch.from_numpy(np.stack([np.asarray(co.quant_table, np.float32) for co in j.coefs[1:]])[None]).cuda()
    pred = net.predict_joint(cy, cc, qy, qc).cpu().numpy()
    return [pred[c, 0].reshape(H, W) for c in range(3)]


def _joint_strong_params(seed):
    p = _strong_params(seed)
    rng = np.random.default_rng(seed + 1)
    o = 0
    for name, cin, cout in WS.LAYERS:
        if name == "head":
            p[o + 4 * 9 * 32:o + 12 * 9 * 32] = (rng.standard_normal(8 * 9 * 32) * 0.05).astype(np.float32)
        o += cout * 9 * cin + cout
    return p


@pytest.mark.parametrize("shape", [(96, 64, 75, "4:2:0", False), (200, 136, 30, "4:2:0", False)])
@pytest.mark.parametrize("iterations,step_iterations,tail,tail_step", [(0, 0, 0, 0), (8, 2, 2, 100)])
def test_joint_learned_start_matches_oracle(gpu, ctx, shape, iterations, step_iterations, tail, tail_step):
    """A 4:2:0 image with a joint network attached: the solver's learned start
    and refinement against the oracle started from the joint prediction."""
    j = jpeg_of(*shape)
    W, H, _ = j.max_rounded()
    n = j.nchannel
    net = WS.WarmStartNet(_joint_strong_params(8))
    ctx.set_joint_warm_start(net)
    try:
        got = ctx.compute(n, j.coefs, WEIGHT, PW, iterations, W, H, init_mode=N.ART_INIT_LEARNED,
                          step_iterations=step_iterations, tail_iterations=tail, tail_step_iterations=tail_step)
        ev = ctx.evaluate()
    finally:
        ctx.set_joint_warm_start(None)
    start = _joint_prediction(net, j)
    ref = O.compute_from(n, j.coefs, WEIGHT, PW, iterations, W, H, start, step_iterations, tail_iterations=tail,
                         tail_step_iterations=tail_step)
    d = max(float(np.abs(a.astype(np.float64) - b).max()) for a, b in zip(got, ref))
    er = O.objective(n, j.coefs, WEIGHT, PW, W, H, ref)
    moved = max(float(np.abs(s.ravel() - a).max()) for s, a in zip(start, ref))
    print(f"{shape} it={iterations}: max|gpu-oracle| {d:.3g}, start moved by {moved:.3g}")
    assert d <= 1.0
    assert abs(ev["E"] - er) <= 1e-4 * abs(er)
    assert ev["infeasibility"] <= 1e-3


def test_joint_network_needs_per_component_network_for_other_samplings(gpu, ctx):
    """A joint network alone serves 4:2:0 images only; a 4:4:4 learned solve
    then asks for the per-component network."""
    j = jpeg_of(48, 32, 30, "4:4:4", False)
    W, H, _ = j.max_rounded()
    net = WS.WarmStartNet(_joint_strong_params(9))
    ctx.set_joint_warm_start(net)
    try:
        with pytest.raises(N.ArtError, match="not 4:2:0"):
            ctx.compute(j.nchannel, j.coefs, WEIGHT, PW, 2, W, H, init_mode=N.ART_INIT_LEARNED)
    finally:
        ctx.set_joint_warm_start(None)


def test_step_decay_is_validated(gpu, ctx):
    j = jpeg_of(*CASES[0])
    W, H, _ = j.max_rounded()
    with pytest.raises(N.ArtError, match="step_decay"):
        ctx.compute(j.nchannel, j.coefs, WEIGHT, PW, 2, W, H, step_decay=1.5)


@pytest.mark.parametrize("shape", CASES[:3], ids=IDS[:3])
def test_zero_residual_start_equals_decoded_start(gpu, ctx, shape):
    """With a zero head the prediction is the decoded image, whose projection
    is itself: without subsampled components the learned path then follows the
    plain solver; with them it starts from the decoded components upsampled
    smoothly, and follows the oracle from that start."""
    j = jpeg_of(*shape)
    W, H, _ = j.max_rounded()
    n = j.nchannel
    p = WS.init_params(3)
    offs = 0
    for name, cin, cout in WS.LAYERS:
        if name == "head":
            p[offs:offs + cout * 9 * cin + cout] = 0.0
        offs += cout * 9 * cin + cout
    net = WS.WarmStartNet(p)
    ctx.set_warm_start(net)
    try:
        a = ctx.compute(n, j.coefs, WEIGHT, PW, 10, W, H, init_mode=N.ART_INIT_LEARNED)
    finally:
        ctx.set_warm_start(None)
    if all(co.horizontal_samp_factor == 1 and co.vertical_samp_factor == 1 for co in j.coefs):
        b = ctx.compute(n, j.coefs, WEIGHT, PW, 10, W, H)
        d = max(float(np.abs(x - y).max()) for x, y in zip(a, b))
        assert d <= 1e-2, d
    else:
        ref = O.compute_from(n, j.coefs, WEIGHT, PW, 10, W, H, _upsampled_prediction(net, j))
        d = max(float(np.abs(x.astype(np.float64) - y).max()) for x, y in zip(a, ref))
        assert d <= 1.0, d


def test_learned_start_graph_replay(gpu):
    """The learned start runs eagerly the first time a geometry is seen, is
    captured into a CUDA graph the second time and replayed after that. Every
    run gives the same planes, across a change of geometry, and after a
    training step changes the weights (and reallocates the network's buffers)
    the replayed context agrees with a fresh one."""
    import torch

    c = Context(0)
    fresh = Context(0)
    net = WS.WarmStartNet(_strong_params(11))
    try:
        c.set_warm_start(net)
        fresh.set_warm_start(net)

        def run(ctx_, j):
            W, H, _ = j.max_rounded()
            return ctx_.compute(j.nchannel, j.coefs, WEIGHT, PW, 6, W, H, init_mode=N.ART_INIT_LEARNED,
                                step_iterations=2, tail_iterations=2, tail_step_iterations=100)

        def same(a, b):
            return all(np.array_equal(x, y) for x, y in zip(a, b))

        ja, jb = jpeg_of(*CASES[3]), jpeg_of(*CASES[1])
        ref_a = run(c, ja)
        for _ in range(3):  # captured, then replayed
            assert same(run(c, ja), ref_a)
        ref_b = run(c, jb)
        assert same(run(c, jb), ref_b) and same(run(c, jb), ref_b)
        assert same(run(c, ja), ref_a) and same(run(c, ja), ref_a)
        # A training step: new weights (repacked before the next prediction).
        jt = jpeg_of(256, 256, 50, "4:4:4", True, seed=3)
        co = jt.coefs[0]
        coef = torch.from_numpy(WS.coef_image(co)[None]).cuda()
        q = torch.from_numpy(np.asarray(co.quant_table, np.float32)[None].copy()).cuda()
        target = net.predict_decoded(coef, q) + 1.0
        net.train_step(coef, q, target, lr=1e-3)
        got = [run(c, ja) for _ in range(3)]
        want = run(fresh, ja)
        assert not same(want, ref_a)
        assert all(same(g, want) for g in got)
        # Another network in place of the first (often at the same host
        # address once the first is freed): the graph recorded with the first
        # network's buffers must not be replayed.
        for seed in (13, 14):
            c.set_warm_start(None)
            fresh.set_warm_start(None)
            net.close()
            net = WS.WarmStartNet(_strong_params(seed))
            c.set_warm_start(net)
            fresh.set_warm_start(net)
            got = [run(c, ja) for _ in range(3)]
            want = run(fresh, ja)
            assert all(same(g, want) for g in got)
    finally:
        c.set_warm_start(None)
        fresh.set_warm_start(None)
        c.close()
        fresh.close()
        net.close()


def test_learned_start_needs_a_network(gpu, ctx):
    j = jpeg_of(*CASES[0])
    W, H, _ = j.max_rounded()
    with pytest.raises(N.ArtError, match="no network attached"):
        ctx.compute(j.nchannel, j.coefs, WEIGHT, PW, 2, W, H, init_mode=N.ART_INIT_LEARNED)


@pytest.mark.skipif(not WS.DEFAULT_WEIGHTS.exists(), reason="no trained weights in the package")
@pytest.mark.parametrize("quality", [30, 50, 75])
def test_trained_network_gain(gpu, ctx, quality):
    """The trained network's start against the decoded start on an image it
    was not trained on (seed outside the training range), with the same
    refinement (8 and 24 iterations: steps of a 4-iteration run, the last two
    restarted with steps of a 100-iteration run): the learned path's
    objective is below the decoded path's, both stay feasible, and with 24
    iterations the learned path is within 0.1 % of the plain 50-iteration
    objective while the decoded path is not closer."""
    j = jpeg_of(512, 384, quality, "4:2:0", False, seed=7000 + quality)
    W, H, _ = j.max_rounded()
    net = WS.WarmStartNet.load()
    ctx.compute(3, j.coefs, WEIGHT, PW, 50, W, H)
    e50 = ctx.evaluate()["E"]
    for k in (8, 24):
        sched = dict(step_iterations=4, tail_iterations=2, tail_step_iterations=100)
        ctx.set_warm_start(net)
        try:
            ctx.compute(3, j.coefs, WEIGHT, PW, k, W, H, init_mode=N.ART_INIT_LEARNED, **sched)
            el = ctx.evaluate()
        finally:
            ctx.set_warm_start(None)
        ctx.compute(3, j.coefs, WEIGHT, PW, k, W, H, **sched)
        ed = ctx.evaluate()
        print(f"q{quality} K={k}: E rel to plain 50: learned {el['E'] / e50 - 1:+.2e}, decoded {ed['E'] / e50 - 1:+.2e}")
        assert el["E"] < ed["E"]
        assert el["infeasibility"] <= 1e-3 and ed["infeasibility"] <= 1e-3
        if k == 24:
            assert el["E"] <= e50 * (1 + 1e-3)
