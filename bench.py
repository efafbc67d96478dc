#!/usr/bin/env python
"""Benchmark of the B200 restoration solver (one JSON line on rank 0).

Workloads (``--workload``; seeded synthetic JPEGs, ``artefact_b200.synth``):

* ``1080p`` (default): one plain 50-iteration solve of a 1920x1080 YCbCr
  4:2:0 baseline JPEG at quality 75 (weight 0.3, pweight 0.001), the
  configuration the headline metric is quoted on.
* ``24mp``: 6000x4000 YCbCr 4:4:4 at quality 30, 100 iterations; the working
  set (~1.7 GB) exceeds L2, so the iteration runs against HBM.
* ``batch256``: 256 JPEGs, W, H ~ U[256, 2048] rounded to 16, 4:2:0 or 4:4:4
  with p = 0.5, quality ~ U[20, 90], 50 iterations, solved as one batch.
* ``learned``: 1920x1080 4:2:0 at quality 30/50/75: the learned warm start +
  the fewest refinement iterations whose objective reaches the plain
  50-iteration one (the value), against the plain 50-iteration solve; a fixed
  8-iteration refinement beside it.
* ``network``: the warm-start network's forward pass alone (TFLOP/s).

A step is one solve of the whole workload. Metric: megapixels per second of
real image area.

* value    -- coefficients already in HBM, result planes written to HBM,
              timed per step with CUDA events; L2 flushed (256 MiB write)
              between steps, outside the timed events.
* e2e      -- the same through the public C ABI with host buffers
              (art_context_compute, or art_context_compute_batch), pinned host
              coefficients in and host planes out, copies inside the timed region.
* roofline -- the dominant kernel's algorithmic bytes per launch (its
              sweep of the two-sweep minimum: 8 N + 2 N_c per channel for the
              gradient sweep, 12 N + 2 N_c for the projection) over its mean
              launch time, from CUDA event nodes inside the captured graph,
              taken in a separate pass so they do not perturb `value`; the
              kernel's own I/O bytes beside it.
* iteration -- timed step / iterations against the algorithmic bytes
              sum_c (20 N + 4 N_c) (the two-sweep minimum).
* cpu_baseline -- the oracle (fp32 C restatement of pipeline_scalar) on one
              host thread; a bounded sample, extrapolated when stated; with the
              host's CPU model and core counts.
* --impl reference -- the oracle as the reference arm, steps spread over the
              host's threads, on inputs from the oracle's own JPEG decoder
              (oracle/jpeg_oracle.py): that arm never loads the product library.
* hbm_iteration (1080p run, one GPU) -- the 6000x4000 4:4:4 q30 100-iteration
              solve, whose working set exceeds L2: iteration time and its
              fraction of the measured HBM bandwidth on the algorithmic bytes.
* learned_warm_start (1080p, one GPU) -- the same image through the learned
              warm start: 8 refinement iterations, and the fewest of 8/16/24/32
              that reach the plain 50-iteration objective within 1e-4, with
              their MPix/s (objectives from art_context_evaluate).

Multi-GPU (torchrun): replicas only -- every rank solves its own copy; value
is all ranks' megapixels over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "1080p": dict(name="1920x1080 YCbCr 4:2:0 baseline JPEG q75, plain solver 50 iterations (weight 0.3, pweight 0.001)",
                  metric="MPix/s (plain 50-iteration solve, 1080p 4:2:0 q75)", iterations=50),
    "24mp": dict(name="6000x4000 YCbCr 4:4:4 baseline JPEG q30, plain solver 100 iterations (weight 0.3, pweight 0.001)",
                 metric="MPix/s (plain 100-iteration solve, 6000x4000 4:4:4 q30)", iterations=100),
    "batch256": dict(name="256 JPEGs, W,H~U[256,2048] (x16), 4:2:0|4:4:4 p=.5, q~U[20,90], one batch, 50 iterations",
                     metric="MPix/s (plain 50-iteration batched solve, 256 images)", iterations=50),
    "learned": dict(name="1920x1080 YCbCr 4:2:0 baseline JPEGs at q30/50/75: learned warm start + refinement "
                         "against the plain 50-iteration solve",
                    metric="MPix/s to the plain 50-iteration objective (learned warm start + the fewest refinement "
                           "iterations that reach it, 1080p 4:2:0 q30/50/75)", iterations=8),
}
WORKLOADS["network"] = dict(
    name="warm-start network forward on one 1920x1080 4:2:0 JPEG (joint 4:2:0 pass over the luma's 960x544 level 0; "
         "per component: luma 1920x1088, chroma 2 x 960x544)",
    metric="TFLOP/s (warm-start network forward, 1080p 4:2:0)", iterations=0)
LEARNED_QUALITIES = (30, 50, 75)
REFINE_ITERATIONS = 8
REFINE_STEP_ITERATIONS = 1         # first refinement phase: steps of a 1-iteration run ...
REFINE_STEP_DECAY = 0.9            # ... shrinking by this factor every iteration
REFINE_TAIL = 2                    # runs of at most 12: the last two iterations restart FISTA ...
REFINE_TAIL_STEP_ITERATIONS = 100  # ... with steps of a 100-iteration run
WEIGHT, PWEIGHT = 0.3, 0.001


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic(workload, kernel):
    """DRAM bytes per launch of `kernel` on `workload` from the ncu captures
    summarised in profiles/traffic.txt ("workload kernel bytes" lines), or None."""
    p = ROOT / "profiles" / "traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) == 3 and not line.startswith("#") and parts[0] == workload and parts[1] == kernel:
            return float(parts[2])
    return None


SWEEP_NAMES = {0: "narrow", 1: "wide", 2: "quad"}


def tune_candidates(lib, ctx):
    """Every launch shape the context's last autotune run timed, with its time."""
    from artefact_b200 import _native as N

    n = C.c_uint32()
    N.check(lib.art_context_tune_candidates(ctx, None, 0, C.byref(n)))
    arr = (N.ArtTuneCandidate * max(1, n.value))()
    N.check(lib.art_context_tune_candidates(ctx, arr, n.value, C.byref(n)))
    return [{"sweep": SWEEP_NAMES[c.variant], "rows": c.strip_rows, "projection_warps": c.proj_warps, "ms": c.ms}
            for c in arr[:n.value]]


def host_cpu():
    """Host CPU model, logical CPUs and the CPUs this process may use."""
    model = "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count() or 1
    return {"cpu_model": model, "host_logical_cpus": os.cpu_count() or 1, "host_usable_cpus": usable}


def workload_bytes(kind):
    """Encoded JPEG bytes of the workload's images (seeded synthetic)."""
    from artefact_b200 import synth

    if kind == "1080p":
        return [synth.make_jpeg(1920, 1080, 75, "4:2:0", False, seed=2000)]
    if kind == "24mp":
        return [synth.make_jpeg(6000, 4000, 30, "4:4:4", False, seed=3000)]
    if kind == "learned":
        return [synth.make_jpeg(1920, 1080, q, "4:2:0", False, seed=5000 + q) for q in LEARNED_QUALITIES]
    from concurrent.futures import ThreadPoolExecutor

    specs = synth.batch_specs(256, seed=4000)
    with ThreadPoolExecutor(max_workers=min(32, os.cpu_count() or 1)) as ex:
        return list(ex.map(lambda s: synth.make_jpeg(s.width, s.height, s.quality, s.subsampling, False, s.seed),
                           specs))


def make_workload(kind, keep_bytes=None):
    """List of decoded Jpeg objects for the workload (the product's host
    decoder; their encoded bytes are appended to `keep_bytes` when given)."""
    from artefact_b200.api import Jpeg, JpegSource

    datas = workload_bytes(kind)
    if keep_bytes is not None:
        keep_bytes.extend(datas)
    return [Jpeg.from_source(JpegSource.Buffer(d)) for d in datas]


def workload_config(kind, world):
    """The `config` object of the bench line, the same for both arms."""
    wl = WORKLOADS[kind]
    cfg = {"workload": wl["name"], "iterations": 50 if kind == "learned" else wl["iterations"],
           "images": 256 if kind == "batch256" else (len(LEARNED_QUALITIES) if kind == "learned" else 1),
           "l2": "flushed between steps (256 MiB write outside the timed events)",
           "parallelism": f"replicas x{world}"}
    if kind == "learned":
        cfg["refine_schedule"] = refine_schedule(REFINE_ITERATIONS)
        cfg["refine_iterations"] = REFINE_ITERATIONS
    return cfg


class Clocks:
    """Samples the SM clock and the clock-event reasons while GPU work is timed.

    Reads NVML every 5 ms on a thread (read-only queries), so a timed region of
    a few tens of milliseconds still gets many samples; falls back to
    ``nvidia-smi -lms 100`` when NVML is unavailable."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()
        self.samples = []  # (sm MHz, max sm MHz, set of reason names)
        self.source = "none"

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _nvml_loop(self):
        nv, h = self.nvml
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop.is_set():
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.samples.append((float(sm), float(mx), {n for n, b in bits.items() if r & b}))
            self.stop.wait(0.005)

    def _smi_loop(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm, mx = float(parts[1]), float(parts[2])
            except ValueError:
                continue
            self.samples.append((sm, mx, {n for n, v in zip(self.NAMES, parts[5:9]) if v.lower() == "active"}))

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            self.thread = threading.Thread(target=self._nvml_loop, daemon=True)
            self.source = "nvml 5 ms"
        except Exception:
            self.nvml = None
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                     "--format=csv,noheader,nounits", "-lms", "100"],
                    stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.thread = threading.Thread(target=self._smi_loop, daemon=True)
                self.source = "nvidia-smi 100 ms"
            except Exception:
                return self
        self.thread.start()
        t0 = time.time()
        while not self.samples and time.time() - t0 < 5:
            time.sleep(0.002)
        return self

    def __exit__(self, *exc):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.nvml or self.proc:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "source": self.source}
        reasons = set().union(*[r for _, _, r in self.samples])
        return {"sm_mhz": statistics.median([s for s, _, _ in self.samples]),
                "sm_max_mhz": max(m for _, m, _ in self.samples), "reasons": sorted(reasons),
                "samples": len(self.samples), "source": self.source}


def oracle_solve(jpeg, iterations):
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib

    W, H, _ = jpeg.max_rounded()
    return oracle_lib.compute(jpeg.nchannel, jpeg.coefs, WEIGHT, [PWEIGHT] * 3, iterations, W, H)


class DeviceImage:
    """One decoded JPEG with its coefficients and result planes in HBM."""

    def __init__(self, jpeg):
        import torch

        from artefact_b200 import _native as N

        self.jpeg = jpeg
        self.W, self.H, _ = jpeg.max_rounded()
        self.n = jpeg.nchannel
        self.keep = []
        self.ch = (N.ArtChannel * self.n)()
        for c, co in enumerate(jpeg.coefs):
            dev = torch.from_numpy(co.dct_coefs.copy()).cuda()
            q = np.ascontiguousarray(co.quant_table, np.float32)
            self.keep += [dev, q]
            a = self.ch[c]
            a.rounded_px_w, a.rounded_px_h, a.block_w, a.block_h = co.rounded_px_w, co.rounded_px_h, co.block_w, co.block_h
            a.samp_h, a.samp_v, a.coef_type = co.horizontal_samp_factor, co.vertical_samp_factor, N.ART_COEF_I16
            a.dct_coefs = dev.data_ptr()
            a.quant_table = q.ctypes.data_as(C.POINTER(C.c_float))
        self.pitch = (self.W + 31) // 32 * 32
        self.outs = [torch.empty(self.H, self.pitch, device="cuda") for _ in range(self.n)]
        self.ptrs = (C.c_void_p * self.n)(*[o.data_ptr() for o in self.outs])

    def solve(self, lib, ctx, iterations, init_mode, step_iterations, stream, tail=0, tail_step=0, decay=0.0):
        from artefact_b200 import _native as N

        opts = N.ArtOptions()
        opts.init_mode, opts.device, opts.step_iterations = init_mode, -1, step_iterations
        opts.tail_iterations, opts.tail_step_iterations, opts.step_decay = tail, tail_step, decay
        pw = (C.c_float * 3)(PWEIGHT, PWEIGHT, PWEIGHT)
        N.check(lib.art_context_compute_device(ctx, self.n, self.ch, WEIGHT, pw, iterations, self.W, self.H,
                                               self.ptrs, self.pitch, C.byref(opts), C.c_void_p(stream.cuda_stream)))


def refine_schedule(k):
    """Refinement after a learned start: k plain iterations whose step starts
    at that of a REFINE_STEP_ITERATIONS-iteration run and shrinks by
    REFINE_STEP_DECAY every iteration (large steps remove the prediction's
    error, the shrinking lets the iterate settle); runs of at most 12 end with
    REFINE_TAIL iterations restarted with the step of a
    REFINE_TAIL_STEP_ITERATIONS-iteration run. Chosen on a grid over the
    1080p evaluation images and six held-out ones (first-phase step of a 1-8
    iteration run, decay 0, 0.8 or 0.9, tails of 0 or 2 iterations at 100- or
    300-iteration steps)."""
    return dict(step=REFINE_STEP_ITERATIONS, decay=REFINE_STEP_DECAY, tail=min(REFINE_TAIL, k - 1) if k <= 12 else 0,
                tail_step=REFINE_TAIL_STEP_ITERATIONS)


def learned_comparison(lib, device, steps, warmup, refine=REFINE_ITERATIONS, qualities=LEARNED_QUALITIES,
                       images=None, ladder=(8, 12, 16, 20, 24, 28, 32, 40, 48)):
    """Learned warm start + `refine` plain iterations against the plain
    50-iteration solve, per quality, on seeded 1920x1080 4:2:0 JPEGs (seeds
    5000 + quality, outside the network's training seeds). Each path is timed
    from device-resident coefficients to device-resident planes (CUDA events,
    L2 flushed between steps); its objective and feasibility come from
    art_context_evaluate. Also finds the fewest refinement iterations (of a
    fixed ladder) whose objective reaches the plain 50-iteration one within
    1e-4 relative, and times that. The decoded start with the same schedule
    is the control. `images` (a list of (label, Jpeg)) replaces the seeded
    1080p images. None when the package holds no trained weights."""
    import torch

    from artefact_b200 import _native as N
    from artefact_b200 import synth
    from artefact_b200 import warmstart as WS
    from artefact_b200.api import Jpeg, JpegSource

    if not WS.DEFAULT_WEIGHTS.exists():
        return None
    net = WS.WarmStartNet.load(device=device)
    ctx = C.c_void_p()
    N.check(lib.art_context_create(device, C.byref(ctx)))
    N.check(lib.art_context_set_warm_start(ctx, net.handle))
    joint = WS.WarmStartNet.load(WS.DEFAULT_JOINT_WEIGHTS, device) if WS.DEFAULT_JOINT_WEIGHTS.exists() else None
    if joint is not None:
        N.check(lib.art_context_set_joint_warm_start(ctx, joint.handle))
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def evaluate():
        out = (C.c_double * 5)()
        N.check(lib.art_context_evaluate(ctx, 0, out))
        return out[0], out[4]

    def run(img, its, mode, sched):
        if sched is None:
            img.solve(lib, ctx, its, mode, 0, stream)
        else:
            img.solve(lib, ctx, its, mode, sched["step"], stream, sched["tail"], sched["tail_step"], sched["decay"])

    def timed(img, its, mode, sched):
        for _ in range(warmup):
            flush.fill_(1.0)
            run(img, its, mode, sched)
        torch.cuda.synchronize()
        ms = []
        for k in range(steps):
            flush.fill_(float(k))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            run(img, its, mode, sched)
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        N.check(lib.art_context_synchronize(ctx))
        return statistics.median(ms)

    rows = []
    if images is None:
        images = [(q, Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(1920, 1080, q, "4:2:0", False, seed=5000 + q))))
                  for q in qualities]
    for q, j in images:
        img = DeviceImage(j)
        mpix = j.real_px_w * j.real_px_h / 1e6
        plain_ms = timed(img, 50, N.ART_INIT_DECODED, None)
        e50, f50 = evaluate()
        sched = refine_schedule(refine)
        learned_ms = timed(img, refine, N.ART_INIT_LEARNED, sched)
        el, fl = evaluate()
        run(img, refine, N.ART_INIT_DECODED, sched)
        ed, _ = evaluate()
        run(img, refine, N.ART_INIT_LEARNED, None)
        el_plain_step = evaluate()[0]
        run(img, 0, N.ART_INIT_LEARNED, None)
        e_start = evaluate()[0]
        kmin, ek_min, fk_min = None, None, None
        for k in ladder:
            run(img, k, N.ART_INIT_LEARNED, refine_schedule(k))
            ek, fk = evaluate()
            if ek <= e50 * (1 + 1e-4) and fk <= 1e-3:
                kmin, ek_min, fk_min = k, ek, fk
                break
        kmin_ms = timed(img, kmin, N.ART_INIT_LEARNED, refine_schedule(kmin)) if kmin else None
        dk = None
        if kmin:
            run(img, kmin, N.ART_INIT_DECODED, refine_schedule(kmin))
            dk = (evaluate()[0] - e50) / e50
        rows.append(dict(quality=q, plain50_ms=plain_ms, plain50_mpix_s=mpix / plain_ms * 1e3,
                         learned_ms=learned_ms, learned_mpix_s=mpix / learned_ms * 1e3,
                         speedup=plain_ms / learned_ms, E_plain50=e50, E_learned=el,
                         E_learned_rel=(el - e50) / e50, E_decoded_same_schedule_rel=(ed - e50) / e50,
                         E_learned_single_phase_rel=(el_plain_step - e50) / e50,
                         E_after_projection_only_rel=(e_start - e50) / e50,
                         infeasibility_learned=fl, infeasibility_plain=f50,
                         reaches_plain50=bool(el <= e50 * (1 + 1e-4) and fl <= 1e-3),
                         min_refine_to_reach=kmin,
                         min_refine_E_rel=((ek_min - e50) / e50) if kmin else None,
                         min_refine_infeasibility=fk_min,
                         min_refine_decoded_same_schedule_E_rel=dk,
                         min_refine_ms=kmin_ms, min_refine_speedup=(plain_ms / kmin_ms) if kmin_ms else None))
        log(f"learned q{q}: plain50 {plain_ms:.3f} ms E {e50:.7g}; learned+{refine} {learned_ms:.3f} ms "
            f"E {(el - e50) / e50:+.2e} (decoded start, same schedule {(ed - e50) / e50:+.2e}); "
            f"reaches at K={kmin} in {kmin_ms} ms")
    lib.art_context_set_warm_start(ctx, None)
    lib.art_context_set_joint_warm_start(ctx, None)
    lib.art_context_destroy(ctx)
    net.close()
    if joint is not None:
        joint.close()
    mp_total = sum(j.real_px_w * j.real_px_h / 1e6 for _, j in images)
    reach = all(r["min_refine_to_reach"] for r in rows)
    return dict(refine_iterations=refine, schedule=refine_schedule(refine), images=rows,
                network=("joint 4:2:0 (one pass, all three components at full resolution)" if joint is not None
                         else "per component"),
                plain50_mpix_s=mp_total / sum(r["plain50_ms"] for r in rows) * 1e3,
                learned_mpix_s=mp_total / sum(r["learned_ms"] for r in rows) * 1e3,
                all_reach_plain50=all(r["reaches_plain50"] for r in rows),
                reach_mpix_s=(mp_total / sum(r["min_refine_ms"] for r in rows) * 1e3) if reach else None)


def iteration_bytes(jpegs):
    """Algorithmic bytes of one iteration, sum over images and channels of
    20 N + 4 N_c (the two-sweep minimum: read x_k, x_{k-1} and the int16
    coefficients twice, write x_{k+1})."""
    total = 0
    for j in jpegs:
        W, H, _ = j.max_rounded()
        total += sum(20 * W * H + 4 * co.rounded_px_w * co.rounded_px_h for co in j.coefs)
    return total


def hbm_iteration(lib, device, steps, warmup, peak):
    """The HBM-bound configuration inside the default run: one 6000x4000
    4:4:4 q30 image, 100 plain iterations (its ~1.3 GB working set exceeds
    L2). Whole solves timed with CUDA events (L2 flushed between them), the
    iteration as solve time / 100 against the algorithmic bytes, and the two
    kernels' mean launch times from the graph's event nodes (separate pass)."""
    import torch

    from artefact_b200 import _native as N

    jpegs = make_workload("24mp")
    j = jpegs[0]
    iters = WORKLOADS["24mp"]["iterations"]
    img = DeviceImage(j)
    from artefact_b200.api import Context

    context = Context(device)
    ctx = context.handle
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # Autotune on the image itself (10 iterations per candidate).
    tr = context.autotune_batch([dict(coefs=j.coefs, weight=WEIGHT, pweight=[PWEIGHT] * 3)], 10)
    tuned = {"sweep_variant": SWEEP_NAMES[tr["variant"]], "strip_rows": tr["strip_rows"],
             "projection_warps": tr["proj_warps"], "tuned_ms_per_10_iterations": tr["best_ms"],
             "heuristic_ms_per_10_iterations": tr["heuristic_ms"],
             "candidates_ms_per_10_iterations": [
                 {"sweep": SWEEP_NAMES[k], "rows": r, "projection_warps": p, "ms": m} for k, r, p, m in tr["candidates_ms"]]}
    for _ in range(warmup):
        img.solve(lib, ctx, iters, N.ART_INIT_DECODED, 0, stream)
    torch.cuda.synchronize()
    ms = []
    for k in range(steps):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        img.solve(lib, ctx, iters, N.ART_INIT_DECODED, 0, stream)
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    N.check(lib.art_context_synchronize(ctx))
    N.check(lib.art_context_set_timing(ctx, 1))
    lm, gm, um, nl = C.c_float(), C.c_float(), C.c_float(), C.c_uint32()
    gs, us = [], []
    for k in range(2):
        flush.fill_(float(k))
        img.solve(lib, ctx, iters, N.ART_INIT_DECODED, 0, stream)
        N.check(lib.art_context_synchronize(ctx))
        N.check(lib.art_context_last_timing(ctx, C.byref(lm), C.byref(gm), C.byref(um), C.byref(nl)))
        gs.append(gm.value / iters)
        us.append(um.value / iters)
    N.check(lib.art_context_set_timing(ctx, 0))
    context.close()
    solve_ms = statistics.median(ms)
    it_ms = solve_ms / iters
    ib = iteration_bytes(jpegs)
    W, H, _ = j.max_rounded()
    moved = sum(28 * W * H + 10 * co.rounded_px_w * co.rounded_px_h for co in j.coefs)
    return {"workload": WORKLOADS["24mp"]["name"], "solve_ms": solve_ms, "steps": steps,
            "mpix_s": j.real_px_w * j.real_px_h / 1e6 / solve_ms * 1e3,
            "iteration_ms": it_ms, "algorithmic_bytes_per_iteration": ib,
            "gbs": ib / (it_ms * 1e-3) / 1e9, "frac_of_hbm": ib / (it_ms * 1e-3) / 1e9 / peak,
            "bytes_moved_per_iteration": moved, "moved_gbs": moved / (it_ms * 1e-3) / 1e9,
            "gradient_launch_ms": statistics.mean(gs), "projection_launch_ms": statistics.mean(us), "autotuned": tuned,
            "source": "whole 100-iteration solves, CUDA events, L2 flushed between solves; iteration = solve / 100"}


def batch_block(lib, device, steps, warmup, peak):
    """The 256-image batch inside the default run: its device-resident batched
    solve (CUDA events, L2 flushed between solves, 50 iterations), the
    iteration against the algorithmic bytes, and JPEG bytes -> RGB8 through
    the decode pipeline (batched solves)."""
    import torch

    from artefact_b200 import _native as N

    encoded = []
    jpegs = make_workload("batch256", encoded)
    iters = WORKLOADS["batch256"]["iterations"]
    keep = []
    imgs = (N.ArtImage * len(jpegs))()
    for i, j in enumerate(jpegs):
        W, H, _ = j.max_rounded()
        n = j.nchannel
        cd = (N.ArtChannel * n)()
        for c, co in enumerate(j.coefs):
            dev = torch.from_numpy(co.dct_coefs.copy()).cuda()
            q = np.ascontiguousarray(co.quant_table, np.float32)
            keep += [dev, q]
            a = cd[c]
            a.rounded_px_w, a.rounded_px_h, a.block_w, a.block_h = co.rounded_px_w, co.rounded_px_h, co.block_w, co.block_h
            a.samp_h, a.samp_v, a.coef_type = co.horizontal_samp_factor, co.vertical_samp_factor, N.ART_COEF_I16
            a.dct_coefs = dev.data_ptr()
            a.quant_table = q.ctypes.data_as(C.POINTER(C.c_float))
        pitch = (W + 31) // 32 * 32
        outs = [torch.empty(H, pitch, device="cuda") for _ in range(n)]
        ptrs = (C.c_void_p * n)(*[o.data_ptr() for o in outs])
        keep += [cd, outs, ptrs]
        im = imgs[i]
        im.nchannel, im.max_rounded_px_w, im.max_rounded_px_h, im.out_pitch = n, W, H, pitch
        im.channels = C.cast(cd, C.POINTER(N.ArtChannel))
        im.weight = WEIGHT
        im.pweight = (C.c_float * 3)(PWEIGHT, PWEIGHT, PWEIGHT)
        im.out_planes = C.cast(ptrs, C.POINTER(C.c_void_p))
    from artefact_b200.api import Context

    context = Context(device)
    ctx = context.handle
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # Autotune on the batch itself (host coefficients, 5 iterations per candidate).
    tr = context.autotune_batch([dict(coefs=j.coefs, weight=WEIGHT, pweight=[PWEIGHT] * 3) for j in jpegs], 5)
    tuned = {"sweep_variant": SWEEP_NAMES[tr["variant"]], "strip_rows": tr["strip_rows"],
             "projection_warps": tr["proj_warps"], "candidates": tr["candidates"],
             "tuned_ms_per_5_iterations": tr["best_ms"], "heuristic_ms_per_5_iterations": tr["heuristic_ms"],
             "candidates_ms_per_5_iterations": [
                 {"sweep": SWEEP_NAMES[k], "rows": r, "projection_warps": p, "ms": m} for k, r, p, m in tr["candidates_ms"]]}

    def solve():
        N.check(lib.art_context_compute_batch_device(ctx, len(jpegs), imgs, iters, None, C.c_void_p(stream.cuda_stream)))

    for _ in range(warmup):
        solve()
    torch.cuda.synchronize()
    ms = []
    for k in range(steps):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        solve()
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    N.check(lib.art_context_synchronize(ctx))
    context.close()
    del keep, flush
    torch.cuda.empty_cache()
    mpix = sum(j.real_px_w * j.real_px_h for j in jpegs) / 1e6
    solve_ms = statistics.median(ms)
    ib = iteration_bytes(jpegs)
    it_ms = solve_ms / iters
    pipe = pipeline_e2e(encoded, iters, device)
    return {"workload": WORKLOADS["batch256"]["name"], "images": len(jpegs), "mpix": mpix, "solve_ms": solve_ms,
            "steps": steps, "mpix_s": mpix / solve_ms * 1e3, "iteration_ms": it_ms,
            "algorithmic_bytes_per_iteration": ib, "gbs": ib / (it_ms * 1e-3) / 1e9,
            "frac_of_hbm": ib / (it_ms * 1e-3) / 1e9 / peak,
            "source": "device-resident batched solves (art_context_compute_batch_device), CUDA events, L2 flushed "
                      "between solves; iteration = solve / 50",
            "autotuned": tuned,
            "decode_pipeline": pipe}


def network_flops(H, W):
    """Multiply-add FLOPs (x2) of one forward pass of the warm-start network
    on an H x W component, as executed: its first level is H0 x W0 =
    ceil(H / 16) * 8 x ceil(W / 16) * 8 (2x2 cells of samples per pixel), input
    features padded to 16 channels, head to 16 outputs."""
    H0, W0 = (H + 15) // 16 * 8, (W + 15) // 16 * 8
    P0, P1, P2, P3 = H0 * W0, (H0 // 2) * (W0 // 2), (H0 // 4) * (W0 // 4), (H0 // 8) * (W0 // 8)
    macs = 9 * (16 * 32 * P0 + 32 * 64 * P1 + 64 * 96 * P2 + 96 * 128 * P3 + 224 * 96 * P2 + 160 * 64 * P1
                + 96 * 32 * P0 + 32 * 16 * P0)
    return 2 * macs


def time_network(device, steps, warmup, joint=False):
    """The network's forward pass on one 1080p 4:2:0 image, CUDA events:
    (ms, TFLOP/s, FLOP). Per component: luma 1920x1088, then both chroma
    planes of 960x544 as a batch of two; joint: one pass over the luma's
    level-0 grid predicting all three components (the joint 4:2:0 network)."""
    import torch

    from artefact_b200 import synth
    from artefact_b200 import warmstart as WS
    from artefact_b200.api import Jpeg, JpegSource

    j = Jpeg.from_source(JpegSource.Buffer(synth.make_jpeg(1920, 1080, 50, "4:2:0", False, seed=5050)))
    if joint:
        net = WS.WarmStartNet.load(WS.DEFAULT_JOINT_WEIGHTS, device)
        cy = torch.from_numpy(WS.coef_image(j.coefs[0])[None]).cuda()
        cc = torch.from_numpy(np.stack([WS.coef_image(co) for co in j.coefs[1:]])[None]).cuda()
        qy = torch.from_numpy(np.asarray(j.coefs[0].quant_table, np.float32)[None].copy()).cuda()
        qc = torch.from_numpy(np.stack([np.asarray(co.quant_table, np.float32) for co in j.coefs[1:]])[None]).cuda()
        flops = network_flops(cy.shape[1], cy.shape[2])
        out = net.predict_joint(cy, cc, qy, qc)
        for _ in range(warmup):
            net.predict_joint(cy, cc, qy, qc, out=out)
        torch.cuda.synchronize()
        ms = []
        for _ in range(steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            net.predict_joint(cy, cc, qy, qc, out=out)
            b.record()
            b.synchronize()
            ms.append(a.elapsed_time(b))
        net.close()
        t = statistics.median(ms)
        return t, flops / (t * 1e-3) / 1e12, flops
    net = WS.WarmStartNet.load(device=device) if WS.DEFAULT_WEIGHTS.exists() else WS.WarmStartNet(device=device)
    groups = [[j.coefs[0]], j.coefs[1:]]
    inputs = []
    flops = 0
    for g in groups:
        c = torch.from_numpy(np.stack([WS.coef_image(co) for co in g])).cuda()
        q = torch.from_numpy(np.stack([np.asarray(co.quant_table, np.float32) for co in g])).cuda()
        inputs.append((c, q))
        flops += len(g) * network_flops(c.shape[1], c.shape[2])
    outs = [net.predict(c, q) for c, q in inputs]
    for _ in range(warmup):
        for (c, q), o in zip(inputs, outs):
            net.predict(c, q, out=o)
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for (c, q), o in zip(inputs, outs):
            net.predict(c, q, out=o)
        b.record()
        b.synchronize()
        ms.append(a.elapsed_time(b))
    net.close()
    t = statistics.median(ms)
    return t, flops / (t * 1e-3) / 1e12, flops


def WS_joint_weights_exist():
    from artefact_b200 import warmstart as WS

    return WS.DEFAULT_JOINT_WEIGHTS.exists()


def run_learned(args, lib, local, rank, world, dist):
    """Config 5: learned warm start + the fewest refinement iterations that reach
    the plain 50-iteration objective, against the plain 50-iteration solve (the
    fixed 8-iteration refinement is reported beside it)."""
    import torch

    wl = WORKLOADS["learned"]
    with Clocks(local) as clk:
        res = learned_comparison(lib, local, args.steps, args.warmup)
    if res is None:
        if rank == 0:
            print(json.dumps({"metric": wl["metric"], "unavailable": "no trained warm-start weights in the package"}))
        return
    net_ms, net_tflops, net_flops = time_network(local, args.steps, args.warmup,
                                                 joint=WS_joint_weights_exist())
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    tc_peak = float(peaks.get("bf16_tflops", 1590.0))
    # The headline: each image solved to the plain 50-iteration objective
    # (learned start + the fewest ladder iterations that reach it). The fixed
    # 8-iteration refinement, which stops short of that objective, is
    # reported beside it.
    reach = all(r["min_refine_ms"] for r in res["images"])
    total_ms = sum(r["min_refine_ms"] for r in res["images"]) if reach else float("nan")
    k8_ms = sum(r["learned_ms"] for r in res["images"])
    if dist:
        t = torch.tensor([total_ms, k8_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, k8_ms = float(t[0].item()), float(t[1].item())
    mpix = world * len(res["images"]) * 1920 * 1080 / 1e6
    value = mpix / (total_ms * 1e-3) if reach else None
    k8 = mpix / (k8_ms * 1e-3)
    if rank == 0:
        line = {
            "metric": wl["metric"], "value": value, "unit": "MPix/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": (total_ms / len(res["images"])) if reach else None,
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 solver, bf16 network (fp32 accumulation)",
            "data": "synthetic",
            "config": workload_config("learned", world),
            "plain50_mpix_s": res["plain50_mpix_s"],
            "speedup_vs_plain50": (value / res["plain50_mpix_s"]) if value else None,
            "refine_iterations_to_reach": [r["min_refine_to_reach"] for r in res["images"]],
            "fixed_refine": {"iterations": res["refine_iterations"], "mpix_s": k8,
                             "speedup_vs_plain50": k8 / res["plain50_mpix_s"],
                             "all_reach_plain50": res["all_reach_plain50"],
                             "max_E_rel_to_plain50": max(r["E_learned_rel"] for r in res["images"])},
            "images": res["images"],
            "roofline": {"bound": "tensor", "kernel": "warm-start network forward (k_conv3x3 and glue)",
                         "achieved": net_tflops, "peak": tc_peak, "unit": "TFLOP/s", "frac": net_tflops / tc_peak,
                         "traffic": None, "peak_kind": "measured" if peaks else "fallback",
                         "algorithmic_flops_per_launch": net_flops, "launch_ms": net_ms},
            "e2e": None, "cpu_baseline": None, "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)


def pipeline_e2e(datas, iterations, device):
    """JPEG bytes to RGB8 for every image of the workload through
    Artefact::process semantics, host decode included: one image after the
    other (decode, then process_jpeg), and overlapped (artefact_b200.pipeline:
    host threads for decoding -- all but two, at most 16 -- and 2 solver
    contexts). Wall clock, MPix/s of real area."""
    from artefact_b200 import process_jpeg
    from artefact_b200.api import Context, Jpeg, JpegSource
    from artefact_b200.pipeline import process_stream

    mpix = 0.0
    ctx = Context(device)
    for d in datas[:4]:  # warm-up: buffers and graphs for the first shapes
        process_jpeg(Jpeg.from_source(JpegSource.Buffer(d)), [WEIGHT] * 3, [PWEIGHT] * 3, [iterations] * 3, False,
                     context=ctx)
    t = time.perf_counter()
    for d in datas:
        j = Jpeg.from_source(JpegSource.Buffer(d))
        mpix += j.real_px_w * j.real_px_h / 1e6
        process_jpeg(j, [WEIGHT] * 3, [PWEIGHT] * 3, [iterations] * 3, False, context=ctx)
    serial = time.perf_counter() - t
    ctx.close()
    decoders = max(1, min(16, (os.cpu_count() or 4) - 2))
    batch_images, batch_pixels, solvers = 32, 32 << 20, 2
    # Two solver contexts kept across streams, as a long-running server keeps
    # them: one untimed pass over the stream sizes their buffers and captures
    # their graphs, then the timed pass.
    contexts = [Context(device) for _ in range(solvers)]
    stream = lambda: process_stream(datas, [WEIGHT] * 3, [PWEIGHT] * 3, [iterations] * 3, decoders=decoders,
                                    solvers=solvers, batch_images=batch_images, batch_pixels=batch_pixels,
                                    device=device, contexts=contexts)
    sum(1 for _ in stream())
    t = time.perf_counter()
    n = sum(1 for _ in stream())
    piped = time.perf_counter() - t
    for c in contexts:
        c.close()
    assert n == len(datas)
    # Host decode alone on the same threads, for the bound it sets.
    from concurrent.futures import ThreadPoolExecutor

    t = time.perf_counter()
    with ThreadPoolExecutor(decoders) as ex:
        list(ex.map(lambda d: Jpeg.from_source(JpegSource.Buffer(d)), datas))
    decode = time.perf_counter() - t
    return {"serial_mpix_s": mpix / serial, "pipelined_mpix_s": mpix / piped, "images": len(datas),
            "decode_only_mpix_s": mpix / decode, "decoders": decoders, "solver_contexts": solvers,
            "batch_images": batch_images, "batch_pixels": batch_pixels,
            "what": "JPEG bytes -> RGB8 (host decode, H2D, batched solve, RGB, D2H), wall clock, the second of two "
                    "passes over the stream on the same two contexts; serial = one image after the other through "
                    "process_jpeg"}


def cpu_sample(kind, jpegs, iterations):
    """Bounded CPU measurement of the oracle: (MPix/s, description)."""
    real = sum(j.real_px_w * j.real_px_h for j in jpegs) / 1e6
    if kind == "1080p":
        t = time.perf_counter()
        oracle_solve(jpegs[0], iterations)
        return real / (time.perf_counter() - t), "one full solve of the workload by the fp32 C restatement of pipeline_scalar"
    if kind == "24mp":
        t = time.perf_counter()
        oracle_solve(jpegs[0], 0)
        t_init = time.perf_counter() - t
        t = time.perf_counter()
        oracle_solve(jpegs[0], 2)
        t_iter = (time.perf_counter() - t - t_init) / 2
        total = t_init + iterations * t_iter
        return real / total, (f"init alone and a 2-iteration solve of the full image, extrapolated to {iterations} "
                              f"iterations ({t_init:.1f} s + {iterations} x {t_iter:.2f} s)")
    sample = jpegs[:4]
    t = time.perf_counter()
    for j in sample:
        oracle_solve(j, iterations)
    dt = time.perf_counter() - t
    px = sum(j.real_px_w * j.real_px_h for j in sample) / 1e6
    return px / dt, f"the first 4 images of the batch ({px:.2f} MPix), {iterations} iterations each"


def run_reference(args, rank, world):
    """Reference arm: the oracle port of pipeline_scalar on the host cores.

    Its inputs come from the oracle's own JPEG decoder (oracle/jpeg_oracle.py)
    on the same seeded JPEG bytes as the GPU arm, so this arm never loads the
    product library; only the oracle runs in its timed region."""
    if rank != 0:
        return
    from concurrent.futures import ThreadPoolExecutor

    wl = WORKLOADS[args.workload]
    if args.workload == "network":
        print(json.dumps({"impl": "reference", "metric": wl["metric"],
                          "unavailable": "the warm-start network has no counterpart in the reference"}), flush=True)
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import jpeg_oracle

    jpegs = [jpeg_oracle.decode(d) for d in workload_bytes(args.workload)]
    iters = 50 if args.workload == "learned" else wl["iterations"]
    cpu = host_cpu()
    threads = max(1, min(cpu["host_usable_cpus"], 64))
    if args.workload in ("1080p", "learned"):
        # Full solves: one image per step (the three qualities in turn for the
        # learned workload, which the reference solves with plain iterations).
        work = [jpegs[k % len(jpegs)] for k in range(args.steps)]
        warm = [jpegs[k % len(jpegs)] for k in range(min(args.warmup, threads))]
        sample = f"{args.steps} full {iters}-iteration solves of the workload's images spread over {threads} host threads"
    else:
        # Bounded: one image-solve per step (the batch's first images, or a
        # 4-iteration solve of the 24 MP image scaled per iteration).
        work = jpegs[:args.steps] if args.workload == "batch256" else [jpegs[0]] * min(args.steps, 4)
        warm = []
        sample = f"{len(work)} image solves of the workload spread over {threads} host threads"
    mpix = sum(j.real_px_w * j.real_px_h for j in work) / 1e6
    its = iters if args.workload != "24mp" else 4
    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(lambda j: oracle_solve(j, its), warm))
        t0 = time.perf_counter()
        list(ex.map(lambda j: oracle_solve(j, its), work))
        dt = time.perf_counter() - t0
    if args.workload == "24mp":
        dt *= iters / its  # per-iteration cost scaled to the full solve
        sample += f" at {its} iterations, scaled to {iters}"
    value = mpix / dt
    line = {
        "impl": "reference", "metric": wl["metric"], "value": value, "unit": "MPix/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(1, len(work)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.workload, world),
        "cpu_baseline": {"value": value, "unit": "MPix/s", "cores": threads, "kind": "port", **cpu,
                         "sample": sample + " (fp32 C restatement of pipeline_scalar, inputs from the oracle's JPEG "
                                            "decoder; the Rust reference is not buildable here)"},
        "e2e": {"value": value, "unit": "MPix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="1080p", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start comparison")
    ap.add_argument("--no-hbm", action="store_true", help="skip the 6000x4000 HBM iteration block of the default run")
    ap.add_argument("--no-batch", action="store_true", help="skip the 256-image batch block of the default run")
    ap.add_argument("--no-tune", action="store_true", help="solve with the size heuristic's launch shapes")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod

    from artefact_b200 import _native as N

    lib = N.lib()
    wl = WORKLOADS[args.workload]
    if args.workload == "learned":
        run_learned(args, lib, local, rank, world, dist)
        return
    if args.workload == "network":
        # The network the learned start uses on this workload's 4:2:0 image:
        # the joint one when it ships, with the per-component passes beside it.
        joint = WS_joint_weights_exist()
        ms, tflops, flops = time_network(local, args.steps, args.warmup, joint=joint)
        other = time_network(local, args.steps, args.warmup, joint=False) if joint else None
        if rank == 0:
            peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
            peak = float(peaks.get("bf16_tflops", 1590.0))
            print(json.dumps({"metric": wl["metric"], "value": tflops, "unit": "TFLOP/s", "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None, "dtype": "bf16 (fp32 accumulation)",
                              "data": "synthetic", "config": workload_config("network", world),
                              "roofline": {"bound": "tensor", "achieved": tflops, "peak": peak, "unit": "TFLOP/s",
                                           "frac": tflops / peak, "traffic": None,
                                           "peak_kind": "measured" if peaks else "fallback",
                                           "algorithmic_flops_per_launch": flops, "launch_ms": ms},
                              "network": "joint 4:2:0" if joint else "per component",
                              "per_component_forward": ({"ms": other[0], "tflops": other[1], "gflop": other[2] / 1e9}
                                                        if other else None)}), flush=True)
        return
    iters = wl["iterations"]
    encoded = []
    jpegs = make_workload(args.workload, encoded)
    nimg = len(jpegs)
    mpix = sum(j.real_px_w * j.real_px_h for j in jpegs) / 1e6

    keep = []
    imgs_dev = (N.ArtImage * nimg)()
    imgs_host = (N.ArtImage * nimg)()
    pw = (C.c_float * 3)(PWEIGHT, PWEIGHT, PWEIGHT)
    h2d = d2h = 0
    for i, j in enumerate(jpegs):
        W, H, _ = j.max_rounded()
        n = j.nchannel
        cd = (N.ArtChannel * n)()
        ch_ = (N.ArtChannel * n)()
        for c, co in enumerate(j.coefs):
            dev = torch.from_numpy(co.dct_coefs.copy()).cuda()
            pin = torch.from_numpy(co.dct_coefs.copy()).pin_memory()
            q = np.ascontiguousarray(co.quant_table, np.float32)
            keep += [dev, pin, q]
            h2d += co.dct_coefs.nbytes
            for arr, ptr in ((cd, dev.data_ptr()), (ch_, pin.data_ptr())):
                a = arr[c]
                a.rounded_px_w, a.rounded_px_h, a.block_w, a.block_h = co.rounded_px_w, co.rounded_px_h, co.block_w, co.block_h
                a.samp_h, a.samp_v, a.coef_type = co.horizontal_samp_factor, co.vertical_samp_factor, N.ART_COEF_I16
                a.dct_coefs = ptr
                a.quant_table = q.ctypes.data_as(C.POINTER(C.c_float))
        pitch = (W + 31) // 32 * 32
        douts = [torch.empty(H, pitch, device="cuda") for _ in range(n)]
        houts = [torch.empty(W * H, dtype=torch.float32).pin_memory() for _ in range(n)]
        d2h += n * W * H * 4
        dptr = (C.c_void_p * n)(*[o.data_ptr() for o in douts])
        hptr = (C.c_void_p * n)(*[o.data_ptr() for o in houts])
        keep += [cd, ch_, douts, houts, dptr, hptr]
        for arr, chans, ptrs, op in ((imgs_dev, cd, dptr, pitch), (imgs_host, ch_, hptr, W)):
            im = arr[i]
            im.nchannel, im.max_rounded_px_w, im.max_rounded_px_h, im.out_pitch = n, W, H, op
            im.channels = C.cast(chans, C.POINTER(N.ArtChannel))
            im.weight = WEIGHT
            im.pweight = (C.c_float * 3)(PWEIGHT, PWEIGHT, PWEIGHT)
            im.out_planes = C.cast(ptrs, C.POINTER(C.c_void_p))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    ctx = C.c_void_p()
    N.check(lib.art_context_create(local, C.byref(ctx)))
    stream = torch.cuda.current_stream()
    # Autotune the launch shapes on the workload itself (10 iterations per
    # candidate, host coefficients); the solves below use the choice.
    tuned = None
    if not args.no_tune:
        tr = N.ArtTuneResult()
        N.check(lib.art_context_autotune_batch(ctx, nimg, imgs_host, 10, C.byref(tr)))
        tuned = {"sweep_variant": SWEEP_NAMES[tr.variant], "strip_rows": tr.strip_rows,
                 "projection_warps": tr.proj_warps, "candidates": tr.candidates,
                 "tuned_ms_per_10_iterations": tr.best_ms, "heuristic_ms_per_10_iterations": tr.heuristic_ms,
                 "heuristic": {"sweep_variant": SWEEP_NAMES[tr.heuristic_variant],
                               "strip_rows": tr.heuristic_strip_rows, "projection_warps": 4},
                 "candidates_ms_per_10_iterations": tune_candidates(lib, ctx)}

    def solve_device():
        if nimg == 1:
            im = imgs_dev[0]
            N.check(lib.art_context_compute_device(ctx, im.nchannel, im.channels, WEIGHT, pw, iters,
                                                   im.max_rounded_px_w, im.max_rounded_px_h, im.out_planes,
                                                   im.out_pitch, None, C.c_void_p(stream.cuda_stream)))
        else:
            N.check(lib.art_context_compute_batch_device(ctx, nimg, imgs_dev, iters, None,
                                                         C.c_void_p(stream.cuda_stream)))

    def solve_host():
        if nimg == 1:
            im = imgs_host[0]
            N.check(lib.art_context_compute(ctx, im.nchannel, im.channels, WEIGHT, pw, iters, im.max_rounded_px_w,
                                            im.max_rounded_px_h, im.out_planes, None))
        else:
            N.check(lib.art_context_compute_batch(ctx, nimg, imgs_host, iters, None))

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        flush.fill_(1.0)
        solve_device()
    torch.cuda.synchronize()
    N.check(lib.art_context_synchronize(ctx))

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    with Clocks(local) as clk:
        t0 = time.perf_counter()
        for k in range(args.steps):
            flush.fill_(float(k))
            starts[k].record(stream)
            solve_device()
            ends[k].record(stream)
        barrier()
        wall = time.perf_counter() - t0
        N.check(lib.art_context_synchronize(ctx))
        step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
        total_ms = sum(step_ms)
        if dist:
            t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total_ms = float(t.item())
        value = world * args.steps * mpix / (total_ms / 1e3)

        # Kernel timing pass (event nodes inside the graph).
        N.check(lib.art_context_set_timing(ctx, 1))
        grad_ms, upd_ms, loop_ms = [], [], []
        lm, gm, um, nl = C.c_float(), C.c_float(), C.c_float(), C.c_uint32()
        for k in range(4):
            flush.fill_(float(k))
            solve_device()
            N.check(lib.art_context_synchronize(ctx))
            N.check(lib.art_context_last_timing(ctx, C.byref(lm), C.byref(gm), C.byref(um), C.byref(nl)))
            if k > 0:
                loop_ms.append(lm.value)
                grad_ms.append(gm.value)
                upd_ms.append(um.value)
        N.check(lib.art_context_set_timing(ctx, 0))
    clocks = clk.summary()

    # e2e through the public API with host buffers.
    for _ in range(max(1, args.warmup // 2)):
        solve_host()
    barrier()
    e2e_ms = []
    e2e_steps = min(args.steps, 10)
    for k in range(e2e_steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        solve_host()
        e2e_ms.append((time.perf_counter() - t1) * 1e3)
    e2e_total = sum(e2e_ms)
    if dist:
        t = torch.tensor([e2e_total], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * e2e_steps * mpix / (e2e_total / 1e3)

    it_ms = total_ms / args.steps / iters
    g_launch = statistics.mean(grad_ms) / iters
    u_launch = statistics.mean(upd_ms) / iters
    loop = statistics.mean(loop_ms)
    # Algorithmic bytes per launch (summed over the workload's images), the
    # two-sweep minimum per kernel: the gradient sweep reads x_k, x_{k-1} and
    # the int16 coefficients (8 N + 2 N_c per channel), the projection the same
    # again and writes x_{k+1} (12 N + 2 N_c); together sum_c (20 N + 4 N_c)
    # per iteration. The kernels' own I/O is reported beside it: the sweep
    # reads y and the DCT-distance plane and writes g (8 N + 4 N_c), the
    # projection reads y, g, x and the coefficients and writes x, y and the
    # DCT-distance plane (20 N + 6 N_c).
    grad_bytes = upd_bytes = iter_bytes = grad_io = upd_io = 0
    for j in jpegs:
        W, H, _ = j.max_rounded()
        for co in j.coefs:
            nc = co.rounded_px_w * co.rounded_px_h
            grad_bytes += 8 * W * H + 2 * nc
            upd_bytes += 12 * W * H + 2 * nc
            iter_bytes += 20 * W * H + 4 * nc
            grad_io += 8 * W * H + 4 * nc
            upd_io += 20 * W * H + 6 * nc
    peak, peak_kind = load_peaks()
    if g_launch >= u_launch:
        dom, dbytes, dio, dms = "k_grad_sweep", grad_bytes, grad_io, g_launch
    else:
        dom, dbytes, dio, dms = "k_project", upd_bytes, upd_io, u_launch
    achieved = dbytes / (dms * 1e-3) / 1e9
    traffic = read_traffic(args.workload, dom)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, desc = cpu_sample(args.workload, jpegs, iters)
        cpu = {"value": v, "unit": "MPix/s", "cores": 1, "kind": "port", **host_cpu(),
               "sample": desc + " on one host thread"}

    # The HBM-bound configuration (6000x4000, 100 iterations) inside the
    # default run, one GPU.
    hbm = None
    if args.workload == "1080p" and world == 1 and not args.no_hbm:
        hbm = hbm_iteration(lib, local, 3, 1, peak)
    # The 256-image batch and its decode pipeline inside the default run.
    batch = None
    if args.workload == "1080p" and world == 1 and not args.no_batch:
        batch = batch_block(lib, local, 3, 1, peak)

    # Learned warm start (one GPU) on the learned workload's 1080p 4:2:0
    # images at q30/50/75: 8 iterations, and the fewest ladder iterations that
    # reach the plain 50-iteration objective.
    learned = None
    if args.workload == "1080p" and world == 1 and not args.no_learned:
        res = learned_comparison(lib, local, min(args.steps, 10), args.warmup,
                                 ladder=(8, 10, 12, 14, 16, 18, 20, 24, 28, 32, 40, 48))
        if res is not None:
            rows = res["images"]
            learned = {"workload": WORKLOADS["learned"]["name"], "network": res["network"], "schedule": res["schedule"],
                       "refine_iterations": res["refine_iterations"], "plain50_mpix_s": res["plain50_mpix_s"],
                       "mpix_s": res["learned_mpix_s"], "speedup_vs_plain50": res["learned_mpix_s"] / res["plain50_mpix_s"],
                       "max_E_rel_to_plain50": max(r["E_learned_rel"] for r in rows),
                       "iterations_to_reach_plain50": [r["min_refine_to_reach"] for r in rows],
                       "reach_mpix_s": res["reach_mpix_s"],
                       "reach_speedup_vs_plain50": (res["reach_mpix_s"] / res["plain50_mpix_s"]) if res["reach_mpix_s"] else None,
                       "reach_E_rel": [r["min_refine_E_rel"] for r in rows],
                       "reach_infeasibility": [r["min_refine_infeasibility"] for r in rows],
                       "decoded_start_same_iterations_E_rel": [r["min_refine_decoded_same_schedule_E_rel"] for r in rows],
                       "images": rows}
            nms, ntf, nfl = time_network(local, 10, 3, joint=WS_joint_weights_exist())
            pk = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
            peak_tc = float(pk.get("bf16_tflops", 1590.0))
            learned["network_forward"] = {"ms": nms, "tflops": ntf, "gflop": nfl / 1e9, "frac_of_bf16_peak": ntf / peak_tc,
                                          "peak_kind": "measured" if "bf16_tflops" in pk else "fallback",
                                          "network": "joint 4:2:0" if WS_joint_weights_exist() else "per component"}

    # Host decode overlapped with solving (batch workload, one GPU).
    pipe = None
    if args.workload == "batch256" and world == 1:
        pipe = pipeline_e2e(encoded, iters, local)

    modes = len({(c.horizontal_samp_factor, c.vertical_samp_factor) for j in jpegs for c in j.coefs})
    nchs = len({j.nchannel for j in jpegs})
    per_step = sum(j.nchannel for j in jpegs) + 1 + (nchs + modes) * iters
    if rank == 0:
        line = {
            "metric": wl["metric"], "value": value, "unit": "MPix/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.workload, world),
            "e2e": {"value": e2e_value, "unit": "MPix/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_total / e2e_steps,
                    "api": "art_context_compute" if nimg == 1 else "art_context_compute_batch"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": dbytes, "kernel_io_bytes_per_launch": dio,
                         "kernel_io_gbs": dio / (dms * 1e-3) / 1e9, "launch_ms": dms},
            # From the timed steps: step time / iterations (the step's start-up
            # launches included, so this slightly understates the iteration).
            "iteration": {"ms": it_ms, "algorithmic_bytes": iter_bytes, "gbs": iter_bytes / (it_ms * 1e-3) / 1e9,
                          "frac_of_hbm": iter_bytes / (it_ms * 1e-3) / 1e9 / peak,
                          "source": "timed step / iterations"},
            # Separate pass with event nodes in the graph (not the timed steps).
            "event_timing_pass": {"loop_ms_per_iteration": loop / iters, "gradient_ms": g_launch,
                                  "update_ms": u_launch},
            "cpu_baseline": cpu, "gpu_launches": args.steps * per_step, "clocks": clocks, "wall_s": wall,
            "autotuned": tuned,
        }
        if hbm is not None:
            line["hbm_iteration"] = hbm
        if batch is not None:
            line["batch256"] = batch
        if learned is not None:
            line["learned_warm_start"] = learned
        if pipe is not None:
            line["decode_pipeline"] = pipe
        print(json.dumps(line), flush=True)
    lib.art_context_destroy(ctx)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
