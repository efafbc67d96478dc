#!/usr/bin/env python
"""Benchmark of the B200 restoration solver (one JSON line on rank 0).

Workload (one "step"): one plain 50-iteration solve of a seeded synthetic
1920x1080 YCbCr 4:2:0 baseline JPEG at quality 75 (weight 0.3, pweight 0.001),
the configuration the headline metric is quoted on. Metric: megapixels per
second of real image area (1920*1080 per step).

* value   -- coefficients already in HBM, result planes written to HBM,
             timed per step with CUDA events; L2 flushed (256 MiB write)
             between steps, outside the timed events.
* e2e     -- the same solve through the public C ABI (art_context_compute)
             from pinned host coefficient buffers to pinned host planes,
             host<->device copies inside the timed region.
* roofline -- the dominant kernel's own I/O bytes per launch over its mean
             launch time (CUDA event nodes inside the captured graph, taken
             in a separate pass so they do not perturb `value`).
* cpu_baseline -- the oracle (fp32 C restatement of pipeline_scalar) on the
             same image, 50 iterations, one host thread.
* --impl reference -- the oracle as the reference arm, steps spread over the
             host's threads.

Multi-GPU (torchrun): replicas only -- every rank solves its own copy; value is
all ranks' megapixels over the slowest rank's time.
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

WORKLOAD = dict(width=1920, height=1080, quality=75, subsampling="4:2:0", gray=False, seed=2000, iterations=50,
                weight=0.3, pweight=0.001)
WORKLOAD_NAME = "1920x1080 YCbCr 4:2:0 baseline JPEG q75, plain solver 50 iterations (weight 0.3, pweight 0.001)"
METRIC = "MPix/s (plain 50-iteration solve, 1080p 4:2:0 q75)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_workload():
    from artefact_b200 import synth
    from artefact_b200.api import Jpeg, JpegSource

    w = WORKLOAD
    data = synth.make_jpeg(w["width"], w["height"], w["quality"], w["subsampling"], w["gray"], w["seed"])
    return Jpeg.from_source(JpegSource.Buffer(data))


class Clocks:
    """Samples nvidia-smi during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def oracle_solve(jpeg, iterations):
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib

    W, H, _ = jpeg.max_rounded()
    w = WORKLOAD
    return oracle_lib.compute(jpeg.nchannel, jpeg.coefs, w["weight"], [w["pweight"]] * 3, iterations, W, H)


def run_reference(args, rank, world):
    """Reference arm: the oracle port of pipeline_scalar on the host cores."""
    if rank != 0:
        return
    from concurrent.futures import ThreadPoolExecutor

    jpeg = make_workload()
    w = WORKLOAD
    mpix = w["width"] * w["height"] / 1e6
    threads = max(1, min(args.steps, os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(lambda _: oracle_solve(jpeg, w["iterations"]), range(min(args.warmup, threads))))
        t0 = time.perf_counter()
        list(ex.map(lambda _: oracle_solve(jpeg, w["iterations"]), range(args.steps)))
        dt = time.perf_counter() - t0
    value = args.steps * mpix / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "MPix/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps * threads,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "iterations": w["iterations"]},
        "cpu_baseline": {"value": value, "unit": "MPix/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full solves of the workload spread over {threads} host threads "
                                   "(fp32 C restatement of pipeline_scalar; the Rust reference is not buildable here)"},
        "e2e": {"value": value, "unit": "MPix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    jpeg = make_workload()
    W, H, _ = jpeg.max_rounded()
    w = WORKLOAD
    nch = jpeg.nchannel
    iters = w["iterations"]
    mpix = w["width"] * w["height"] / 1e6

    # Device-resident inputs and outputs.
    dev_coefs = [torch.from_numpy(c.dct_coefs.copy()).cuda() for c in jpeg.coefs]
    qs = [np.ascontiguousarray(c.quant_table, np.float32) for c in jpeg.coefs]
    chans_dev = (N.ArtChannel * nch)()
    chans_host = (N.ArtChannel * nch)()
    pinned_coefs = [torch.from_numpy(c.dct_coefs.copy()).pin_memory() for c in jpeg.coefs]
    for i, c in enumerate(jpeg.coefs):
        for arr, ptr in ((chans_dev, dev_coefs[i].data_ptr()), (chans_host, pinned_coefs[i].data_ptr())):
            ch = arr[i]
            ch.rounded_px_w, ch.rounded_px_h, ch.block_w, ch.block_h = (c.rounded_px_w, c.rounded_px_h, c.block_w,
                                                                        c.block_h)
            ch.samp_h, ch.samp_v, ch.coef_type = c.horizontal_samp_factor, c.vertical_samp_factor, N.ART_COEF_I16
            ch.dct_coefs = ptr
            ch.quant_table = qs[i].ctypes.data_as(C.POINTER(C.c_float))
    pitch = (W + 31) // 32 * 32
    outs = [torch.empty(H, pitch, device="cuda") for _ in range(nch)]
    out_ptrs = (C.c_void_p * nch)(*[o.data_ptr() for o in outs])
    host_outs = [torch.empty(W * H, dtype=torch.float32).pin_memory() for _ in range(nch)]
    host_ptrs = (C.c_void_p * nch)(*[o.data_ptr() for o in host_outs])
    pw = (C.c_float * 3)(w["pweight"], w["pweight"], w["pweight"])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    ctx = C.c_void_p()
    N.check(lib.art_context_create(local, C.byref(ctx)))
    stream = torch.cuda.current_stream()

    def solve_device():
        N.check(lib.art_context_compute_device(ctx, nch, chans_dev, w["weight"], pw, iters, W, H, out_ptrs, pitch,
                                               None, C.c_void_p(stream.cuda_stream)))

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # --- warm-up
    for _ in range(args.warmup):
        flush.fill_(1.0)
        solve_device()
    torch.cuda.synchronize()
    N.check(lib.art_context_synchronize(ctx))

    # --- timed region: value (device-resident)
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
    clocks = clk.summary()

    # --- e2e through the C ABI with pinned host buffers
    for _ in range(max(1, args.warmup // 2)):
        N.check(lib.art_context_compute(ctx, nch, chans_host, w["weight"], pw, iters, W, H, host_ptrs, None))
    barrier()
    e2e_ms = []
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        N.check(lib.art_context_compute(ctx, nch, chans_host, w["weight"], pw, iters, W, H, host_ptrs, None))
        e2e_ms.append((time.perf_counter() - t1) * 1e3)
    e2e_total = sum(e2e_ms)
    if dist:
        t = torch.tensor([e2e_total], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * args.steps * mpix / (e2e_total / 1e3)
    h2d = sum(int(c.dct_coefs.nbytes) for c in jpeg.coefs)
    d2h = nch * W * H * 4

    # --- kernel timing pass (event nodes inside the graph)
    N.check(lib.art_context_set_timing(ctx, 1))
    grad_ms, upd_ms, loop_ms, launches = [], [], [], 0
    lm, gm, um, nl = C.c_float(), C.c_float(), C.c_float(), C.c_uint32()
    for k in range(max(3, min(args.steps, 10))):
        flush.fill_(float(k))
        solve_device()
        N.check(lib.art_context_synchronize(ctx))
        N.check(lib.art_context_last_timing(ctx, C.byref(lm), C.byref(gm), C.byref(um), C.byref(nl)))
        if k > 0:
            loop_ms.append(lm.value)
            grad_ms.append(gm.value)
            upd_ms.append(um.value)
    N.check(lib.art_context_set_timing(ctx, 0))
    g_launch = statistics.mean(grad_ms) / iters
    u_launch = statistics.mean(upd_ms) / iters
    loop = statistics.mean(loop_ms)

    # Algorithmic bytes (per launch): the gradient sweep reads x_k, x_{k-1} and
    # the DCT-distance gradient plane (component resolution) and writes g; the
    # projection reads x_k, x_{k-1}, g and the int16 coefficients and writes
    # x_{k+1} and the next DCT-distance gradient plane.
    n_full = W * H
    nc = [c.rounded_px_w * c.rounded_px_h for c in jpeg.coefs]
    grad_bytes = sum(12 * n_full + 4 * x for x in nc)
    upd_bytes = sum(16 * n_full + 6 * x for x in nc)
    iter_bytes = sum(20 * n_full + 4 * x for x in nc)  # two-sweep minimum per iteration
    peak, peak_kind = load_peaks()
    if g_launch >= u_launch:
        dom, dbytes, dms = "k_grad_sweep", grad_bytes, g_launch
    else:
        dom, dbytes, dms = "k_project", upd_bytes, u_launch
    achieved = dbytes / (dms * 1e-3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        try:
            traffic = json.loads(tf.read_text()).get(dom)
        except Exception:
            traffic = None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t2 = time.perf_counter()
        oracle_solve(jpeg, iters)
        cdt = time.perf_counter() - t2
        cpu = {"value": mpix / cdt, "unit": "MPix/s", "cores": 1, "kind": "port",
               "sample": "one full solve of the workload (50 iterations) by the fp32 C restatement of "
                         "pipeline_scalar on one host thread"}

    modes = len({(c.horizontal_samp_factor, c.vertical_samp_factor) for c in jpeg.coefs})
    gpu_launches = args.steps * (nch + 1 + (1 + modes) * iters)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "MPix/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, "iterations": iters, "channels": nch, "max_rounded": [W, H],
                       "l2": "flushed between steps (256 MiB write outside the timed events)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": "MPix/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_total / args.steps, "api": "art_context_compute (host buffers)"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": dbytes, "launch_ms": dms},
            "iteration": {"ms": loop / iters, "gradient_ms": g_launch, "update_ms": u_launch,
                          "algorithmic_bytes": iter_bytes,
                          "gbs": iter_bytes / (loop / iters * 1e-3) / 1e9,
                          "frac_of_hbm": iter_bytes / (loop / iters * 1e-3) / 1e9 / peak},
            "cpu_baseline": cpu, "gpu_launches": gpu_launches, "clocks": clocks, "wall_s": wall,
        }
        print(json.dumps(line), flush=True)
    lib.art_context_destroy(ctx)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
