"""ctypes access to the CPU oracle (oracle/_build/liboracle.so) -- test infrastructure.

The oracle restates backend/artefact-lib/pipeline_scalar of Delnegend/artefact
in C (fp32 with unfused multiply-adds, and an fp64 twin). Tests use it only as
the checker of the CUDA path.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path
from typing import List, Sequence

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "_build" / "liboracle.so"


class OracleChannel(C.Structure):
    _fields_ = [
        ("rounded_px_w", C.c_uint32), ("rounded_px_h", C.c_uint32),
        ("block_w", C.c_uint32), ("block_h", C.c_uint32),
        ("samp_h", C.c_uint32), ("samp_v", C.c_uint32),
        ("dct_coefs", C.POINTER(C.c_float)), ("quant_table", C.POINTER(C.c_float)),
    ]


_lib = None


def build_oracle() -> Path:
    srcs = [ORACLE_DIR / "artefact_oracle.c", ORACLE_DIR / "oracle_body.inc"]
    if not ORACLE_LIB.exists() or any(s.stat().st_mtime > ORACLE_LIB.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return ORACLE_LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        h = C.CDLL(str(build_oracle()))
        FP, DP = C.POINTER(C.c_float), C.POINTER(C.c_double)
        CH = C.POINTER(OracleChannel)
        for prec, P in (("f32", FP), ("f64", DP)):
            f = getattr(h, f"oracle_{prec}_compute")
            f.restype = C.c_int
            f.argtypes = [C.c_uint32, CH, C.c_float, FP, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                          C.POINTER(P)]
            f2 = getattr(h, f"oracle_{prec}_compute_from")
            f2.restype = C.c_int
            f2.argtypes = [C.c_uint32, CH, C.c_float, FP, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                           C.c_float, C.c_uint32, C.c_uint32, C.c_int, C.POINTER(FP), C.POINTER(P)]
            g = getattr(h, f"oracle_{prec}_gradient")
            g.restype = C.c_int
            g.argtypes = [C.c_uint32, CH, C.c_float, FP, C.c_uint32, C.c_uint32, C.POINTER(P), C.POINTER(P)]
            for n in ("dct8x8", "idct8x8"):
                t = getattr(h, f"oracle_{prec}_{n}")
                t.restype = None
                t.argtypes = [P]
        h.oracle_objective.restype = C.c_double
        h.oracle_objective.argtypes = [C.c_uint32, CH, C.c_float, FP, C.c_uint32, C.c_uint32, C.POINTER(FP), DP]
        h.oracle_objective_f64.restype = C.c_double
        h.oracle_objective_f64.argtypes = [C.c_uint32, CH, C.c_float, FP, C.c_uint32, C.c_uint32, C.POINTER(DP), DP]
        h.oracle_feasibility.restype = C.c_double
        h.oracle_feasibility.argtypes = [C.c_uint32, CH, C.c_uint32, C.c_uint32, C.POINTER(FP)]
        h.oracle_rgb.restype = None
        h.oracle_rgb.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(FP), C.POINTER(C.c_uint8)]
        _lib = h
    return _lib


def _channels(coefs) -> tuple:
    keep = []
    arr = (OracleChannel * len(coefs))()
    for i, c in enumerate(coefs):
        d = np.ascontiguousarray(c.dct_coefs, dtype=np.float32)
        q = np.ascontiguousarray(c.quant_table, dtype=np.float32)
        keep += [d, q]
        arr[i].rounded_px_w, arr[i].rounded_px_h = c.rounded_px_w, c.rounded_px_h
        arr[i].block_w, arr[i].block_h = c.block_w, c.block_h
        arr[i].samp_h, arr[i].samp_v = c.horizontal_samp_factor, c.vertical_samp_factor
        arr[i].dct_coefs = d.ctypes.data_as(C.POINTER(C.c_float))
        arr[i].quant_table = q.ctypes.data_as(C.POINTER(C.c_float))
    return arr, keep


def _pw(pweight: Sequence[float]):
    v = [float(x) for x in pweight][:3]
    return (C.c_float * 3)(*(v + [0.0] * (3 - len(v))))


def compute(nch: int, coefs, weight: float, pweight, iterations: int, W: int, H: int, *, init_mode: int = 0,
            fp64: bool = False) -> List[np.ndarray]:
    """The oracle's pipeline_scalar::compute (fp32, or the fp64 twin)."""
    h = lib()
    chans, keep = _channels(coefs[:nch])
    dt, ct = (np.float64, C.c_double) if fp64 else (np.float32, C.c_float)
    outs = [np.empty(W * H, dtype=dt) for _ in range(nch)]
    ptrs = (C.POINTER(ct) * nch)(*[o.ctypes.data_as(C.POINTER(ct)) for o in outs])
    fn = h.oracle_f64_compute if fp64 else h.oracle_f32_compute
    rc = fn(nch, chans, float(weight), _pw(pweight), int(iterations), W, H, int(init_mode), ptrs)
    if rc != 0:
        raise ValueError("oracle rejected its input")
    return outs


def compute_from(nch: int, coefs, weight: float, pweight, iterations: int, W: int, H: int, start,
                 step_iterations: int = 0, fp64: bool = False, tail_iterations: int = 0,
                 tail_step_iterations: int = 0, step_decay: float = 0.0) -> List[np.ndarray]:
    """The oracle's iteration from given full-resolution start planes (a warm
    start): projection of the start, then `iterations` steps of size
    radius / sqrt(1 + (step_iterations or iterations)), step k of the first
    phase scaled by step_decay^k when step_decay > 0; the last
    `tail_iterations` restart FISTA with steps radius / sqrt(1 + tail_step_iterations)."""
    h = lib()
    chans, keep = _channels(coefs[:nch])
    dt, ct = (np.float64, C.c_double) if fp64 else (np.float32, C.c_float)
    st = [np.ascontiguousarray(p, dtype=np.float32).ravel() for p in start]
    FP = C.POINTER(C.c_float)
    sp = (FP * nch)(*[x.ctypes.data_as(FP) for x in st])
    outs = [np.empty(W * H, dtype=dt) for _ in range(nch)]
    ptrs = (C.POINTER(ct) * nch)(*[o.ctypes.data_as(C.POINTER(ct)) for o in outs])
    fn = h.oracle_f64_compute_from if fp64 else h.oracle_f32_compute_from
    rc = fn(nch, chans, float(weight), _pw(pweight), int(iterations), int(step_iterations), int(tail_iterations),
            int(tail_step_iterations), float(step_decay), W, H, 0, sp, ptrs)
    if rc != 0:
        raise ValueError("oracle rejected its input")
    return outs


def gradient(nch: int, coefs, weight: float, pweight, W: int, H: int, planes) -> List[np.ndarray]:
    """fp64 objective gradient (before normalisation) at the given planes."""
    h = lib()
    chans, keep = _channels(coefs[:nch])
    xs = [np.ascontiguousarray(p, dtype=np.float64).ravel() for p in planes]
    gs = [np.zeros(W * H, dtype=np.float64) for _ in range(nch)]
    DP = C.POINTER(C.c_double)
    xp = (DP * nch)(*[x.ctypes.data_as(DP) for x in xs])
    gp = (DP * nch)(*[g.ctypes.data_as(DP) for g in gs])
    if h.oracle_f64_gradient(nch, chans, float(weight), _pw(pweight), W, H, xp, gp) != 0:
        raise ValueError("oracle rejected its input")
    return gs


def objective(nch: int, coefs, weight: float, pweight, W: int, H: int, planes, terms: bool = False):
    """fp64 objective (TV + TGV + DCT distance) of final planes."""
    h = lib()
    chans, keep = _channels(coefs[:nch])
    t = (C.c_double * 3)()
    if all(np.asarray(p).dtype == np.float64 for p in planes):
        xs = [np.ascontiguousarray(p, dtype=np.float64).ravel() for p in planes]
        DP = C.POINTER(C.c_double)
        ptrs = (DP * nch)(*[x.ctypes.data_as(DP) for x in xs])
        e = h.oracle_objective_f64(nch, chans, float(weight), _pw(pweight), W, H, ptrs, t)
    else:
        xs = [np.ascontiguousarray(p, dtype=np.float32).ravel() for p in planes]
        FP = C.POINTER(C.c_float)
        ptrs = (FP * nch)(*[x.ctypes.data_as(FP) for x in xs])
        e = h.oracle_objective(nch, chans, float(weight), _pw(pweight), W, H, ptrs, t)
    return (e, tuple(t)) if terms else e


def feasibility(nch: int, coefs, W: int, H: int, planes) -> float:
    """Largest fp64 violation of the quantisation box over all output blocks."""
    h = lib()
    chans, keep = _channels(coefs[:nch])
    xs = [np.ascontiguousarray(p, dtype=np.float32).ravel() for p in planes]
    FP = C.POINTER(C.c_float)
    ptrs = (FP * nch)(*[x.ctypes.data_as(FP) for x in xs])
    return h.oracle_feasibility(nch, chans, W, H, ptrs)


def rgb(nch: int, W: int, real_w: int, real_h: int, planes) -> np.ndarray:
    """Output stage of Artefact::process (lib.rs:159-211) on float planes."""
    h = lib()
    xs = [np.ascontiguousarray(p, dtype=np.float32).ravel() for p in planes]
    FP = C.POINTER(C.c_float)
    ptrs = (FP * len(xs))(*[x.ctypes.data_as(FP) for x in xs])
    out = np.empty((real_h, real_w, 3), dtype=np.uint8)
    h.oracle_rgb(nch, W, real_w, real_h, ptrs, out.ctypes.data_as(C.POINTER(C.c_uint8)))
    return out


def dct8x8(block: np.ndarray, fp64: bool = False) -> np.ndarray:
    dt = np.float64 if fp64 else np.float32
    a = np.ascontiguousarray(block, dtype=dt).ravel().copy()
    fn = lib().oracle_f64_dct8x8 if fp64 else lib().oracle_f32_dct8x8
    fn(a.ctypes.data_as(C.POINTER(C.c_double if fp64 else C.c_float)))
    return a.reshape(8, 8)


def idct8x8(block: np.ndarray, fp64: bool = False) -> np.ndarray:
    dt = np.float64 if fp64 else np.float32
    a = np.ascontiguousarray(block, dtype=dt).ravel().copy()
    fn = lib().oracle_f64_idct8x8 if fp64 else lib().oracle_f32_idct8x8
    fn(a.ctypes.data_as(C.POINTER(C.c_double if fp64 else C.c_float)))
    return a.reshape(8, 8)


def process(jpeg, weight, pweight, iterations, separate: bool, init_mode: int = 0) -> np.ndarray:
    """Artefact::process (lib.rs:105-212) on decoded coefficients, with the oracle."""
    W, H, _ = jpeg.max_rounded()
    if jpeg.nchannel == 3 and not separate:
        planes = compute(3, jpeg.coefs, weight[0], pweight, iterations[0], W, H, init_mode=init_mode)
    else:
        planes = [compute(1, [c], weight[i], pweight, iterations[i], W, H, init_mode=init_mode)[0]
                  for i, c in enumerate(jpeg.coefs)]
    nout = 3 if jpeg.nchannel == 3 else 1
    return rgb(nout, W, jpeg.real_px_w, jpeg.real_px_h, planes[:nout])
