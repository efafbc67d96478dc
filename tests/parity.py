"""Conditioning-aware parity check of GPU planes against the CPU oracle.

Bar (floating point, 0..255 pixel units): max |GPU - oracle fp32| <= 1.0 per
pixel of the float planes, final objective within 1e-4 relative, every output
block inside its quantisation box to 1e-3 coefficient units (fp64 DCT). The
error of both against the oracle's fp64 twin is measured on every case. Where
the input is ill-conditioned (the oracle's own fp32 result more than 0.5 from
its fp64 twin, or its objective more than 2.5e-5 relative) the bar becomes the
spread of the oracle's own numerical variants around its fp64 result: fp32,
and fp32/fp64 with the lagged DCT coefficients recomputed from x_k (equal in
exact arithmetic). The GPU must lie within 2x that spread + 0.5 pixel units,
and its objective within 2x + 1e-4.
"""
import numpy as np

import oracle_lib as O
from artefact_b200 import compute

MAX_ABS = 1.0
OBJ_REL = 1e-4
FEAS = 1e-3


def _maxdiff(a, b):
    return max(float(np.abs(x.astype(np.float64) - y.astype(np.float64)).max()) for x, y in zip(a, b))


def check_parity(j, iterations, weight=0.3, pweight=(0.001,) * 3, label="", gpu=None):
    """Checks GPU planes (solved here unless given) against the oracle."""
    W, H, N_ = j.max_rounded()
    n = j.nchannel
    if gpu is None:
        gpu = compute(n, j.coefs, weight, pweight, iterations, W, H, N_)
    ref = O.compute(n, j.coefs, weight, pweight, iterations, W, H)
    r64 = O.compute(n, j.coefs, weight, pweight, iterations, W, H, fp64=True)
    d, d_gpu64, d_ref64 = _maxdiff(gpu, ref), _maxdiff(gpu, r64), _maxdiff(ref, r64)
    eg = O.objective(n, j.coefs, weight, pweight, W, H, gpu)
    er = O.objective(n, j.coefs, weight, pweight, W, H, ref)
    e64 = O.objective(n, j.coefs, weight, pweight, W, H, r64)
    rel, rel_gpu64, rel_ref64 = abs(eg - er) / abs(er), abs(eg - e64) / abs(e64), abs(er - e64) / abs(e64)
    feas = O.feasibility(n, j.coefs, W, H, gpu)
    well = d_ref64 <= 0.5 and rel_ref64 <= 2.5e-5
    msg = (f"{label} it={iterations} max|gpu-f32|={d:.3g} max|gpu-f64|={d_gpu64:.3g} max|f32-f64|={d_ref64:.3g} "
           f"obj rel gpu/f32={rel:.2g} gpu/f64={rel_gpu64:.2g} f32/f64={rel_ref64:.2g} feas={feas:.2g} "
           f"{'well-conditioned' if well else 'ill-conditioned'}")
    print(msg)
    if well:
        assert d <= MAX_ABS, msg
        assert rel <= OBJ_REL, msg
    else:
        spread_d, spread_e = d_ref64, rel_ref64
        for fp64 in (False, True):
            v = O.compute(n, j.coefs, weight, pweight, iterations, W, H, init_mode=2, fp64=fp64)
            spread_d = max(spread_d, _maxdiff(v, r64))
            spread_e = max(spread_e, abs(O.objective(n, j.coefs, weight, pweight, W, H, v) - e64) / abs(e64))
        msg += f" variant spread: planes {spread_d:.3g} objective {spread_e:.2g}"
        print(msg)
        assert d_gpu64 <= 2 * spread_d + 0.5, msg
        assert rel_gpu64 <= 2 * spread_e + OBJ_REL, msg
    assert feas <= FEAS, msg
    return gpu, ref


