"""Conditioning-aware parity check of GPU planes against the CPU oracle.

Bar (floating point, 0..255 pixel units): max |GPU - oracle fp32| <= 1.0 per
pixel of the float planes, final objective within 1e-4 relative, every output
block inside its quantisation box to 1e-3 coefficient units (fp64 DCT). The
error of both against the oracle's fp64 twin is measured on every case. Where
the input is ill-conditioned (the oracle's own fp32 result more than 0.5 from
its fp64 twin, or its objective more than 2.5e-5 relative) the bar becomes the
spread of the oracle's own numerical variants around its fp64 result: fp32,
fp32/fp64 with the lagged DCT coefficients recomputed from x_k, and fp32 with
the projection's IDCTs run rows first (as the GPU runs them) -- each equal in
exact arithmetic. The GPU must lie within 2x that spread + 0.5 pixel units,
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


class OracleRef:
    """The oracle's runs for one input (fp32, fp64 and, where the input is
    ill-conditioned, the variants that set the spread), computed once so that
    several GPU results can be held to the same bar."""

    def __init__(self, j, iterations, weight=0.3, pweight=(0.001,) * 3):
        self.j, self.iterations, self.weight, self.pweight = j, iterations, weight, pweight
        W, H, _ = j.max_rounded()
        n = j.nchannel
        self.args = (n, j.coefs, weight, pweight)
        self.W, self.H = W, H
        self.ref = O.compute(n, j.coefs, weight, pweight, iterations, W, H)
        self.r64 = O.compute(n, j.coefs, weight, pweight, iterations, W, H, fp64=True)
        self.er = O.objective(*self.args, W, H, self.ref)
        self.e64 = O.objective(*self.args, W, H, self.r64)
        self.d_ref64 = _maxdiff(self.ref, self.r64)
        self.rel_ref64 = abs(self.er - self.e64) / abs(self.e64)
        self.well = self.d_ref64 <= 0.5 and self.rel_ref64 <= 2.5e-5
        self.spread_d, self.spread_e = self.d_ref64, self.rel_ref64
        if not self.well:
            for mode, fp64 in ((2, False), (2, True), (4, False), (6, False)):
                v = O.compute(n, j.coefs, weight, pweight, iterations, W, H, init_mode=mode, fp64=fp64)
                self.spread_d = max(self.spread_d, _maxdiff(v, self.r64))
                self.spread_e = max(self.spread_e, abs(O.objective(*self.args, W, H, v) - self.e64) / abs(self.e64))

    def check(self, gpu, label=""):
        """Asserts that GPU planes meet the bar; returns the message."""
        W, H = self.W, self.H
        d, d_gpu64 = _maxdiff(gpu, self.ref), _maxdiff(gpu, self.r64)
        eg = O.objective(*self.args, W, H, gpu)
        rel, rel_gpu64 = abs(eg - self.er) / abs(self.er), abs(eg - self.e64) / abs(self.e64)
        feas = O.feasibility(self.j.nchannel, self.j.coefs, W, H, gpu)
        msg = (f"{label} it={self.iterations} max|gpu-f32|={d:.3g} max|gpu-f64|={d_gpu64:.3g} "
               f"max|f32-f64|={self.d_ref64:.3g} obj rel gpu/f32={rel:.2g} gpu/f64={rel_gpu64:.2g} "
               f"f32/f64={self.rel_ref64:.2g} feas={feas:.2g} {'well-conditioned' if self.well else 'ill-conditioned'}")
        if self.well:
            print(msg)
            assert d <= MAX_ABS, msg
            assert rel <= OBJ_REL, msg
        else:
            msg += f" variant spread: planes {self.spread_d:.3g} objective {self.spread_e:.2g}"
            print(msg)
            assert d_gpu64 <= 2 * self.spread_d + 0.5, msg
            assert rel_gpu64 <= 2 * self.spread_e + OBJ_REL, msg
        assert feas <= FEAS, msg
        return msg


def check_parity(j, iterations, weight=0.3, pweight=(0.001,) * 3, label="", gpu=None):
    """Checks GPU planes (solved here unless given) against the oracle."""
    W, H, N_ = j.max_rounded()
    if gpu is None:
        gpu = compute(j.nchannel, j.coefs, weight, pweight, iterations, W, H, N_)
    ref = OracleRef(j, iterations, weight, pweight)
    ref.check(gpu, label)
    return gpu, ref.ref
