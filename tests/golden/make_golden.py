"""Regenerates the golden fixtures in tests/golden/.

* decoder_malformed.json -- the six malformed streams of the reference's
  decoder tests (backend/zune-jpeg/tests/invalid_images.rs:12-66) with the
  error text the reference expects where it checks one.
* roundtrip_*.jpg / .npz -- JPEGs written by tests/jpeg_encoder.py from known
  random quantised coefficients; the decoder must return them bit-exactly.
* synth_*.jpg -- tiny seeded synthetic JPEGs (artefact_b200.synth), and
  synth_*.npz the oracle's fp32 and fp64 outputs on them, which pin the
  oracle's own behaviour against regressions.

Run from the repository root: python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE.parent))

import jpeg_encoder as E  # noqa: E402
import oracle_lib as O  # noqa: E402
from artefact_b200 import synth  # noqa: E402
from artefact_b200.api import Jpeg, JpegSource  # noqa: E402

MALFORMED = [
    {"name": "eof", "bytes": [0xFF, 0xD8, 0xA4], "message": None},
    {"name": "bad_ff_marker_size", "bytes": [0xFF, 0xD8, 0xFF, 0x00, 0x00, 0x00], "message": None},
    {"name": "bad_number_of_scans", "bytes": [255, 216, 255, 218, 232, 197, 255],
     "message": "Bad SOS length 59589,corrupt jpeg"},
    {"name": "huffman_length_subtraction_overflow", "bytes": [255, 216, 255, 196, 0, 0],
     "message": "Invalid Huffman length in image"},
    {"name": "index_oob", "bytes": [255, 216, 255, 218, 0, 8, 1, 0, 8, 1], "message": None},
    {"name": "mul_with_overflow", "bytes": [255, 216, 255, 192, 255, 1, 8, 9, 119, 48, 255, 192],
     "message": "Length of start of frame differs from expected 584,value is 65281"},
]

ROUNDTRIP = [
    ("gray_37x21", 37, 21, [(1, 1)], 0),
    ("420_100x70_rst3", 100, 70, [(2, 2), (1, 1), (1, 1)], 3),
    ("422_50x30", 50, 30, [(2, 1), (1, 1), (1, 1)], 0),
    ("444_24x40_rst5", 24, 40, [(1, 1), (1, 1), (1, 1)], 5),
]

SYNTH = [
    # name, w, h, quality, subsampling, gray, iterations
    ("gray_40x24_q50", 40, 24, 50, "4:4:4", True, 20),
    ("420_72x40_q75", 72, 40, 75, "4:2:0", False, 20),
    ("444_48x32_q30", 48, 32, 30, "4:4:4", False, 20),
]


def main():
    (HERE / "decoder_malformed.json").write_text(json.dumps(MALFORMED, indent=1) + "\n")
    rng = np.random.default_rng(20240601)
    for name, w, h, samp, ri in ROUNDTRIP:
        comps, expect, _ = E.random_image(rng, w, h, samp)
        data = E.encode(w, h, comps, restart_interval=ri)
        (HERE / f"roundtrip_{name}.jpg").write_bytes(data)
        arrays = {}
        for i, (coefs, qt, bw, bh, sh, sv) in enumerate(expect):
            arrays[f"coefs{i}"] = coefs
            arrays[f"qt{i}"] = qt
            arrays[f"meta{i}"] = np.array([bw, bh, sh, sv], dtype=np.int32)
        np.savez_compressed(HERE / f"roundtrip_{name}.npz", **arrays)
    for i, (name, w, h, q, sub, gray, iters) in enumerate(SYNTH):
        data = synth.make_jpeg(w, h, q, sub, gray, seed=9000 + i)
        (HERE / f"synth_{name}.jpg").write_bytes(data)
        j = Jpeg.from_source(JpegSource.Buffer(data))
        W, H, _ = j.max_rounded()
        out32 = O.compute(j.nchannel, j.coefs, 0.3, [0.001] * 3, iters, W, H)
        out64 = O.compute(j.nchannel, j.coefs, 0.3, [0.001] * 3, iters, W, H, fp64=True)
        np.savez_compressed(HERE / f"synth_{name}.npz", f32=np.stack(out32), f64=np.stack(out64),
                            iterations=np.int32(iters))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
