"""Plain-Python baseline JPEG coefficient decoder -- TEST INFRASTRUCTURE.

This is the oracle's front end: it turns JPEG bytes into what artefact-lib's
host front end hands the solver (backend/artefact-lib/jpeg/zune.rs:5-55),
without the product library. The tests use it to cross-check the product's
decoder (artefact_b200/csrc/jpeg_decode.cpp) coefficient for coefficient,
and bench.py's reference arm uses it so that arm never loads the product
library. Nothing in the product imports it.

Restated from the reference's zune-jpeg fork and ITU-T T.81:
  * markers and segments: DQT (zune-jpeg/src/headers.rs:115-178; 8- and
    16-bit tables, zigzag -> natural order as un_zig_zag, headers.rs:540-553),
    SOF0/SOF1 (headers.rs:182-294), DHT (headers.rs:29-113), SOS
    (headers.rs:295-420), DRI;
  * rounded plane sizes: the image size rounded up to 8 x the largest
    sampling factor, divided by max / component sampling (misc.rs:209-249);
  * canonical Huffman codes (T.81 Annex C; huffman.rs:93-180) and block
    decoding: DC difference + prediction, AC run/size symbols, ZRL, EOB,
    values placed at their natural (row-major) index (bitstream.rs:279-390);
  * MCU order: interleaved scans code, per MCU, each component's V x H blocks
    row by row (mcu.rs:199-290); a single-component scan codes
    ceil(samples / 8) blocks per row (T.81 A.2.2); restart markers reset the
    DC predictions (mcu.rs:339-360).
Only sequential Huffman streams (SOF0/SOF1, 8-bit samples) are handled; the
product's decoder also handles progressive streams, which the bench does not
use. Blocks are placed by their (row, column) position for every sampling
(T.81 A.2.3); the reference's mcu.rs:236-247 places the two blocks of a
vertically doubled component side by side, a difference only 4:4:0 streams
(luma sampled 1x2) would show.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

ZIGZAG = (
    0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5, 12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6, 7, 14,
    21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60,
    61, 54, 47, 55, 62, 63)


class OracleDecodeError(ValueError):
    pass


@dataclass
class OracleCoefficient:
    """One component with the fields of artefact-lib's Coefficient (jpeg/mod.rs:8-27)."""

    rounded_px_w: int
    rounded_px_h: int
    block_w: int
    block_h: int
    horizontal_samp_factor: int
    vertical_samp_factor: int
    dct_coefs: np.ndarray    # int16, block raster, natural order inside a block
    quant_table: np.ndarray  # float32 [64], natural order


@dataclass
class OracleJpeg:
    nchannel: int
    real_px_w: int
    real_px_h: int
    coefs: List[OracleCoefficient]

    def max_rounded(self):
        """(max rounded width, height, pixel count) over components (lib.rs:108-116)."""
        w = max(c.rounded_px_w for c in self.coefs)
        h = max(c.rounded_px_h for c in self.coefs)
        return w, h, w * h


def _huffman_table(counts, values):
    """16-bit lookahead table of a canonical code: entry (length << 8) | symbol,
    0 where no code of length <= 16 matches (T.81 C.2, huffman.rs:93-180)."""
    table = [0] * 65536
    code, k = 0, 0
    for length in range(1, 17):
        for _ in range(counts[length - 1]):
            if code >= (1 << length):
                raise OracleDecodeError("Invalid Huffman table: code overflow")
            span = 1 << (16 - length)
            start = code << (16 - length)
            table[start:start + span] = [(length << 8) | values[k]] * span
            code += 1
            k += 1
        code <<= 1
    return table


class _Component:
    def __init__(self, cid, h, v, tq):
        self.id, self.h, self.v, self.tq = cid, h, v, tq
        self.dc_pred = 0


def _entropy_segments(data: bytes, pos: int):
    """De-stuffed entropy-coded bytes from `pos`, split at restart markers:
    (list of segments, position of the marker that ends the scan)."""
    segs, cur = [], bytearray()
    n = len(data)
    while True:
        j = data.find(b"\xff", pos)
        if j < 0 or j + 1 >= n:
            cur += data[pos:]
            segs.append(bytes(cur))
            return segs, n
        cur += data[pos:j]
        m = data[j + 1]
        if m == 0x00:
            cur.append(0xFF)
            pos = j + 2
        elif m == 0xFF:  # fill byte
            pos = j + 1
        elif 0xD0 <= m <= 0xD7:
            segs.append(bytes(cur))
            cur = bytearray()
            pos = j + 2
        else:
            segs.append(bytes(cur))
            return segs, j


class _Bits:
    """Bit reader over one de-stuffed segment: 32-bit windows at every byte,
    zero bits past the end."""

    def __init__(self, seg: bytes):
        b = np.frombuffer(seg + b"\x00" * 8, dtype=np.uint8).astype(np.uint32)
        w = (b[:-3] << 24) | (b[1:-2] << 16) | (b[2:-1] << 8) | b[3:]
        self.win = w.tolist()
        self.nbits = 8 * len(seg)
        self.p = 0


def decode(data: bytes) -> OracleJpeg:
    """Coefficients and quantisation tables of a sequential Huffman JPEG."""
    data = bytes(data)
    if len(data) < 4 or data[0] != 0xFF or data[1] != 0xD8:
        raise OracleDecodeError("No SOI marker")
    pos = 2
    qt: List[Optional[np.ndarray]] = [None] * 4
    dc_tabs: List[Optional[list]] = [None] * 4
    ac_tabs: List[Optional[list]] = [None] * 4
    comps: List[_Component] = []
    width = height = 0
    restart = 0
    planes = None
    hmax = vmax = 1
    frame = False
    while True:
        while pos < len(data) and data[pos] != 0xFF:
            pos += 1
        while pos < len(data) and data[pos] == 0xFF:
            pos += 1
        if pos >= len(data):
            raise OracleDecodeError("No EOI marker")
        marker = data[pos]
        pos += 1
        if marker == 0xD9:
            break
        if 0xD0 <= marker <= 0xD7 or marker == 0x01:
            continue
        if pos + 2 > len(data):
            raise OracleDecodeError("Truncated segment")
        seglen = (data[pos] << 8) | data[pos + 1]
        seg = data[pos + 2:pos + seglen]
        if len(seg) != seglen - 2:
            raise OracleDecodeError("Truncated segment")
        pos += seglen
        if marker == 0xDB:  # DQT
            i = 0
            while i < len(seg):
                pq, tq = seg[i] >> 4, seg[i] & 15
                i += 1
                if tq > 3:
                    raise OracleDecodeError("Bad quantisation table id")
                if pq == 0:
                    vals = list(seg[i:i + 64])
                    i += 64
                else:
                    vals = [(seg[i + 2 * k] << 8) | seg[i + 2 * k + 1] for k in range(64)]
                    i += 128
                t = np.zeros(64, np.float32)
                for k in range(64):
                    t[ZIGZAG[k]] = vals[k]
                qt[tq] = t
        elif marker in (0xC0, 0xC1):  # SOF0 / SOF1
            if seg[0] != 8:
                raise OracleDecodeError("Only 8-bit samples")
            height, width = (seg[1] << 8) | seg[2], (seg[3] << 8) | seg[4]
            nc = seg[5]
            comps = []
            for k in range(nc):
                cid, hv, tq = seg[6 + 3 * k], seg[7 + 3 * k], seg[8 + 3 * k]
                h, v = hv >> 4, hv & 15
                if h not in (1, 2) or v not in (1, 2):
                    raise OracleDecodeError("Sampling factors other than 1 or 2")
                comps.append(_Component(cid, h, v, tq))
            if width == 0 or height == 0 or nc == 0:
                raise OracleDecodeError("Empty frame")
            hmax, vmax = max(c.h for c in comps), max(c.v for c in comps)
            rw = (width + 8 * hmax - 1) // (8 * hmax) * (8 * hmax)
            rh = (height + 8 * vmax - 1) // (8 * vmax) * (8 * vmax)
            planes = []
            for c in comps:
                cw, ch = rw // (hmax // c.h), rh // (vmax // c.v)
                planes.append((cw, ch, np.zeros(cw * ch, np.int16)))
            frame = True
        elif 0xC2 <= marker <= 0xCF and marker not in (0xC4, 0xC8, 0xCC):
            raise OracleDecodeError("Only sequential Huffman streams")
        elif marker == 0xC4:  # DHT
            i = 0
            while i < len(seg):
                tc, th = seg[i] >> 4, seg[i] & 15
                counts = list(seg[i + 1:i + 17])
                total = sum(counts)
                vals = list(seg[i + 17:i + 17 + total])
                if th > 3 or len(vals) != total or total > 256:
                    raise OracleDecodeError("Invalid Huffman length in image")
                i += 17 + total
                (ac_tabs if tc else dc_tabs)[th] = _huffman_table(counts, vals)
        elif marker == 0xDD:  # DRI
            restart = (seg[0] << 8) | seg[1]
        elif marker == 0xDA:  # SOS
            if not frame:
                raise OracleDecodeError("Scan before frame")
            ns = seg[0]
            members = []
            for k in range(ns):
                cid, tdta = seg[1 + 2 * k], seg[2 + 2 * k]
                idx = [i for i, c in enumerate(comps) if c.id == cid]
                if not idx:
                    raise OracleDecodeError("Scan names an unknown component")
                members.append((idx[0], tdta >> 4, tdta & 15))
            segs, pos = _entropy_segments(data, pos)
            _decode_scan(comps, planes, members, segs, width, height, hmax, vmax, restart, dc_tabs, ac_tabs)
    if not frame:
        raise OracleDecodeError("No frame")
    coefs = []
    for c, (cw, ch, arr) in zip(comps, planes):
        if qt[c.tq] is None:
            raise OracleDecodeError("No quantization table for component")
        # arr holds the blocks in raster order, natural order inside each block.
        coefs.append(OracleCoefficient(cw, ch, cw // 8, ch // 8, hmax // c.h, vmax // c.v, arr, qt[c.tq].copy()))
    return OracleJpeg(len(comps), width, height, coefs)


def _decode_scan(comps, planes, members, segs, width, height, hmax, vmax, restart, dc_tabs, ac_tabs):
    for ci, td, ta in members:
        if dc_tabs[td] is None or ac_tabs[ta] is None:
            raise OracleDecodeError("Scan uses an undefined Huffman table")
        comps[ci].dc_pred = 0
    # Block order of the scan: list of (component, block index or -1 to drop).
    if len(members) == 1:
        ci = members[0][0]
        c = comps[ci]
        cw_, _, _ = planes[ci]
        bwr = cw_ // 8
        bhr = planes[ci][1] // 8
        cw = (width * c.h + hmax - 1) // hmax
        chh = (height * c.v + vmax - 1) // vmax
        bw, bh = (cw + 7) // 8, (chh + 7) // 8
        units = [[(ci, by * bwr + bx if bx < bwr and by < bhr else -1)] for by in range(bh) for bx in range(bw)]
    else:
        mcu_w = (width + 8 * hmax - 1) // (8 * hmax)
        mcu_h = (height + 8 * vmax - 1) // (8 * vmax)
        units = []
        for my in range(mcu_h):
            for mx in range(mcu_w):
                u = []
                for ci, _, _ in members:
                    c = comps[ci]
                    bwr = planes[ci][0] // 8
                    for v in range(c.v):
                        for h in range(c.h):
                            u.append((ci, (my * c.v + v) * bwr + mx * c.h + h))
                units.append(u)
    tabs = {ci: (dc_tabs[td], ac_tabs[ta]) for ci, td, ta in members}
    per = restart if restart else len(units)
    nint = (len(units) + per - 1) // per if units else 0
    if nint > len(segs):
        raise OracleDecodeError("Scan ends before its last restart interval")
    # Decoded (flat index into the block-major plane, value) pairs per component.
    idx = {ci: [] for ci, _, _ in members}
    val = {ci: [] for ci, _, _ in members}
    zz = ZIGZAG
    for it in range(nint):
        for ci, _, _ in members:
            comps[ci].dc_pred = 0
        bits = _Bits(segs[it])
        win = bits.win
        p = 0
        for u in units[it * per:(it + 1) * per]:
            for ci, blk in u:
                dct, act = tabs[ci]
                comp = comps[ci]
                # DC (T.81 F.2.2.1): difference of category s, then the prediction.
                e = dct[(win[p >> 3] >> (16 - (p & 7))) & 0xFFFF]
                if e == 0:
                    raise OracleDecodeError("Bad Huffman code")
                p += e >> 8
                s = e & 255
                diff = 0
                if s:
                    r = (win[p >> 3] >> (32 - s - (p & 7))) & ((1 << s) - 1)
                    p += s
                    diff = r if r >= (1 << (s - 1)) else r - (1 << s) + 1
                comp.dc_pred += diff
                base = blk * 64
                I, V = idx[ci], val[ci]
                if blk >= 0:
                    I.append(base)
                    V.append(comp.dc_pred)
                k = 1
                while k < 64:
                    e = act[(win[p >> 3] >> (16 - (p & 7))) & 0xFFFF]
                    if e == 0:
                        raise OracleDecodeError("Bad Huffman code")
                    p += e >> 8
                    rs = e & 255
                    s = rs & 15
                    if s:
                        k += rs >> 4
                        if k > 63:
                            raise OracleDecodeError("Coefficient index out of range")
                        r = (win[p >> 3] >> (32 - s - (p & 7))) & ((1 << s) - 1)
                        p += s
                        if blk >= 0:
                            I.append(base + zz[k])
                            V.append(r if r >= (1 << (s - 1)) else r - (1 << s) + 1)
                        k += 1
                    elif rs == 0xF0:
                        k += 16
                    else:
                        break
        if p > bits.nbits + 64:
            raise OracleDecodeError("Scan data ended early")
    for ci in idx:
        arr = planes[ci][2]
        if idx[ci]:
            arr[np.asarray(idx[ci], np.int64)] = np.asarray(val[ci], np.int64).astype(np.int16)
