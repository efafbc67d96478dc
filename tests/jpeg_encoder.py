"""Minimal baseline JPEG encoder used by tests to check the decoder bit-exactly.

It writes given quantised coefficients (natural order, block raster per
component) with given quantisation tables, sampling factors and the standard
Huffman tables of ITU-T T.81 Annex K, so the decoder's output can be compared
with the exact values that went in. Entropy coding follows T.81 F.1.2.
"""
from __future__ import annotations

import struct
from typing import List, Optional, Sequence

import numpy as np

ZIGZAG = np.array([
    0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5, 12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6, 7, 14,
    21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60,
    61, 54, 47, 55, 62, 63])

DC_LUMA_BITS = [0, 1, 5, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0]
DC_CHROMA_BITS = [0, 3, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0]
DC_VALS = list(range(12))
AC_LUMA_BITS = [0, 2, 1, 3, 3, 2, 4, 3, 5, 5, 4, 4, 0, 0, 1, 0x7D]
AC_LUMA_VALS = bytes.fromhex(
    "01020300041105122131410613516107227114328191a1082342b1c11552d1f02433627282090a161718191a25262728292a3435363738"
    "393a434445464748494a535455565758595a636465666768696a737475767778797a838485868788898a92939495969798999aa2a3a4a5"
    "a6a7a8a9aab2b3b4b5b6b7b8b9bac2c3c4c5c6c7c8c9cad2d3d4d5d6d7d8d9dae1e2e3e4e5e6e7e8e9eaf1f2f3f4f5f6f7f8f9fa")
AC_CHROMA_BITS = [0, 2, 1, 2, 4, 4, 3, 4, 7, 5, 4, 4, 0, 1, 2, 0x77]
AC_CHROMA_VALS = bytes.fromhex(
    "000102031104052131061241510761711322328108144291a1b1c109233352f0156272d10a162434e125f11718191a262728292a353637"
    "38393a434445464748494a535455565758595a636465666768696a737475767778797a82838485868788898a92939495969798999aa2a3"
    "a4a5a6a7a8a9aab2b3b4b5b6b7b8b9bac2c3c4c5c6c7c8c9cad2d3d4d5d6d7d8d9dae2e3e4e5e6e7e8e9eaf2f3f4f5f6f7f8f9fa")


def _codes(bits: Sequence[int], vals: Sequence[int]) -> dict:
    """Canonical Huffman code of T.81 Annex C: symbol -> (code, length)."""
    table, code, k = {}, 0, 0
    for length in range(1, 17):
        for _ in range(bits[length - 1]):
            table[vals[k]] = (code, length)
            code += 1
            k += 1
        code <<= 1
    return table


class _Bits:
    def __init__(self):
        self.out = bytearray()
        self.acc = 0
        self.n = 0

    def put(self, value: int, length: int):
        for i in range(length - 1, -1, -1):
            self.acc = (self.acc << 1) | ((value >> i) & 1)
            self.n += 1
            if self.n == 8:
                self.out.append(self.acc)
                if self.acc == 0xFF:
                    self.out.append(0)
                self.acc = self.n = 0

    def flush(self):
        while self.n:
            self.put(1, 1)


def _category(v: int) -> int:
    return int(abs(v)).bit_length()


def _magnitude_bits(v: int, t: int) -> int:
    return v if v >= 0 else v + (1 << t) - 1


class Component:
    def __init__(self, h: int, v: int, qt: np.ndarray, coefs: np.ndarray, block_w: int, block_h: int,
                 table: int):
        self.h, self.v, self.qt, self.coefs = h, v, np.asarray(qt), np.asarray(coefs, dtype=np.int64)
        self.block_w, self.block_h, self.table = block_w, block_h, table


def encode(width: int, height: int, comps: List[Component], restart_interval: int = 0,
           qt_16bit: Optional[Sequence[bool]] = None, separate_scans: bool = False,
           omit_scans: Sequence[int] = ()) -> bytes:
    """Encode components (coefs shaped (block_h*block_w, 64), natural order).
    separate_scans: one non-interleaved scan per component (T.81 A.2.2), each
    coding the ceil(component samples / 8) blocks of its rows and columns only;
    the components listed in omit_scans get no scan (an incomplete stream)."""
    out = bytearray(b"\xff\xd8")
    ntab = max(c.table for c in comps) + 1
    for t in range(ntab):
        qt = next(c.qt for c in comps if c.table == t)
        wide = bool(qt_16bit[t]) if qt_16bit else bool(np.max(qt) > 255)
        body = bytes([(1 << 4 if wide else 0) | t])
        for i in range(64):
            val = int(qt[ZIGZAG[i]])
            body += struct.pack(">H", val) if wide else bytes([val])
        out += b"\xff\xdb" + struct.pack(">H", len(body) + 2) + body
    hmax = max(c.h for c in comps)
    vmax = max(c.v for c in comps)
    body = bytes([8]) + struct.pack(">HH", height, width) + bytes([len(comps)])
    for i, c in enumerate(comps):
        body += bytes([i + 1, (c.h << 4) | c.v, c.table])
    out += b"\xff\xc0" + struct.pack(">H", len(body) + 2) + body
    tables = [(0, 0, DC_LUMA_BITS, DC_VALS), (1, 0, AC_LUMA_BITS, AC_LUMA_VALS),
              (0, 1, DC_CHROMA_BITS, DC_VALS), (1, 1, AC_CHROMA_BITS, AC_CHROMA_VALS)]
    for tc, th, bits, vals in tables:
        body = bytes([(tc << 4) | th]) + bytes(bits) + bytes(vals)
        out += b"\xff\xc4" + struct.pack(">H", len(body) + 2) + body
    if restart_interval:
        out += b"\xff\xdd" + struct.pack(">HH", 4, restart_interval)
    sel = [0 if i == 0 else 1 for i in range(len(comps))]
    if separate_scans and len(comps) > 1:
        for ci, c in enumerate(comps):
            if ci in omit_scans:
                continue
            cw = -(-width * c.h // hmax)
            ch = -(-height * c.v // vmax)
            units = [[(ci, by * c.block_w + bx)] for by in range(-(-ch // 8)) for bx in range(-(-cw // 8))]
            out += _scan(comps, [ci], sel, units, restart_interval)
        return bytes(out + b"\xff\xd9")
    if len(comps) == 1:
        c = comps[0]
        units = [[(0, by * c.block_w + bx)] for by in range((height + 7) // 8) for bx in range((width + 7) // 8)]
    else:
        mcu_w = (width + 8 * hmax - 1) // (8 * hmax)
        mcu_h = (height + 8 * vmax - 1) // (8 * vmax)
        units = []
        for my in range(mcu_h):
            for mx in range(mcu_w):
                u = []
                for ci, c in enumerate(comps):
                    for vv in range(c.v):
                        for hh in range(c.h):
                            u.append((ci, (my * c.v + vv) * c.block_w + mx * c.h + hh))
                units.append(u)
    return bytes(out + _scan(comps, list(range(len(comps))), sel, units, restart_interval) + b"\xff\xd9")


def _scan(comps: List[Component], members: List[int], sel: List[int], units, restart_interval: int) -> bytes:
    """SOS header for the scan's components plus its entropy-coded data."""
    body = bytes([len(members)])
    for i in members:
        body += bytes([i + 1, (sel[i] << 4) | sel[i]])
    body += bytes([0, 63, 0])
    out = bytearray(b"\xff\xda" + struct.pack(">H", len(body) + 2) + body)

    dc_codes = [_codes(DC_LUMA_BITS, DC_VALS), _codes(DC_CHROMA_BITS, DC_VALS)]
    ac_codes = [_codes(AC_LUMA_BITS, AC_LUMA_VALS), _codes(AC_CHROMA_BITS, AC_CHROMA_VALS)]
    bw = _Bits()
    preds = [0] * len(comps)

    def block(ci: int, blk: np.ndarray):
        zz = blk[ZIGZAG]
        diff = int(zz[0]) - preds[ci]
        preds[ci] = int(zz[0])
        t = _category(diff)
        code, ln = dc_codes[sel[ci]][t]
        bw.put(code, ln)
        if t:
            bw.put(_magnitude_bits(diff, t), t)
        run = 0
        for k in range(1, 64):
            v = int(zz[k])
            if v == 0:
                run += 1
                continue
            while run > 15:
                code, ln = ac_codes[sel[ci]][0xF0]
                bw.put(code, ln)
                run -= 16
            s = _category(v)
            code, ln = ac_codes[sel[ci]][(run << 4) | s]
            bw.put(code, ln)
            bw.put(_magnitude_bits(v, s), s)
            run = 0
        if run:
            code, ln = ac_codes[sel[ci]][0x00]
            bw.put(code, ln)

    rst = 0
    for n, u in enumerate(units):
        if restart_interval and n and n % restart_interval == 0:
            bw.flush()
            bw.out += bytes([0xFF, 0xD0 + (rst & 7)])
            rst += 1
            preds[:] = [0] * len(comps)
        for ci, bi in u:
            block(ci, comps[ci].coefs[bi])
    bw.flush()
    out += bw.out
    return bytes(out)


def random_image(rng: np.random.Generator, width: int, height: int, sampling: Sequence[tuple],
                 qt_max: int = 255) -> tuple:
    """Random quantised coefficients for the given sampling factors.

    Returns (jpeg bytes, list of (coefs int16 (nblocks, 64), qt float32 (64,),
    block_w, block_h, samp_h, samp_v))."""
    hmax = max(h for h, _ in sampling)
    vmax = max(v for _, v in sampling)
    if len(sampling) == 1:
        hmax = vmax = 1
    rw = -(-width // (8 * hmax)) * 8 * hmax
    rh = -(-height // (8 * vmax)) * 8 * vmax
    comps, expect = [], []
    for ci, (h, v) in enumerate(sampling):
        if len(sampling) == 1:
            h = v = 1
        bw_, bh_ = rw // (hmax // h) // 8, rh // (vmax // v) // 8
        n = bw_ * bh_
        coefs = np.zeros((n, 64), dtype=np.int64)
        coefs[:, 0] = rng.integers(-1024, 1024, n)
        mask = rng.random((n, 63)) < 0.3
        coefs[:, 1:] = np.where(mask, rng.integers(-60, 61, (n, 63)), 0)
        big = rng.random((n, 63)) < 0.01
        coefs[:, 1:] = np.where(big, rng.integers(-1023, 1024, (n, 63)), coefs[:, 1:])
        qt = rng.integers(1, qt_max + 1, 64)
        comps.append(Component(h, v, qt, coefs, bw_, bh_, ci))
        expect.append((coefs.astype(np.int16), qt.astype(np.float32), bw_, bh_, hmax // h, vmax // v))
    return comps, expect, (rw, rh)
