"""Host-side mirror of artefact-lib's public API, backed by the CUDA library.

Names, argument meanings and error behaviour follow Delnegend/artefact
``backend/artefact-lib`` (citations are file:line there):

* :func:`compute` is ``pipeline_scalar::compute`` (pipeline_scalar/mod.rs:17-78),
* :class:`Coefficient` / :class:`Jpeg` / :class:`JpegSource` are jpeg/mod.rs:8-42,
* :class:`ValueCollection` and :class:`Artefact` are lib.rs:34-212.
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass, field
from typing import Generic, List, Optional, Sequence, TypeVar, Union

import numpy as np

from . import _native as N

T = TypeVar("T")


@dataclass
class Coefficient:
    """One JPEG component as the solver receives it (jpeg/mod.rs:8-27)."""

    rounded_px_w: int
    rounded_px_h: int
    block_w: int
    block_h: int
    horizontal_samp_factor: int
    vertical_samp_factor: int
    dct_coefs: np.ndarray  # block_w*block_h*64 values (float32 or int16), block raster, natural order;
    #                        read-only when it views a decoded JPEG (Jpeg.from_source): copy() before editing
    quant_table: np.ndarray  # 64 float32, natural order

    @property
    def rounded_px_count(self) -> int:
        return self.rounded_px_w * self.rounded_px_h

    @property
    def block_count(self) -> int:
        return self.block_w * self.block_h

    def as_c(self, keep: list) -> N.ArtChannel:
        coefs = self.dct_coefs
        if coefs.dtype == np.int16:
            ctype = N.ART_COEF_I16
        else:
            coefs = coefs.astype(np.float32, copy=False)
            ctype = N.ART_COEF_F32
        coefs = np.ascontiguousarray(coefs)
        if coefs.size != self.block_count * 64:
            raise ValueError("Invalid coef's image data length")
        q = np.ascontiguousarray(self.quant_table, dtype=np.float32)
        if q.size != 64:
            raise ValueError("Invalid quant_table length")
        keep.extend([coefs, q])
        ch = N.ArtChannel()
        ch.rounded_px_w, ch.rounded_px_h = self.rounded_px_w, self.rounded_px_h
        ch.block_w, ch.block_h = self.block_w, self.block_h
        ch.samp_h, ch.samp_v = self.horizontal_samp_factor, self.vertical_samp_factor
        ch.coef_type = ctype
        ch.dct_coefs = coefs.ctypes.data
        ch.quant_table = q.ctypes.data_as(C.POINTER(C.c_float))
        return ch


@dataclass
class JpegSource:
    """``JpegSource::File(path)`` or ``JpegSource::Buffer(bytes)`` (jpeg/mod.rs:38-42)."""

    path: Optional[str] = None
    buffer: Optional[bytes] = None

    @staticmethod
    def File(path: str) -> "JpegSource":  # noqa: N802 - mirrors the Rust enum variant
        return JpegSource(path=str(path))

    @staticmethod
    def Buffer(data: bytes) -> "JpegSource":  # noqa: N802
        return JpegSource(buffer=bytes(data))

    def read(self) -> bytes:
        if self.buffer is not None:
            return self.buffer
        try:
            with open(self.path, "rb") as fh:
                return fh.read()
        except OSError as e:
            raise ArtefactError(f"Failed to read JPEG file '{self.path}': {e}") from e


class _NativeJpeg:
    """Owns a decoded image of art_jpeg_decode; freed when the last coefficient
    array viewing its memory is gone."""

    def __init__(self, lib, handle):
        self._lib, self._h = lib, handle

    def __del__(self):
        h, self._h = self._h, None
        if h:
            try:
                self._lib.art_jpeg_free(h)
            except Exception:  # interpreter shutdown
                pass


class _NativePlane:
    """int16 plane inside a _NativeJpeg, exposed to numpy without a copy as a
    read-only array (copy() it before editing coefficients); the array keeps
    this object (and so the decoded image) alive."""

    def __init__(self, owner: _NativeJpeg, address: int, n: int):
        self._owner = owner
        self.__array_interface__ = {"data": (address, True), "shape": (n,), "typestr": "<i2", "version": 3}


@dataclass
class Jpeg:
    """Decoded coefficient data of a JPEG (jpeg/mod.rs:29-36, jpeg/zune.rs:5-55)."""

    nchannel: int
    real_px_w: int
    real_px_h: int
    coefs: List[Coefficient] = field(default_factory=list)

    @staticmethod
    def from_source(source: JpegSource) -> "Jpeg":
        data = source.read()
        lib = N.lib()
        handle = C.c_void_p()
        rc = lib.art_jpeg_decode(data, len(data), C.byref(handle))
        if rc != N.ART_OK:
            raise ArtefactError(lib.art_last_error().decode("utf-8", "replace"))
        # The coefficient arrays are read-only views of the decoder's planes
        # (no copy); the decoded image is freed with the last of them.
        owner = _NativeJpeg(lib, handle)
        nch, rw, rh = C.c_uint32(), C.c_uint32(), C.c_uint32()
        N.check(lib.art_jpeg_info(handle, C.byref(nch), C.byref(rw), C.byref(rh)))
        coefs = []
        for c in range(nch.value):
            ch = N.ArtChannel()
            N.check(lib.art_jpeg_channel(handle, c, C.byref(ch)))
            n = ch.block_w * ch.block_h * 64
            arr = np.asarray(_NativePlane(owner, ch.dct_coefs, n))
            q = np.ctypeslib.as_array(ch.quant_table, shape=(64,)).copy()
            coefs.append(Coefficient(ch.rounded_px_w, ch.rounded_px_h, ch.block_w, ch.block_h,
                                     ch.samp_h, ch.samp_v, arr, q))
        return Jpeg(nch.value, rw.value, rh.value, coefs)

    def max_rounded(self):
        """Largest rounded component size (lib.rs:108-116)."""
        w = max(c.rounded_px_w for c in self.coefs)
        h = max(c.rounded_px_h for c in self.coefs)
        return w, h, w * h


class ArtefactError(RuntimeError):
    """Error of :meth:`Artefact.process` (the reference's ``Err(String)``)."""


def _options(init_mode: int, device: int, step_iterations: int = 0, tail_iterations: int = 0,
             tail_step_iterations: int = 0, step_decay: float = 0.0) -> N.ArtOptions:
    o = N.ArtOptions()
    o.init_mode = init_mode
    o.device = device
    o.step_iterations = int(step_iterations)
    o.tail_iterations = int(tail_iterations)
    o.tail_step_iterations = int(tail_step_iterations)
    o.step_decay = float(step_decay)
    return o


def compute(nchannel: int, coefs: Sequence[Coefficient], weight: float, pweight: Sequence[float], iterations: int,
            max_rounded_px_w: int, max_rounded_px_h: int, max_rounded_px_count: int, *,
            init_mode: int = N.ART_INIT_DECODED, device: int = -1) -> List[np.ndarray]:
    """Run the solver; the B200 replacement of ``pipeline_scalar::compute``.

    Returns ``nchannel`` float32 planes of ``max_rounded_px_count`` values (row
    stride ``max_rounded_px_w``), level-shifted like the reference's output.
    Channel ``c`` uses ``pweight[c]`` (compute_step.rs:19-26).
    """
    lib = N.lib()
    keep: list = []
    chans = (N.ArtChannel * nchannel)(*[coefs[c].as_c(keep) for c in range(nchannel)])
    pw = (C.c_float * 3)(*[float(v) for v in list(pweight)[:3]] + [0.0] * (3 - min(3, len(pweight))))
    outs = [np.empty(max_rounded_px_count, dtype=np.float32) for _ in range(nchannel)]
    ptrs = (C.c_void_p * nchannel)(*[o.ctypes.data for o in outs])
    opts = _options(init_mode, device)
    rc = lib.art_compute(nchannel, chans, float(weight), pw, int(iterations), max_rounded_px_w, max_rounded_px_h,
                         max_rounded_px_count, ptrs, C.byref(opts))
    N.check(rc)
    return outs


class ValueCollection(Generic[T]):
    """``ValueCollection::ForAll(v)`` / ``ForEach([a, b, c])`` (lib.rs:34-47)."""

    def __init__(self, values: Sequence[T]):
        self._values = list(values)

    @staticmethod
    def ForAll(v: T) -> "ValueCollection[T]":  # noqa: N802
        return ValueCollection([v, v, v])

    @staticmethod
    def ForEach(v: Sequence[T]) -> "ValueCollection[T]":  # noqa: N802
        if len(v) != 3:
            raise ValueError("ForEach takes exactly three values")
        return ValueCollection(list(v))

    def to_slice(self) -> List[T]:
        return list(self._values)


_tls = threading.local()


def _context(device: int = -1):
    ctxs = getattr(_tls, "ctxs", None)
    if ctxs is None:
        ctxs = _tls.ctxs = {}
    if device not in ctxs:
        h = C.c_void_p()
        N.check(N.lib().art_context_create(device, C.byref(h)))
        ctxs[device] = h
    return ctxs[device]


class Artefact:
    """Builder of one restoration run (lib.rs:49-212); defaults 0.3 / 0.001 / 50."""

    def __init__(self):
        self._weight = ValueCollection.ForAll(0.3)
        self._pweight = ValueCollection.ForAll(0.001)
        self._iterations = ValueCollection.ForAll(50)
        self._separate = False
        self._benchmark = False
        self._source: Optional[JpegSource] = None
        self._init_mode = N.ART_INIT_DECODED
        self._device = -1

    @staticmethod
    def default() -> "Artefact":
        return Artefact()

    def source(self, source: JpegSource) -> "Artefact":
        self._source = source
        return self

    def weight(self, v: Union[ValueCollection, float]) -> "Artefact":
        self._weight = v if isinstance(v, ValueCollection) else ValueCollection.ForAll(float(v))
        return self

    def pweight(self, v: Union[ValueCollection, float]) -> "Artefact":
        self._pweight = v if isinstance(v, ValueCollection) else ValueCollection.ForAll(float(v))
        return self

    def iterations(self, v: Union[ValueCollection, int]) -> "Artefact":
        self._iterations = v if isinstance(v, ValueCollection) else ValueCollection.ForAll(int(v))
        return self

    def benchmark(self, v: bool) -> "Artefact":
        self._benchmark = bool(v)
        return self

    def separate_components(self, v: bool) -> "Artefact":
        self._separate = bool(v)
        return self

    def init_mode(self, mode: int) -> "Artefact":
        self._init_mode = int(mode)
        return self

    def device(self, device: int) -> "Artefact":
        self._device = int(device)
        return self

    def process(self) -> np.ndarray:
        """Decode, solve and convert to RGB8 (lib.rs:105-212).

        Returns an ``(real_h, real_w, 3)`` uint8 array. Raises
        :class:`ArtefactError` on decode errors, and with the message
        ``"BENCHMARK"`` when benchmark mode is set (lib.rs:155-157).
        """
        if self._source is None:
            raise ArtefactError("Source is not set")
        try:
            jpeg = Jpeg.from_source(self._source)
        except ArtefactError as e:
            raise ArtefactError(f"Failed to read JPEG: {e}") from e
        return process_jpeg(jpeg, self._weight.to_slice(), self._pweight.to_slice(), self._iterations.to_slice(),
                            self._separate, self._benchmark, init_mode=self._init_mode, device=self._device)


def process_jpeg(jpeg: Jpeg, weight: Sequence[float], pweight: Sequence[float], iterations: Sequence[int],
                 separate: bool, benchmark: bool = False, *, init_mode: int = N.ART_INIT_DECODED,
                 device: int = -1, context: Optional["Context"] = None) -> np.ndarray:
    """Solver dispatch and output stage of ``Artefact::process`` on decoded
    data, on `context` (default: the calling thread's own context)."""
    lib = N.lib()
    keep: list = []
    n = jpeg.nchannel
    chans = (N.ArtChannel * n)(*[c.as_c(keep) for c in jpeg.coefs])
    w = (C.c_float * 3)(*[float(v) for v in weight])
    pw = (C.c_float * 3)(*[float(v) for v in pweight])
    it = (C.c_uint32 * 3)(*[int(v) for v in iterations])
    rgb = None if benchmark else np.empty((jpeg.real_px_h, jpeg.real_px_w, 3), dtype=np.uint8)
    opts = _options(init_mode, device)
    handle = context.handle if context is not None else _context(device)
    rc = lib.art_context_process(handle, n, chans, w, pw, it, int(bool(separate)), jpeg.real_px_w,
                                 jpeg.real_px_h, None if rgb is None else rgb.ctypes.data, C.byref(opts))
    N.check(rc)
    if benchmark:
        raise ArtefactError("BENCHMARK")
    return rgb


def process_jpegs(jpegs: Sequence[Jpeg], weight: Sequence[float], pweight: Sequence[float],
                  iterations: Sequence[int], separate: bool, *, init_mode: int = N.ART_INIT_DECODED,
                  device: int = -1, context: Optional["Context"] = None) -> List[np.ndarray]:
    """:func:`process_jpeg` for many decoded images, solved as one batch
    (``art_context_process_batch``): the RGB8 image of each, in order, equal
    to what :func:`process_jpeg` returns for it. The batch runs one iteration
    count: ``iterations[0]`` for joint solves (as the reference, lib.rs:122-132);
    in separate mode with different per-component counts the images go one by
    one through :func:`process_jpeg` instead."""
    jpegs = list(jpegs)
    if not jpegs:
        return []
    its = [int(v) for v in iterations]
    counts = {its[0]} if not separate and all(j.nchannel == 3 for j in jpegs) else set(
        its[min(c, len(its) - 1)] for j in jpegs for c in range(j.nchannel if j.nchannel != 3 or separate else 1))
    if len(counts) != 1:
        return [process_jpeg(j, weight, pweight, iterations, separate, init_mode=init_mode, device=device,
                             context=context) for j in jpegs]
    lib = N.lib()
    keep: list = []
    imgs = (N.ArtProcessImage * len(jpegs))()
    outs = []
    w3 = [float(v) for v in (list(weight) + [0.0] * 3)[:3]]
    pw3 = [float(v) for v in (list(pweight) + [0.0] * 3)[:3]]
    for i, j in enumerate(jpegs):
        chans = (N.ArtChannel * j.nchannel)(*[c.as_c(keep) for c in j.coefs])
        keep.append(chans)
        rgb = np.empty((j.real_px_h, j.real_px_w, 3), dtype=np.uint8)
        outs.append(rgb)
        im = imgs[i]
        im.nchannel, im.real_w, im.real_h = j.nchannel, j.real_px_w, j.real_px_h
        im.channels = C.cast(chans, C.POINTER(N.ArtChannel))
        im.weight = (C.c_float * 3)(*w3)
        im.pweight = (C.c_float * 3)(*pw3)
        im.rgb_out = rgb.ctypes.data
    handle = context.handle if context is not None else _context(device)
    N.check(lib.art_context_process_batch(handle, len(jpegs), imgs, counts.pop(), int(bool(separate)),
                                          C.byref(_options(init_mode, device))))
    return outs


def _tune_dict(r) -> dict:
    return dict(variant=r.variant, strip_rows=r.strip_rows, proj_warps=r.proj_warps, candidates=r.candidates,
                best_ms=r.best_ms, heuristic_ms=r.heuristic_ms, heuristic_variant=r.heuristic_variant,
                heuristic_strip_rows=r.heuristic_strip_rows)


class Context:
    """An explicit solver context (``art_context_*``): one CUDA stream, device
    buffers, the captured iteration graph and the autotuner's cache, reused
    across calls. Not to be shared by two threads at once."""

    def __init__(self, device: int = -1):
        self._h = C.c_void_p()
        N.check(N.lib().art_context_create(device, C.byref(self._h)))

    def close(self) -> None:
        if self._h:
            N.lib().art_context_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def set_warm_start(self, net) -> None:
        """Attach a :class:`artefact_b200.warmstart.WarmStartNet` (or None) for
        ``init_mode=ART_INIT_LEARNED`` solves; the context does not own it."""
        self._net = net
        N.check(N.lib().art_context_set_warm_start(self._h, net.handle if net is not None else None))

    def set_joint_warm_start(self, net) -> None:
        """Attach a joint 4:2:0 network (or None): learned solves of 4:2:0
        images predict all three components with it in one pass
        (``art_context_set_joint_warm_start``)."""
        self._net_joint = net
        N.check(N.lib().art_context_set_joint_warm_start(self._h, net.handle if net is not None else None))

    def evaluate(self, image: int = 0) -> dict:
        """Objective and feasibility of the last solve's result for `image`
        (``art_context_evaluate``, fp64 on the GPU): keys E, tv, tgv, prob, infeasibility."""
        out = (C.c_double * 5)()
        N.check(N.lib().art_context_evaluate(self._h, int(image), out))
        return dict(E=out[0], tv=out[1], tgv=out[2], prob=out[3], infeasibility=out[4])

    def compute(self, nchannel: int, coefs: Sequence[Coefficient], weight: float, pweight: Sequence[float],
                iterations: int, max_rounded_px_w: int, max_rounded_px_h: int,
                init_mode: int = N.ART_INIT_DECODED, step_iterations: int = 0, tail_iterations: int = 0,
                tail_step_iterations: int = 0, step_decay: float = 0.0) -> List[np.ndarray]:
        keep: list = []
        chans = (N.ArtChannel * nchannel)(*[coefs[c].as_c(keep) for c in range(nchannel)])
        pw = (C.c_float * 3)(*[float(v) for v in list(pweight)[:3]])
        outs = [np.empty(max_rounded_px_w * max_rounded_px_h, np.float32) for _ in range(nchannel)]
        ptrs = (C.c_void_p * nchannel)(*[o.ctypes.data for o in outs])
        N.check(N.lib().art_context_compute(self._h, nchannel, chans, float(weight), pw, int(iterations),
                                            max_rounded_px_w, max_rounded_px_h, ptrs,
                                            C.byref(_options(init_mode, -1, step_iterations, tail_iterations,
                                                             tail_step_iterations, step_decay))))
        return outs

    def compute_batch(self, jobs: Sequence[dict], iterations: int, init_mode: int = N.ART_INIT_DECODED,
                      step_iterations: int = 0, tail_iterations: int = 0,
                      tail_step_iterations: int = 0, step_decay: float = 0.0) -> List[List[np.ndarray]]:
        """Solve many images together (one launch per kernel and iteration over
        all of them, the loop in one CUDA graph). Each job is a dict with keys
        ``coefs`` (list of :class:`Coefficient`), ``weight``, ``pweight`` and
        optionally ``nchannel``, ``max_w``, ``max_h`` (default: from the coefs)."""
        keep: list = []
        imgs, results = self._images(jobs, keep)
        N.check(N.lib().art_context_compute_batch(self._h, len(jobs), imgs, int(iterations),
                                                  C.byref(_options(init_mode, -1, step_iterations, tail_iterations,
                                                                   tail_step_iterations, step_decay))))
        return results

    def _images(self, jobs: Sequence[dict], keep: list):
        """ArtImage array of host coefficients (and host output planes) for `jobs`."""
        imgs = (N.ArtImage * len(jobs))()
        results = []
        for i, job in enumerate(jobs):
            coefs = job["coefs"]
            n = job.get("nchannel", len(coefs))
            w = job.get("max_w", max(c.rounded_px_w for c in coefs))
            h = job.get("max_h", max(c.rounded_px_h for c in coefs))
            chans = (N.ArtChannel * n)(*[coefs[c].as_c(keep) for c in range(n)])
            outs = [np.empty(w * h, np.float32) for _ in range(n)]
            ptrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
            keep += [chans, ptrs]
            im = imgs[i]
            im.nchannel, im.max_rounded_px_w, im.max_rounded_px_h, im.out_pitch = n, w, h, w
            im.channels = C.cast(chans, C.POINTER(N.ArtChannel))
            im.weight = float(job.get("weight", 0.3))
            pw = list(job.get("pweight", [0.001] * 3))
            im.pweight = (C.c_float * 3)(*[float(v) for v in (pw + [0.0] * 3)[:3]])
            im.out_planes = C.cast(ptrs, C.POINTER(C.c_void_p))
            results.append(outs)
        return imgs, results

    def autotune_batch(self, jobs: Sequence[dict], iterations: int = 10) -> dict:
        """Tune the launch shapes on this batch of images (jobs as for
        :meth:`compute_batch`); later batches of its bucket use the choice.
        Returns the choice and the timings (``art_context_autotune_batch``)."""
        keep: list = []
        imgs, _ = self._images(jobs, keep)
        r = N.ArtTuneResult()
        N.check(N.lib().art_context_autotune_batch(self._h, len(jobs), imgs, int(iterations), C.byref(r)))
        d = _tune_dict(r)
        d["candidates_ms"] = self.tune_candidates()
        return d

    def last_tune(self) -> dict:
        """Choice and timings of the last autotune run on this context."""
        r = N.ArtTuneResult()
        N.check(N.lib().art_context_last_tune(self._h, C.byref(r)))
        d = _tune_dict(r)
        d["candidates_ms"] = self.tune_candidates()
        return d

    def tune_candidates(self) -> list:
        """Every (variant, strip_rows, proj_warps, ms) the last autotune run timed."""
        n = C.c_uint32()
        N.check(N.lib().art_context_tune_candidates(self._h, None, 0, C.byref(n)))
        arr = (N.ArtTuneCandidate * max(1, n.value))()
        N.check(N.lib().art_context_tune_candidates(self._h, arr, n.value, C.byref(n)))
        return [(c.variant, c.strip_rows, c.proj_warps, c.ms) for c in arr[:n.value]]

    def autotune(self, nchannel: int, samp_h: Sequence[int], samp_v: Sequence[int], max_w: int, max_h: int,
                 iterations: int = 10) -> tuple:
        """Time the sweep variants and strip heights for this geometry; returns (and
        caches) the fastest as (variant, strip_rows), variant 0 narrow or 1 wide."""
        sh = (C.c_uint32 * 3)(*(list(samp_h) + [1, 1, 1])[:3])
        sv = (C.c_uint32 * 3)(*(list(samp_v) + [1, 1, 1])[:3])
        kind, rows = C.c_uint32(), C.c_uint32()
        N.check(N.lib().art_context_autotune(self._h, nchannel, sh, sv, max_w, max_h, iterations, C.byref(kind),
                                             C.byref(rows)))
        return kind.value, rows.value

    def save_tune_cache(self, path: str) -> None:
        N.check(N.lib().art_context_tune_cache(self._h, str(path).encode(), 1))

    def load_tune_cache(self, path: str) -> None:
        N.check(N.lib().art_context_tune_cache(self._h, str(path).encode(), 0))
