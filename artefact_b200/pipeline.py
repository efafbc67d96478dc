"""Many JPEGs through ``Artefact::process`` with decoding and solving overlapped.

The reference processes one file per call: ``Jpeg::from`` decodes on the host
(jpeg/zune.rs:5-55), then ``process`` solves and converts (lib.rs:105-212).
For a stream of files the host decode of later images can run while the GPU
solves earlier ones. Here a pool of `decoders` host threads runs the baseline
decoder (``art_jpeg_decode``; ctypes releases the GIL for the native call)
and `solvers` threads submit ``art_context_process`` calls. Each solver thread
has its own context and CUDA stream, so one image's copies overlap another's
kernels. Results come back in input order, exactly as ``process_jpeg``
returns them for the same options; the contexts are closed when the stream
ends.
"""
from __future__ import annotations

import queue
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from typing import Callable, Iterable, Iterator, Optional, Sequence

import numpy as np

from .api import Context, Jpeg, JpegSource, process_jpeg


def _decode(data: bytes) -> Jpeg:
    return Jpeg.from_source(JpegSource.Buffer(data))


def process_stream(datas: Iterable[bytes], weight: Sequence[float] = (0.3,) * 3,
                   pweight: Sequence[float] = (0.001,) * 3, iterations: Sequence[int] = (50,) * 3,
                   separate: bool = False, *, decoders: int = 4, solvers: int = 2, depth: int = 8,
                   device: int = -1, solve: Optional[Callable[[Jpeg], np.ndarray]] = None) -> Iterator[np.ndarray]:
    """Yields the RGB8 image of each JPEG in `datas`, in order, keeping up to
    `depth` images in flight. `solve` replaces the GPU call (tests)."""
    if depth < 1 or decoders < 1 or solvers < 1:
        raise ValueError("depth, decoders and solvers must be at least 1")
    contexts: list = []
    if solve is None:
        # One explicit context (stream, buffers, graph) per solver slot, lent
        # to whichever solver thread runs the next image and closed at the end.
        contexts = [Context(device) for _ in range(solvers)]
        free: queue.Queue = queue.Queue()
        for c in contexts:
            free.put(c)

        def solve(j: Jpeg) -> np.ndarray:
            ctx = free.get()
            try:
                return process_jpeg(j, list(weight), list(pweight), list(iterations), separate, context=ctx)
            finally:
                free.put(ctx)
    try:
        yield from _run(iter(datas), solve, decoders, solvers, depth)
    finally:
        for c in contexts:
            c.close()


def _run(it, solve, decoders: int, solvers: int, depth: int) -> Iterator[np.ndarray]:
    with ThreadPoolExecutor(decoders) as dec, ThreadPoolExecutor(solvers) as sol:
        pending: deque = deque()

        def submit_next() -> bool:
            try:
                data = next(it)
            except StopIteration:
                return False
            djob = dec.submit(_decode, data)
            pending.append(sol.submit(lambda f=djob: solve(f.result())))
            return True

        for _ in range(depth):
            if not submit_next():
                break
        while pending:
            out = pending.popleft().result()
            submit_next()
            yield out
