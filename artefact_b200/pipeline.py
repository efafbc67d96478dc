"""Many JPEGs through ``Artefact::process`` with decoding and solving overlapped.

The reference processes one file per call: ``Jpeg::from`` decodes on the host
(jpeg/zune.rs:5-55), then ``process`` solves and converts (lib.rs:105-212).
For a stream of files the host decode of later images runs while the GPU
solves earlier ones. A pool of `decoders` host threads runs the baseline
decoder (``art_jpeg_decode``; ctypes releases the GIL for the native call).
Decoded images are grouped, in input order, into batches of at most
`batch_images` images or `batch_pixels` pixels, and each batch is one
``art_context_process_batch`` call (one batched solve of all its images, then
the fused RGB stage) on one of `solvers` contexts, each with its own CUDA
stream, so one batch's copies overlap another's kernels. Results come back
in input order, exactly as ``process_jpeg`` returns them for the same
options. Contexts created here are closed when the stream ends; contexts the
caller passes in stay open, with their buffers sized and graphs captured.
"""
from __future__ import annotations

import queue
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from typing import Callable, Iterable, Iterator, List, Optional, Sequence

import numpy as np

from .api import Context, Jpeg, JpegSource, process_jpeg, process_jpegs


def _decode(data: bytes) -> Jpeg:
    return Jpeg.from_source(JpegSource.Buffer(data))


def process_stream(datas: Iterable[bytes], weight: Sequence[float] = (0.3,) * 3,
                   pweight: Sequence[float] = (0.001,) * 3, iterations: Sequence[int] = (50,) * 3,
                   separate: bool = False, *, decoders: int = 4, solvers: int = 2, depth: int = 0,
                   batch_images: int = 32, batch_pixels: int = 32 << 20, device: int = -1,
                   solve: Optional[Callable[[Jpeg], np.ndarray]] = None,
                   contexts: Optional[Sequence[Context]] = None) -> Iterator[np.ndarray]:
    """Yields the RGB8 image of each JPEG in `datas`, in order, keeping up to
    `depth` decoded or decoding images ahead of the batches being solved
    (0: twice a batch). `batch_images` = 1 solves image by image
    (``art_context_process``). `contexts` (one per solver; default: created
    here and closed at the end) lets a long-running caller keep their device
    buffers and captured graphs from one stream to the next. `solve` replaces
    the GPU call per image (tests)."""
    if decoders < 1 or solvers < 1 or batch_images < 1 or batch_pixels < 1 or depth < 0:
        raise ValueError("decoders, solvers, batch_images and batch_pixels must be at least 1, depth at least 0")
    if contexts is not None and len(contexts) != solvers:
        raise ValueError("give one context per solver")
    depth = depth or 2 * batch_images
    owned: list = []
    if solve is not None:
        def solve_batch(group: List[Jpeg]) -> List[np.ndarray]:
            return [solve(j) for j in group]
    else:
        # One explicit context (stream, buffers, graph) per solver slot, lent
        # to whichever solver thread runs the next batch.
        if contexts is None:
            owned = [Context(device) for _ in range(solvers)]
            contexts = owned
        free: queue.Queue = queue.Queue()
        for c in contexts:
            free.put(c)

        def solve_batch(group: List[Jpeg]) -> List[np.ndarray]:
            ctx = free.get()
            try:
                if len(group) == 1:
                    return [process_jpeg(group[0], list(weight), list(pweight), list(iterations), separate,
                                         context=ctx)]
                return process_jpegs(group, list(weight), list(pweight), list(iterations), separate, context=ctx)
            finally:
                free.put(ctx)
    try:
        yield from _run(iter(datas), solve_batch, decoders, solvers, depth, batch_images, batch_pixels)
    finally:
        for c in owned:
            c.close()


def _run(it, solve_batch, decoders: int, solvers: int, depth: int, batch_images: int,
         batch_pixels: int) -> Iterator[np.ndarray]:
    with ThreadPoolExecutor(decoders) as dec, ThreadPoolExecutor(solvers) as sol:
        decoding: deque = deque()
        batches: deque = deque()
        exhausted = False

        def fill() -> None:
            nonlocal exhausted
            while not exhausted and len(decoding) < depth:
                try:
                    data = next(it)
                except StopIteration:
                    exhausted = True
                    return
                decoding.append(dec.submit(_decode, data))

        fill()
        while decoding or batches:
            # Keep `solvers` batches in flight; a batch takes decoded images in
            # input order up to its image and pixel budgets.
            # An image that failed to decode ends its batch; its error is raised
            # after the images before it have been yielded.
            while decoding and len(batches) < solvers:
                group, px = [], 0
                while decoding and len(group) < batch_images and px < batch_pixels:
                    if group and decoding[0].exception() is not None:
                        break
                    j = decoding.popleft().result()
                    group.append(j)
                    px += j.real_px_w * j.real_px_h
                    fill()
                if not group:
                    break
                batches.append(sol.submit(solve_batch, group))
            if not batches:
                decoding.popleft().result()  # raises the decode error at the head of the stream
                continue
            out = batches.popleft().result()
            fill()
            yield from out
