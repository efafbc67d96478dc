"""artefact_b200: B200-native (sm_100a) JPEG restoration solver.

Drop-in for the solver of Delnegend/artefact's artefact-lib: the same
``compute`` entry point and ``Artefact`` builder, backed by hand-written CUDA
kernels in ``libartefact_b200.so`` (C ABI: include/artefact_b200.h).
"""
from .api import (Artefact, ArtefactError, Coefficient, Context, Jpeg, JpegSource, ValueCollection, compute,
                  process_jpeg)
from ._native import ART_INIT_DECODED, ART_INIT_SCALAR_COMPAT, ArtError

__all__ = [
    "Artefact", "ArtefactError", "ArtError", "Coefficient", "Context", "Jpeg", "JpegSource", "ValueCollection", "compute",
    "process_jpeg", "ART_INIT_DECODED", "ART_INIT_SCALAR_COMPAT",
]
__version__ = "0.1.0"
