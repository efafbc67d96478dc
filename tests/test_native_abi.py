"""The C-ABI library loads and exports every function include/*.h declares (CPU only)."""
import ctypes as C
import re
from pathlib import Path

from artefact_b200 import _native as N

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names.update(re.findall(r"\b(art_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("art_compute", "art_context_compute", "art_context_compute_device", "art_context_process",
                     "art_jpeg_decode", "art_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(N.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_symbol():
    assert set(declared_functions()) <= set(N.EXPORTS)


def test_version_and_error_without_gpu():
    lib = N.lib()
    assert b"sm_100a" in lib.art_version()
    assert isinstance(lib.art_last_error(), bytes)


def test_host_api_mirrors_reference_defaults():
    from artefact_b200 import Artefact, ValueCollection

    a = Artefact.default()
    assert a._weight.to_slice() == [0.3] * 3
    assert a._pweight.to_slice() == [0.001] * 3
    assert a._iterations.to_slice() == [50] * 3
    assert ValueCollection.ForEach([1, 2, 3]).to_slice() == [1, 2, 3]


def test_process_without_source_errors():
    import pytest

    from artefact_b200 import Artefact, ArtefactError

    with pytest.raises(ArtefactError, match="Source is not set"):
        Artefact.default().process()
