"""The C-ABI library loads and exports every entry point include/pxl.h declares
(no compute call: no GPU needed)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> list[str]:
    text = (ROOT / "include" / "pxl.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pxl_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from pixeltrack import _native
    lib = ctypes.CDLL(str(_native.LIBDIR / "libpxl_b200.so"))
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_the_header():
    from pixeltrack import _native
    assert set(declared_functions()) == set(_native.exported_symbols())


def test_version_without_gpu():
    from pixeltrack import _native
    assert _native.lib().pxl_version() == 3


def test_params_default_are_the_reference_capacities():
    from pixeltrack.chain import default_params
    p = default_params()
    assert p.hits_per_event == 48 * 1024
    assert p.doublets_per_event == 458752
    assert p.tuples_per_event == 32 * 1024
    assert p.fits_per_multiplicity == 24 * 1024
    assert p.columns_per_event == 64 * 1024
    assert p.max_words == 150 * 2000


def test_params_extended_raise_only_the_per_event_capacities():
    from pixeltrack.chain import default_params, extended_params
    d, x = default_params(), extended_params()
    assert x.hits_per_event == 256 * 1024 and x.doublets_per_event == 4 * 1024 * 1024
    assert x.tuples_per_event == 256 * 1024 and x.fits_per_multiplicity == 256 * 1024
    assert x.columns_per_event == 4 * 1024 * 1024
    for f in ("max_events", "max_words", "max_hits", "max_doublets", "max_tuples", "include_errors", "use_quality"):
        assert getattr(x, f) == getattr(d, f)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from pixeltrack import _native
    monkeypatch.setattr(_native, "_lib", None)
    monkeypatch.setattr(_native, "LIBDIR", tmp_path)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _native.lib()
