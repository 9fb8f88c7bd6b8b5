"""The C-ABI library builds, loads, and exports every entry point the public
header declares (no compute calls: these run without a GPU)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = []
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(vlr_[a-z0-9_]+)\s*\(", text):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "vlr_advect_level_set" in names and "vlr_rebuild_narrow_band" in names
    assert len(names) >= 10


def test_library_exports_every_declared_symbol():
    from sharc.volrus_b200 import _lib
    lib = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_header():
    from sharc.volrus_b200 import _lib
    missing = [n for n in declared_functions() if n not in _lib.SIGNATURES]
    assert not missing, f"no ctypes signature for: {missing}"


def test_no_cpu_fallback_without_library(tmp_path, monkeypatch):
    from sharc.volrus_b200 import _lib
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "missing.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load()


def test_oracle_library_loads(oracle):
    assert oracle.load() is not None
