"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:int|const char\*)\s+(sgb_\w+)\s*\(", src, flags=re.M)
    return names


def test_header_declares_entry_points():
    names = _declared()
    assert "sgb_create" in names and "sgb_flush" in names and "sgb_apply_stencil" in names
    assert len(names) == len(set(names))


def test_library_exports_every_declared_symbol():
    from openfpm_data_b200 import _lib, build
    build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from openfpm_data_b200 import _lib
    assert set(_declared()) == set(_lib.SIGNATURES)


def test_status_strings_without_gpu():
    from openfpm_data_b200 import _lib
    lib = _lib.load()
    assert lib.sgb_status_string(0) == b"ok"
    assert b"outside" in lib.sgb_status_string(_lib.ERANGE)
    assert lib.sgb_version() >= 10000


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from openfpm_data_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(ImportError, match="no fallback"):
        _lib.load()
