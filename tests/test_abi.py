"""CPU checks of the C-ABI boundary: the library loads, exports every symbol the
header declares, and reports errors as status codes (no GPU needed)."""
import ctypes
import os
import re

import pytest

from hpcscan_b200 import _lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "hpcscan_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(b200_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(lib, s), s
    # and the ctypes prototypes cover exactly the declared entry points
    assert sorted(_lib.SIGNATURES) == syms


def test_errors_are_status_codes_not_exits():
    lib = _lib.load()
    # NULL layout: argument error reported through the status and last_error
    rc = lib.b200_fill_const(None, _lib.Field(None, 0, 1.0), None, 0.0, None)
    assert rc == -1
    assert "layout" in _lib.last_error()
    lay = _lib.Layout(10, 10, 10, 2, 7, 2, 7, 2, 7, 3, 2)
    rc = lib.b200_fd_d2(ctypes.byref(lay), 4, 4, _lib.Field(None, 0, 1.0),
                        _lib.Field(None, 0, 1.0), 1.0, 1.0, 1.0, None)
    assert rc == -1 and "axis" in _lib.last_error()
    rc = lib.b200_laplacian(ctypes.byref(lay), 5, _lib.Field(1, 0, 1.0), _lib.Field(2, 0, 1.0),
                            1.0, 1.0, 1.0, None)
    assert rc == -1 and "order" in _lib.last_error()
    bad = _lib.Layout(10, 10, 10, 1, 7, 2, 7, 2, 7, 3, 2)    # halo does not fit before s1
    rc = lib.b200_laplacian(ctypes.byref(bad), 4, _lib.Field(1, 0, 1.0), _lib.Field(2, 0, 1.0),
                            1.0, 1.0, 1.0, None)
    assert rc == -1 and "axis 1" in _lib.last_error()


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(_lib.B200Error):
        _lib.load()
