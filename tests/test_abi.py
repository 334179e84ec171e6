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


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_box_with_end_before_start_is_an_argument_error(axis):
    """A box inside the array whose end lies before its start is refused before any launch
    (fills, norms and the no-allocation norm): negative extents would otherwise walk rows past
    the box."""
    lib = _lib.load()
    lay = _lib.Layout(16, 16, 16, 4, 11, 4, 11, 4, 11, 3, 4)
    ends = [[4, 11], [4, 11], [4, 11]]
    ends[axis] = [9, 6]
    box = _lib.Box(ends[0][0], ends[0][1], ends[1][0], ends[1][1], ends[2][0], ends[2][1])
    u = _lib.Field(1, _lib.B200_F32, 1.0)         # never dereferenced: the box check comes first
    rc = lib.b200_fill_const(ctypes.byref(lay), u, ctypes.byref(box), 1.0, None)
    assert rc == -1 and "end before its start" in _lib.last_error()
    out = ctypes.c_double()
    rc = lib.b200_sum_abs(ctypes.byref(lay), u, ctypes.byref(box), ctypes.byref(out), None)
    assert rc == -1 and "end before its start" in _lib.last_error()
    tab = (ctypes.c_double * 16)()
    rc = lib.b200_l1_sums_separable_noalloc(ctypes.byref(lay), u, ctypes.byref(box), tab, tab, tab,
                                            1.0, _lib.B200_F32, ctypes.byref(out),
                                            ctypes.byref(out), None)
    assert rc == -1 and "end before its start" in _lib.last_error()


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(_lib.B200Error):
        _lib.load()


def test_pressure_refuses_grids_of_another_geometry():
    """A coef grid laid out for another storage type (here FP32 padding against FP16
    wavefields, a different n1) is refused on the host before any library call: the kernels
    read every grid with the wavefield's layout, so its array would be read past its end."""
    from hpcscan_b200 import layout as L
    from hpcscan_b200.grid import Grid, RTN_CODE_KO
    lay16 = L.b200_layout(3, 64, 40, 30, order=8, prec="f16")
    lay32 = L.b200_layout(3, 64, 40, 30, order=8, prec="f32")
    assert lay16.n1 != lay32.n1
    prn, prc, coef = Grid(lay16), Grid(lay16), Grid(lay32)     # no device arrays: never reached
    assert prn.computePressureWithFD(prc, coef, 8) == RTN_CODE_KO
    assert prn.propagateStep(prc, coef, 8) == RTN_CODE_KO
    assert prn.updatePressure(L.INNER_POINTS, prc, coef, prc) == RTN_CODE_KO
