"""Grid index layout of hpcscan, restated for the host side.

A grid is one flat array with i1 fastest, idx = i1 + i2*n1 + i3*n1*n2, and
along each axis the regions (src/grid.cpp:15-38)

    [Offset][Halo1][Layer1][Inner][Layer2][Halo2][Pad]

Grid::initializeGrid (src/grid.cpp:252-583), padGridn1..3 (:839-976) and
offsetGridn1..3 (:979-1076) fix those regions for one MPI rank; this module
reproduces them for a single rank with no absorbing layer (nlayer = 0, the
reference default), which is the configuration every test case of the hot
path uses.

Two layout policies are provided:

* ``reference_layout``: exactly what the reference Grid builds, so that grids
  written by the reference (-writeGrid) can be read back;
* ``b200_layout``: the layout Grid_B200 uses on the device. Grid lets a test
  mode choose its own padding (the protected virtual hook padGridn1,
  src/grid.h:327-335). B200 keeps the reference's offsets, so the inner points
  sit at the same indices and get bit-identical coordinates (the origin is
  derived from the inner start, src/grid.cpp:417 and :1924-1957), and pads n1
  so that the row pitch is a multiple of 32 bytes: tensor-memory-accelerator
  (TMA) tile loads need 16-byte strides, and the z-marching kernel tiles n1
  from a 16-byte aligned index.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import Optional, Tuple

import numpy as np

from .fdm import check_order, halo_width

# src/constant.h:12 and src/config.cpp:35-37 (DEFAULT_D1..3 = PI / 30)
PI = 3.1415926535897
DEFAULT_D = PI / 30

ELEM_SIZE = {"f32": 4, "f64": 8, "f16": 2, "bf16": 2}
NP_DTYPE = {"f32": np.float32, "f64": np.float64, "f16": np.float16}

# Point types (src/type_def.h:96-98)
INNER_POINTS, ALL_POINTS, MIDDLE_POINT = 0, 1, 2
I1HALO1, I1HALO2, I2HALO1, I2HALO2, I3HALO1, I3HALO2 = 3, 4, 5, 6, 7, 8
I1INNERHALO1, I1INNERHALO2, I2INNERHALO1, I2INNERHALO2, I3INNERHALO1, I3INNERHALO2 = range(9, 15)


@dataclass(frozen=True)
class Axis:
    """Index regions along one axis (inclusive bounds, as the reference keeps them)."""
    n: int            # total points on this axis
    offset: int       # points before Halo1
    halo1_start: int
    inner_start: int
    inner_end: int
    halo2_end: int


@dataclass(frozen=True)
class GridLayout:
    dim: int
    order: int
    prec: str                       # storage type: f32, f64, f16, bf16
    a1: Axis
    a2: Axis
    a3: Axis
    n_inner: Tuple[int, int, int]   # global inner sizes (Config n1, n2, n3)

    # ---- array shape -------------------------------------------------------------------------
    @property
    def halo(self) -> int:
        return halo_width(self.order)

    @property
    def n1(self) -> int:
        return self.a1.n

    @property
    def n2(self) -> int:
        return self.a2.n

    @property
    def n3(self) -> int:
        return self.a3.n

    @property
    def npoint(self) -> int:
        return self.n1 * self.n2 * self.n3

    @property
    def elem_size(self) -> int:
        return ELEM_SIZE[self.prec]

    @property
    def nbytes(self) -> int:
        return self.npoint * self.elem_size

    @property
    def shape3(self) -> Tuple[int, int, int]:
        """numpy shape (n3, n2, n1) of the flat array (C order, i1 fastest)."""
        return (self.n3, self.n2, self.n1)

    @property
    def inner_points(self) -> int:
        return self.n_inner[0] * (self.n_inner[1] if self.dim >= 2 else 1) * (
            self.n_inner[2] if self.dim >= 3 else 1)

    # ---- boxes (Grid::getGridIndex, src/grid.cpp:2682-2843) -------------------------------------
    def box(self, point_type: int) -> Tuple[int, int, int, int, int, int]:
        a1, a2, a3 = self.a1, self.a2, self.a3
        h = self.halo
        inner = (a1.inner_start, a1.inner_end, a2.inner_start, a2.inner_end, a3.inner_start,
                 a3.inner_end)
        if point_type == INNER_POINTS:
            return inner
        if point_type == ALL_POINTS:
            return (a1.halo1_start, a1.halo2_end, a2.halo1_start, a2.halo2_end, a3.halo1_start,
                    a3.halo2_end)
        if point_type == MIDDLE_POINT:
            return (self.n1 // 2, self.n1 // 2, self.n2 // 2, self.n2 // 2, self.n3 // 2,
                    self.n3 // 2)
        s1, e1, s2, e2, s3, e3 = inner
        if point_type == I1HALO1:
            return (a1.halo1_start, s1 - 1, s2, e2, s3, e3)
        if point_type == I1HALO2:
            return (e1 + 1, a1.halo2_end, s2, e2, s3, e3)
        if point_type == I2HALO1:
            return (s1, e1, a2.halo1_start, s2 - 1, s3, e3)
        if point_type == I2HALO2:
            return (s1, e1, e2 + 1, a2.halo2_end, s3, e3)
        if point_type == I3HALO1:
            return (s1, e1, s2, e2, a3.halo1_start, s3 - 1)
        if point_type == I3HALO2:
            return (s1, e1, s2, e2, e3 + 1, a3.halo2_end)
        if point_type == I1INNERHALO1:
            return (s1, s1 + h, s2, e2, s3, e3)
        if point_type == I1INNERHALO2:
            return (e1 - h, e1, s2, e2, s3, e3)
        if point_type == I2INNERHALO1:
            return (s1, e1, s2, s2 + h, s3, e3)
        if point_type == I2INNERHALO2:
            return (s1, e1, e2 - h, e2, s3, e3)
        if point_type == I3INNERHALO1:
            return (s1, e1, s2, e2, s3, s3 + h)
        if point_type == I3INNERHALO2:
            return (s1, e1, s2, e2, e3 - h, e3)
        raise ValueError(f"invalid point type {point_type}")

    # ---- numpy helpers ------------------------------------------------------------------------
    def view3(self, flat: np.ndarray) -> np.ndarray:
        return flat.reshape(self.shape3)

    def box_slices(self, point_type: int):
        b = self.box(point_type)
        return (slice(b[4], b[5] + 1), slice(b[2], b[3] + 1), slice(b[0], b[1] + 1))

    def inner(self, flat: np.ndarray) -> np.ndarray:
        """Inner points as a (N3, N2, N1) array (copy-free view)."""
        return self.view3(flat)[self.box_slices(INNER_POINTS)]

    def c_struct_fields(self):
        """(n1, n2, n3, s1, e1, s2, e2, s3, e3, dim, halo) for the C ABI layout struct."""
        return (self.n1, self.n2, self.n3, self.a1.inner_start, self.a1.inner_end,
                self.a2.inner_start, self.a2.inner_end, self.a3.inner_start, self.a3.inner_end,
                self.dim, self.halo)


def _axis(n_inner: int, halo: int, offset: int, pad_mode: str = "none", pad_arg: int = 0,
          odd_pad: bool = False) -> Axis:
    """One axis of Grid::initializeGrid with nlayer = 0 (src/grid.cpp:387-420)."""
    halo1_start = offset
    inner_start = halo1_start + halo
    inner_end = inner_start + n_inner - 1
    halo2_start = inner_end + 1
    halo2_end = halo2_start + halo - 1
    if pad_mode == "auto":               # src/grid.cpp:843-862 (n1 only)
        n_tot = halo2_end + 1
        pad_end = halo2_end + 1 if (n_tot % 2 and odd_pad) else halo2_end
    elif pad_mode == "add":              # :864-868
        pad_end = halo2_end + pad_arg
    elif pad_mode == "mul":              # :869-883
        pad_start = halo2_end + 1
        n_tmp = (pad_start + 1) // pad_arg
        if pad_arg * n_tmp < pad_start:
            pad_end = (n_tmp + 1) * pad_arg - 1
        else:
            pad_end = n_tmp * pad_arg - 1
    else:                                # :884-888
        pad_end = halo2_end
    return Axis(n=pad_end + 1, offset=offset, halo1_start=halo1_start, inner_start=inner_start,
                inner_end=inner_end, halo2_end=halo2_end)


_FLAT_AXIS = Axis(n=1, offset=0, halo1_start=0, inner_start=0, inner_end=0, halo2_end=0)


def reference_layout(dim: int, n1: int, n2: int = 1, n3: int = 1, order: int = 8,
                     prec: str = "f32", auto_pad: bool = False,
                     add_pad: Tuple[Optional[int], ...] = (None, None, None),
                     mul_pad: Tuple[Optional[int], ...] = (None, None, None),
                     offset: Tuple[Optional[int], ...] = (None, None, None)) -> GridLayout:
    """The layout the reference Grid builds for one rank (src/grid.cpp:252-583, 839-1076)."""
    check_order(order)
    if dim not in (1, 2, 3):
        raise ValueError("dim must be 1, 2 or 3")
    h = halo_width(order)
    fp64 = prec == "f64"
    axes = []
    for a, n in enumerate((n1, n2, n3)):
        if a + 1 > dim:
            axes.append(_FLAT_AXIS)
            continue
        if offset[a] is not None:
            off = offset[a]
        elif a == 0 and h % 2 == 1 and not fp64:   # src/grid.cpp:986-999
            off = 1
        else:
            off = 0
        if auto_pad:
            mode, arg = ("auto", 0) if a == 0 else ("none", 0)
        elif add_pad[a] is not None:
            mode, arg = "add", add_pad[a]
        elif mul_pad[a] is not None:
            mode, arg = "mul", mul_pad[a]
        else:
            mode, arg = "none", 0
        axes.append(_axis(n, h, off, mode, arg, odd_pad=not fp64))
    return GridLayout(dim=dim, order=order, prec=prec, a1=axes[0], a2=axes[1], a3=axes[2],
                      n_inner=(n1, n2 if dim >= 2 else 1, n3 if dim >= 3 else 1))


def b200_layout(dim: int, n1: int, n2: int = 1, n3: int = 1, order: int = 8,
                prec: str = "f32") -> GridLayout:
    """The device layout of Grid_B200: the reference's offsets, n1 padded to a
    multiple of 32 bytes."""
    ref = reference_layout(dim, n1, n2, n3, order=order, prec=prec)
    a32 = 32 // ELEM_SIZE[prec]
    n1_tot = -(-(ref.a1.halo2_end + 1) // a32) * a32
    return replace(ref, a1=replace(ref.a1, n=n1_tot))


# ---- coordinates and separable fills ----------------------------------------------------------

@dataclass(frozen=True)
class Sampling:
    """Grid spacing and origin per axis (Grid::d1..d3, Orig1..3)."""
    d: Tuple[float, float, float]
    orig: Tuple[float, float, float]


def default_sampling(lay: GridLayout, d=(DEFAULT_D, DEFAULT_D, DEFAULT_D)) -> Sampling:
    """After initializeGrid: Orig = (0 - InnerStart) * d (src/grid.cpp:417, 471, 525)."""
    orig = []
    dd = []
    for a, ax in enumerate((lay.a1, lay.a2, lay.a3)):
        if a + 1 <= lay.dim:
            dd.append(d[a])
            orig.append((0 - ax.inner_start) * d[a])
        else:
            dd.append(0.0)
            orig.append(0.0)
    return Sampling(tuple(dd), tuple(orig))


def unit_sampling(lay: GridLayout) -> Sampling:
    """Grid::defineUnitGrid (src/grid.cpp:1924-1957): d = 1/(N-1); the new origin
    is computed in FP64 and stored through the storage type Myfloat."""
    prev = default_sampling(lay)
    store = np.float64 if lay.prec == "f64" else np.float32
    d = []
    orig = []
    for a in range(3):
        if a + 1 <= lay.dim:
            dn = 1.0 / (lay.n_inner[a] - 1)
            o = prev.orig[a] * dn / prev.d[a]
            d.append(dn)
            orig.append(float(store(o)))
        else:
            d.append(0.0)
            orig.append(0.0)
    return Sampling(tuple(d), tuple(orig))


FUNC_NONE, FUNC_SINE, FUNC_COSINE, FUNC_CONST, FUNC_LINEAR = 0, 1, 2, 3, 4


def fill_table(lay: GridLayout, samp: Sampling, axis: int, i_start: int, i_end: int,
               func: int, param: float) -> np.ndarray:
    """One FP64 1-D table of Grid::fill (src/grid.cpp:1665-1770):
    coord = Orig + i*d, value = sin(coord*param) etc.; 1.0 on axes beyond dim.
    math.sin is the C library sin the reference calls."""
    out = np.empty(i_end - i_start + 1, dtype=np.float64)
    for j, i in enumerate(range(i_start, i_end + 1)):
        coord = samp.orig[axis] + i * samp.d[axis]
        if axis + 1 > lay.dim:
            v = 1.0
        elif func == FUNC_SINE:
            v = math.sin(coord * param)
        elif func == FUNC_COSINE:
            v = math.cos(coord * param)
        elif func == FUNC_LINEAR:
            v = coord
        else:
            v = 1.0
        out[j] = v
    return out


def fill_tables(lay: GridLayout, samp: Sampling, point_type: int, funcs, params):
    b = lay.box(point_type)
    return tuple(fill_table(lay, samp, a, b[2 * a], b[2 * a + 1], funcs[a], params[a])
                 for a in range(3))


def inv_spacing(samp: Sampling, prec: str) -> Tuple[float, float, float]:
    """inv_d = ONE/d in the compute type Myfloat2, the FD_D1 operators' factor
    (src/grid.cpp:3414-3416). Axes beyond dim have d = 0 and give 0."""
    t = np.float64 if prec == "f64" else np.float32
    return tuple(0.0 if d == 0.0 else float(t(1.0 / d)) for d in samp.d)


def inv2_spacing(samp: Sampling, prec: str) -> Tuple[float, float, float]:
    """inv2_d = (ONE/d)^2 evaluated in the compute type Myfloat2 (src/grid.cpp:3252-3258).
    Axes beyond dim have d = 0 and are never used."""
    t = np.float64 if prec == "f64" else np.float32
    out = []
    for d in samp.d:
        if d == 0.0:
            out.append(0.0)
            continue
        inv = t(1.0 / d)        # ONE / d: FP64 division, result stored in Myfloat2
        out.append(float(inv * inv))
    return tuple(out)
