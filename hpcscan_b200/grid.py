"""Python mirror of the hpcscan Grid interface for the B200 test mode.

Each method keeps the name, argument meaning and error behaviour of the
reference's Grid virtual it stands for (src/grid.h:50-208 of vetienne74/hpcscan)
and calls one entry point of the C ABI (include/hpcscan_b200.h). Device memory
comes from torch's CUDA allocator; torch is plumbing only, every operation on
the data is a hpcscan_b200 kernel.

Error behaviour, as in the reference: a size mismatch prints an error and
returns RTN_CODE_KO (operators) or -1.0 (norms). A failing CUDA call raises
B200Error (the reference's CUDA modes exit the process instead).
"""
from __future__ import annotations

import ctypes
import sys
from typing import Optional

import numpy as np
import torch

from . import _lib
from .fdm import check_order
from .layout import (ALL_POINTS, INNER_POINTS, GridLayout, Sampling, default_sampling,
                     fill_tables, inv2_spacing, inv_spacing, unit_sampling)

RTN_CODE_OK, RTN_CODE_KO = 0, -1
TORCH_DTYPE = {"f32": torch.float32, "f64": torch.float64, "f16": torch.float16,
               "bf16": torch.bfloat16}
NP_DTYPE = {"f32": np.float32, "f64": np.float64, "f16": np.float16}
MAX_ERR_FLOAT = {"f32": 1.0e-5, "f64": 1.0e-11, "f16": 1.0e-3, "bf16": 1.0e-3}


def print_error(msg: str) -> None:
    print(f"ERROR: {msg}", file=sys.stderr)


_initialised = set()


def init_device(device: int = 0) -> None:
    if device not in _initialised:
        torch.cuda.set_device(device)
        _lib.call("b200_init", device)
        _initialised.add(device)


def _stream_ptr(stream: Optional[torch.cuda.Stream]) -> ctypes.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def tuned_config(grid: "Grid", op: int) -> dict:
    """Launch parameters the library uses for `op` on grids of this layout (b200_get_tuned_config):
    tile shape, planes per CTA (0 = heuristic), fused step (op OP_STEP), measured or default."""
    sh, ch, fu, me = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lay = grid.c_layout()
    _lib.call("b200_get_tuned_config", ctypes.byref(lay), grid.layout.order,
              _lib.DTYPE_CODE[grid.layout.prec], op, ctypes.byref(sh), ctypes.byref(ch),
              ctypes.byref(fu), ctypes.byref(me))
    return {"shape": sh.value, "nz_chunk": ch.value, "fused": bool(fu.value),
            "measured": bool(me.value)}


class Grid:
    """A grid of the B200 test mode: layout + device array (+ spacing/origin)."""

    def __init__(self, layout: GridLayout, sampling: Optional[Sampling] = None,
                 device: int = 0, scale: float = 1.0):
        self.layout = layout
        self.sampling = sampling if sampling is not None else default_sampling(layout)
        self.device = device
        self.scale = float(scale)
        self.data: Optional[torch.Tensor] = None
        self.grid_mode = "B200"

    # ---- Grid::initializeGrid / defineUnitGrid ---------------------------------------------------
    def initializeGrid(self) -> int:
        init_device(self.device)
        if self.data is not None:
            print_error(" In Grid::initializeGrid, grid_3d != NULL")
            return RTN_CODE_OK
        self.data = torch.zeros(self.layout.npoint, dtype=TORCH_DTYPE[self.layout.prec],
                                device=f"cuda:{self.device}")
        return RTN_CODE_OK

    def defineUnitGrid(self) -> None:
        self.sampling = unit_sampling(self.layout)

    # ---- C ABI plumbing ---------------------------------------------------------------------------
    @property
    def dim(self) -> int:
        return self.layout.dim

    @property
    def haloWidth(self) -> int:
        return self.layout.halo

    @property
    def npoint(self) -> int:
        return self.layout.npoint

    def c_layout(self) -> _lib.Layout:
        return _lib.Layout(*self.layout.c_struct_fields())

    def c_field(self) -> _lib.Field:
        return _lib.Field(ctypes.c_void_p(self.data.data_ptr()), _lib.DTYPE_CODE[self.layout.prec],
                          self.scale)

    def c_box(self, point_type: int) -> _lib.Box:
        return _lib.Box(*self.layout.box(point_type))

    def sameSize(self, other: "Grid") -> bool:
        a, b = self.layout, other.layout
        return (a.npoint, a.n1, a.n2, a.n3) == (b.npoint, b.n1, b.n2, b.n3)

    def inv2(self):
        return inv2_spacing(self.sampling, "f64" if self.layout.prec == "f64" else "f32")

    def inv(self):
        return inv_spacing(self.sampling, "f64" if self.layout.prec == "f64" else "f32")

    # ---- fills -----------------------------------------------------------------------------------
    def fill(self, point_type: int, *args, stream=None) -> None:
        """fill(pointType, val) or fill(pointType, f1, f2, f3, p1, p2, p3, amp)."""
        lay = self.c_layout()
        box = self.c_box(point_type)
        if len(args) == 1:
            _lib.call("b200_fill_const", ctypes.byref(lay), self.c_field(), ctypes.byref(box),
                      float(args[0]), _stream_ptr(stream))
            return
        f1, f2, f3, p1, p2, p3, amp = args
        tabs = fill_tables(self.layout, self.sampling, point_type, (f1, f2, f3), (p1, p2, p3))
        ptrs = [t.ctypes.data_as(ctypes.c_void_p) for t in tabs]
        _lib.call("b200_fill_separable", ctypes.byref(lay), self.c_field(), ctypes.byref(box),
                  *ptrs, float(amp), _stream_ptr(stream))

    # ---- whole-array operations (Grid::fillArray .. addUpdateArray, src/grid.cpp:1828-1918) ------
    def _array_op(self, op: int, a: Optional["Grid"], b: Optional["Grid"], val: float,
                  stream=None) -> None:
        none = _lib.Field(None, self.c_field().dtype, 1.0)
        _lib.call("b200_array_op", op, self.layout.npoint, self.c_field(),
                  a.c_field() if a is not None else none, b.c_field() if b is not None else none,
                  float(val), _stream_ptr(stream))

    def fillArray(self, val: float, stream=None) -> None:
        self._array_op(_lib.B200_ARRAY_FILL, None, None, val, stream)

    def copyArray(self, gridIn: "Grid", stream=None) -> None:
        self._array_op(_lib.B200_ARRAY_COPY, gridIn, None, 0.0, stream)

    def addArray(self, gridIn1: "Grid", gridIn2: "Grid", stream=None) -> None:
        self._array_op(_lib.B200_ARRAY_ADD, gridIn1, gridIn2, 0.0, stream)

    def multiplyArray(self, gridIn1: "Grid", gridIn2: "Grid", stream=None) -> None:
        self._array_op(_lib.B200_ARRAY_MUL, gridIn1, gridIn2, 0.0, stream)

    def addUpdateArray(self, gridIn: "Grid", stream=None) -> None:
        self._array_op(_lib.B200_ARRAY_ADD_UPDATE, gridIn, None, 0.0, stream)

    # ---- FD operators (`self` is the input, W the output; INNER points) --------------------------
    def _fd(self, axis: int, W: "Grid", order: int, name: str, stream=None) -> int:
        if not self.sameSize(W):
            print_error(f"Grid::{name}, grids have not same size")
            return RTN_CODE_KO
        check_order(order)
        i1, i2, i3 = self.inv2()
        lay = self.c_layout()
        if axis == 0:
            _lib.call("b200_laplacian", ctypes.byref(lay), order, self.c_field(), W.c_field(),
                      i1, i2, i3, _stream_ptr(stream))
        else:
            _lib.call("b200_fd_d2", ctypes.byref(lay), axis, order, self.c_field(), W.c_field(),
                      i1, i2, i3, _stream_ptr(stream))
        return RTN_CODE_OK

    def FD_D2_N1(self, pType: int, W: "Grid", fdOrder: int, stream=None) -> int:
        return self._fd(1, W, fdOrder, "FD_D2_N1", stream)

    def FD_D2_N2(self, pType: int, W: "Grid", fdOrder: int, stream=None) -> int:
        return self._fd(2, W, fdOrder, "FD_D2_N2", stream)

    def FD_D2_N3(self, pType: int, W: "Grid", fdOrder: int, stream=None) -> int:
        return self._fd(3, W, fdOrder, "FD_D2_N3", stream)

    def _fd_d1(self, axis: int, W: "Grid", order: int, stream=None) -> int:
        if not self.sameSize(W):
            print_error(f"Grid::FD_D1_N{axis}, grids have not same size")
            return RTN_CODE_KO
        check_order(order)
        i1, i2, i3 = self.inv()
        lay = self.c_layout()
        _lib.call("b200_fd_d1", ctypes.byref(lay), axis, order, self.c_field(), W.c_field(),
                  i1, i2, i3, _stream_ptr(stream))
        return RTN_CODE_OK

    def FD_D1_N1(self, pType: int, W: "Grid", fdOrder: int, stream=None) -> int:
        """Staggered first derivative at i1 - 1/2 (src/grid.cpp:3401)."""
        return self._fd_d1(1, W, fdOrder, stream)

    def FD_D1_N2(self, pType: int, W: "Grid", fdOrder: int, stream=None) -> int:
        return self._fd_d1(2, W, fdOrder, stream)

    def FD_D1_N3(self, pType: int, W: "Grid", fdOrder: int, stream=None) -> int:
        return self._fd_d1(3, W, fdOrder, stream)

    def FD_LAPLACIAN(self, pType: int, W: "Grid", fdOrder: int, stream=None) -> int:
        return self._fd(0, W, fdOrder, "FD_LAPLACIAN", stream)

    def _same_geometry(self, caller: str, *grids: "Grid") -> bool:
        """Every grid a kernel reads with this grid's layout must have its array geometry (the
        library indexes them all with one layout); a grid of another geometry is refused here,
        before any launch (its array would be read past its end)."""
        for g in grids:
            if not self.sameSize(g):
                print_error(f"In Grid::{caller}, grids have not same size")
                return False
        return True

    def updatePressure(self, pType: int, prc: "Grid", coef: "Grid", lapla: "Grid",
                       stream=None) -> int:
        if not self._same_geometry("updatePressure", prc, coef, lapla):
            return RTN_CODE_KO
        lay = self.c_layout()
        _lib.call("b200_update_pressure", ctypes.byref(lay), self.c_field(), prc.c_field(),
                  coef.c_field(), lapla.c_field(), _stream_ptr(stream))
        return RTN_CODE_OK

    def computePressureWithFD(self, prc: "Grid", coef: "Grid", fdOrder: int, stream=None) -> int:
        if not self._same_geometry("computePressureWithFD", prc, coef):
            return RTN_CODE_KO
        i1, i2, i3 = self.inv2()
        lay = self.c_layout()
        _lib.call("b200_compute_pressure", ctypes.byref(lay), fdOrder, self.c_field(),
                  prc.c_field(), coef.c_field(), i1, i2, i3, _stream_ptr(stream))
        return RTN_CODE_OK

    def propagateStep(self, prc: "Grid", coef: "Grid", fdOrder: int,
                      boundCondType: int = _lib.B200_BOUND_COND_ANTI_MIRROR, stream=None) -> int:
        """prc.applyBoundaryCondition(boundCondType) then self.computePressureWithFD(prc, coef)
        in one library call (b200_propagate_step)."""
        if not self._same_geometry("computePressureWithFD", prc, coef):
            return RTN_CODE_KO
        i1, i2, i3 = self.inv2()
        lay = self.c_layout()
        _lib.call("b200_propagate_step", ctypes.byref(lay), fdOrder, self.c_field(), prc.c_field(),
                  coef.c_field(), i1, i2, i3, boundCondType, _stream_ptr(stream))
        return RTN_CODE_OK

    def applyBoundaryCondition(self, boundCondType: int = _lib.B200_BOUND_COND_ANTI_MIRROR,
                               stream=None) -> int:
        if boundCondType not in (_lib.B200_NO_BOUND_COND, _lib.B200_BOUND_COND_ANTI_MIRROR):
            print_error(f"IN Grid::applyBoundaryCondition, invalid boundCondType {boundCondType}")
            return RTN_CODE_KO
        lay = self.c_layout()
        _lib.call("b200_apply_boundary", ctypes.byref(lay), self.c_field(), boundCondType, 0x3F,
                  _stream_ptr(stream))
        return RTN_CODE_OK

    # ---- norms -----------------------------------------------------------------------------------
    def getSumAbs(self, pType: int, stream=None) -> float:
        out = ctypes.c_double()
        lay, box = self.c_layout(), self.c_box(pType)
        _lib.call("b200_sum_abs", ctypes.byref(lay), self.c_field(), ctypes.byref(box),
                  ctypes.byref(out), _stream_ptr(stream))
        return out.value

    def getSumAbsDiff(self, pType: int, other: "Grid", stream=None) -> float:
        if not self.sameSize(other):
            print_error("Grid::getSumAbsDiff, grids have different size")
            return -1.0
        out = ctypes.c_double()
        lay, box = self.c_layout(), self.c_box(pType)
        _lib.call("b200_sum_abs_diff", ctypes.byref(lay), self.c_field(), other.c_field(),
                  ctypes.byref(box), ctypes.byref(out), _stream_ptr(stream))
        return out.value

    def l1Sums(self, pType: int, other: "Grid", stream=None):
        s1, s2 = ctypes.c_double(), ctypes.c_double()
        lay, box = self.c_layout(), self.c_box(pType)
        _lib.call("b200_l1_sums", ctypes.byref(lay), self.c_field(), other.c_field(),
                  ctypes.byref(box), ctypes.byref(s1), ctypes.byref(s2), _stream_ptr(stream))
        return s1.value, s2.value

    def L1Err(self, pType: int, other: "Grid", stream=None) -> float:
        if not self.sameSize(other):
            print_error("Grid::L1Err, grids have different size")
            return -1.0
        s1, s2 = self.l1Sums(pType, other, stream)
        if s2 < MAX_ERR_FLOAT[self.layout.prec]:
            s2 = 1.0 * self.npoint
        return s1 / s2

    def maxErr(self, pType: int, other: "Grid", stream=None) -> float:
        if not self.sameSize(other):
            print_error("Grid::maxErr, grids have different size")
            return -1.0
        out = ctypes.c_double()
        lay, box = self.c_layout(), self.c_box(pType)
        _lib.call("b200_max_err", ctypes.byref(lay), self.c_field(), other.c_field(),
                  ctypes.byref(box), MAX_ERR_FLOAT[self.layout.prec], ctypes.byref(out),
                  _stream_ptr(stream))
        return out.value

    def getMinMax(self, pType: int, stream=None):
        mn, mx = ctypes.c_double(), ctypes.c_double()
        lay, box = self.c_layout(), self.c_box(pType)
        _lib.call("b200_min_max", ctypes.byref(lay), self.c_field(), ctypes.byref(box),
                  ctypes.byref(mn), ctypes.byref(mx), _stream_ptr(stream))
        return mn.value, mx.value

    def getMin(self, pType: int) -> float:
        return self.getMinMax(pType)[0]

    def getMax(self, pType: int) -> float:
        return self.getMinMax(pType)[1]

    # ---- host transfers (Grid::write / read equivalents) ------------------------------------------
    def to_numpy(self) -> np.ndarray:
        """The whole array on the host, physical values (stored value * scale), as float32/64."""
        t = self.data.detach()
        if self.layout.prec in ("f16", "bf16"):
            t = t.float()
        a = t.cpu().numpy()
        return a * self.scale if self.scale != 1.0 else a

    def from_numpy(self, a: np.ndarray) -> None:
        src = torch.from_numpy(np.ascontiguousarray(a).reshape(-1) / (self.scale if self.scale != 1.0 else 1))
        self.data.copy_(src.to(TORCH_DTYPE[self.layout.prec]))
