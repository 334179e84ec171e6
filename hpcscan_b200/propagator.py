"""Python mirror of the hpcscan acoustic propagator and of the Propa test case
for the B200 test mode.

Propagator_Ac2 / Propagator_Ac2SplitComp follow src/propagator_Ac2.cpp and
src/propagator_Ac2SplitComp.cpp of vetienne74/hpcscan (initialize(EIGEN_MODE),
computeWavefieldNextTimeStep, computePressureWithFD, getCFL, initializeGrid);
run_propa follows TestCase_Propa::run (src/testCase_Propa.cpp:31-262): the
time loop, the analytic check every snapInc steps on try 0, and
errTestCase = sum1 / sum2 with the reference's FP32 accumulators.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np
import torch

from . import _lib
from .grid import Grid, init_device, tuned_config
from .layout import ALL_POINTS, INNER_POINTS, GridLayout, b200_layout
from .propa_setup import EIGEN_FUNCS, EigenSetup, eigen_setup, init_times

PROPA_TYPE_AC2STANDARD = "Ac2Standard"
PROPA_TYPE_AC2SPLITCOMP = "Ac2SplitComp"


class Propagator_Ac2:
    """2nd-order acoustic leapfrog, constant density (src/propagator_Ac2.cpp:1-37)."""

    kernel_type = "Standard implementation"

    def __init__(self, layout: GridLayout, device: int = 0, coef_prec: Optional[str] = None,
                 wave_scale: float = 1.0):
        self.layout = layout
        self.device = device
        self.boundCondType = _lib.B200_BOUND_COND_ANTI_MIRROR
        self.fdOrder = layout.order
        self.coef_prec = coef_prec or layout.prec
        self.wave_scale = wave_scale
        self.setup: Optional[EigenSetup] = None
        self.coefGrid = self.prnGrid = self.prcGrid = None

    # ---- Propagator_Ac2::initialize(EIGEN_MODE) ----------------------------------------------------
    def initialize(self, ratio_cfl: float = 1.0, tmax=None, nt: int = 20, snap_inc: int = 1,
                   modes=(0.8, 0.9, 1.0), dt: float = 0.0) -> int:
        init_device(self.device)
        lay = self.layout
        self.setup = s = eigen_setup(lay, ratio_cfl=ratio_cfl, tmax=tmax, nt=nt, dt=dt,
                                     snap_inc=snap_inc, modes=modes)
        coef_lay = lay if self.coef_prec == lay.prec else GridLayout(
            dim=lay.dim, order=lay.order, prec=self.coef_prec, a1=lay.a1, a2=lay.a2, a3=lay.a3,
            n_inner=lay.n_inner)
        coef_scale = 1.0
        if self.coef_prec in ("f16", "bf16"):
            # power-of-two scale that brings v^2 dt^2 near 1 in 16-bit storage
            coef_scale = 2.0 ** int(np.floor(np.log2(s.coef)))
        self.coefGrid = Grid(coef_lay, s.samp, self.device, scale=coef_scale)
        self.prnGrid = Grid(lay, s.samp, self.device, scale=self.wave_scale)
        self.prcGrid = Grid(lay, s.samp, self.device, scale=self.wave_scale)
        for g in (self.coefGrid, self.prnGrid, self.prcGrid):
            g.initializeGrid()
        self.coefGrid.fill(INNER_POINTS, s.coef)
        t_prn, t_prc = init_times(s, lay.prec if lay.prec == "f64" else "f32")
        self.initializeGrid(self.prnGrid, t_prn)
        self.initializeGrid(self.prcGrid, t_prc)
        self.prepare()
        return 0

    def prepare(self) -> None:
        """Ready the step's kernels before the time loop (b200_prepare_stencil: the first-use
        tuning for this grid size, or one launch on scratch grids)."""
        lay = self.prnGrid.c_layout()
        _lib.call("b200_prepare_stencil", ctypes.byref(lay), self.fdOrder,
                  _lib.DTYPE_CODE[self.layout.prec], self.prepare_op,
                  _lib.DTYPE_CODE[self.coef_prec])

    prepare_op = _lib.OP_STEP

    def initializeGrid(self, grid: Grid, time_sec) -> int:
        """Eigen mode at time t on ALL_POINTS (src/propagator_Ac2.cpp:441-545)."""
        s = self.setup
        p = s.params(self.layout)
        grid.fill(ALL_POINTS, *EIGEN_FUNCS, p[0], p[1], p[2], s.amplitude(time_sec))
        return 0

    def getCFL(self) -> float:
        return self.setup.cfl

    # ---- time step -----------------------------------------------------------------------------
    def computeWavefieldNextTimeStep(self, prn: Grid, prc: Grid, stream=None) -> int:
        """halo exchange (none on one GPU) -> boundary condition -> FD kernel
        (src/propagator_Ac2.cpp:366-395), as one b200_propagate_step call: the library runs
        the boundary-condition kernel and the pressure kernel, or, where the tuner measured it
        faster for this grid, the pressure kernel with the boundary condition built inside its
        tiles. prn and the inner points of prc are bit-identical either way (prc's halo points,
        which no later read uses before the next boundary condition, are then left as they
        were)."""
        if not prn.sameSize(prc):
            return self.computePressureWithFD(prn, prc, stream=stream)
        return prn.propagateStep(prc, self.coefGrid, self.fdOrder, self.boundCondType,
                                 stream=stream)

    def step_config(self) -> dict:
        """The launch parameters the library uses for this propagator's grids: the pressure
        kernel's tile shape and planes per CTA, and whether the fused step was chosen
        (measured = False: untuned defaults)."""
        out = {}
        for name, op in (("pressure", _lib.OP_PRESSURE), ("step", _lib.OP_STEP)):
            out[name] = tuned_config(self.prnGrid, op)
        return out

    def computePressureWithFD(self, prn: Grid, prc: Grid, stream=None) -> int:
        return prn.computePressureWithFD(prc, self.coefGrid, self.fdOrder, stream=stream)


class Propagator_Ac2SplitComp(Propagator_Ac2):
    """Laplacian then updatePressure (src/propagator_Ac2SplitComp.cpp:72-85)."""

    kernel_type = "With Laplacian operator"
    prepare_op = _lib.OP_LAPLACIAN

    def initialize(self, **kw) -> int:
        rc = super().initialize(**kw)
        self.laplaGrid = Grid(self.layout, self.setup.samp, self.device, scale=self.wave_scale)
        self.laplaGrid.initializeGrid()
        return rc

    def computeWavefieldNextTimeStep(self, prn: Grid, prc: Grid, stream=None) -> int:
        """boundary condition, then the Laplacian and the update (two operators, as the
        reference's SplitComp propagator runs them)."""
        prc.applyBoundaryCondition(self.boundCondType, stream=stream)
        return self.computePressureWithFD(prn, prc, stream=stream)

    def computePressureWithFD(self, prn: Grid, prc: Grid, stream=None) -> int:
        prc.FD_LAPLACIAN(INNER_POINTS, self.laplaGrid, self.fdOrder, stream=stream)
        return prn.updatePressure(INNER_POINTS, prc, self.coefGrid, self.laplaGrid, stream=stream)


def create_propagator(name: str, layout: GridLayout, **kw) -> Propagator_Ac2:
    """Propagator_Factory::create (src/propagator_Factory.cpp:19-40)."""
    if name == PROPA_TYPE_AC2STANDARD:
        return Propagator_Ac2(layout, **kw)
    if name == PROPA_TYPE_AC2SPLITCOMP:
        return Propagator_Ac2SplitComp(layout, **kw)
    raise ValueError(f"IN Propagator_Factory::create, invalid propagator {name}")


@dataclass
class PropaResult:
    nt: int
    dt: float
    err_test_case: float
    n_check: int
    time_total_s: float
    gpoint_per_s: float
    checks: list = field(default_factory=list)


def run_propa(layout: GridLayout, propagator: str = PROPA_TYPE_AC2STANDARD, ratio_cfl=1.0,
              tmax=None, nt=20, snap_inc=1, modes=(0.8, 0.9, 1.0), device: int = 0,
              on_check: Optional[Callable] = None, fused_check: bool = True,
              coef_prec: Optional[str] = None, wave_scale: float = 1.0) -> PropaResult:
    """TestCase_Propa::run for one try (src/testCase_Propa.cpp:111-181).

    With fused_check, the analytic reference is not materialised: its sums come
    from b200_l1_sums_separable (same values as fill + getSumAbsDiff + getSumAbs
    up to FP64 summation order)."""
    propa = create_propagator(propagator, layout, device=device, coef_prec=coef_prec,
                              wave_scale=wave_scale)
    propa.initialize(ratio_cfl=ratio_cfl, tmax=tmax, nt=nt, snap_inc=snap_inc, modes=modes)
    s = propa.setup
    prn, prc = propa.prnGrid, propa.prcGrid
    ref = None
    if not fused_check:
        ref = Grid(layout, s.samp, device)
        ref.initializeGrid()
    sum1 = np.float32(0.0)
    sum2 = np.float32(0.0)
    n_check = 0
    checks = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for it in range(s.nt):
        propa.computeWavefieldNextTimeStep(prn, prc)
        if it % s.snap_inc == 0:
            tsec = s.time_of_step(it, layout.prec if layout.prec == "f64" else "f32")
            amp = s.amplitude(tsec)
            if fused_check:
                s1, s2 = l1_sums_eigen(prn, propa, amp)
            else:
                propa.initializeGrid(ref, tsec)
                s1 = prn.getSumAbsDiff(INNER_POINTS, ref)
                s2 = ref.getSumAbs(INNER_POINTS)
            # Myfloat returned, accumulated in Myfloat32 (src/testCase_Propa.cpp:148-149)
            store = np.float64 if layout.prec == "f64" else np.float32
            sum1 = np.float32(sum1 + np.float32(store(s1)))
            sum2 = np.float32(sum2 + np.float32(store(s2)))
            n_check += 1
            checks.append((it, float(s1), float(s2)))
            if on_check is not None:
                on_check(it, prn, ref)
        prn, prc = prc, prn
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    propa.prnGrid, propa.prcGrid = prn, prc
    err = float(np.float32(sum1 / sum2)) if sum2 != 0 else float("nan")
    return PropaResult(nt=s.nt, dt=s.dt, err_test_case=err, n_check=n_check, time_total_s=t,
                       gpoint_per_s=s.nt * layout.inner_points / t / 1e9, checks=checks)


def l1_sums_eigen(prn: Grid, propa: Propagator_Ac2, amp: float):
    """sum|prn - ref| and sum|ref| over INNER points for the eigen-mode reference at
    amplitude `amp`, without writing the reference grid."""
    import ctypes
    from .layout import fill_tables
    lay = prn.layout
    # the 1-D tables depend on the grid only (the amplitude is a factor): built once per grid
    key = (id(propa.setup), lay.n1, lay.n2, lay.n3, lay.prec)
    cache = propa.__dict__.setdefault("_eigen_tables", {})
    tabs = cache.get(key)
    if tabs is None:
        tabs = fill_tables(lay, propa.setup.samp, INNER_POINTS, EIGEN_FUNCS, propa.setup.params(lay))
        cache[key] = tabs
    s1, s2 = ctypes.c_double(), ctypes.c_double()
    cl, box = prn.c_layout(), prn.c_box(INNER_POINTS)
    ref_dtype = _lib.DTYPE_CODE["f64" if lay.prec == "f64" else "f32"]
    _lib.call("b200_l1_sums_separable", ctypes.byref(cl), prn.c_field(), ctypes.byref(box),
              *[t.ctypes.data_as(ctypes.c_void_p) for t in tabs], float(amp), ref_dtype,
              ctypes.byref(s1), ctypes.byref(s2), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return s1.value, s2.value
