"""Host-side set-up of the acoustic propagator (time step, number of steps,
physical coefficient, eigen-mode initial condition), restated from
Propagator_Ac2::initialize / getCFL / initializeGrid
(src/propagator_Ac2.cpp:84-303, 410-545) of vetienne74/hpcscan.

The reference evaluates these in its storage type Myfloat (FP32 or FP64
build); every rounding step is reproduced here so that dt, nt and the initial
fields are bit-identical to the reference's for the same flags.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np

from . import fdm
from .layout import FUNC_SINE, PI, GridLayout, Sampling, unit_sampling


def _T(prec: str):
    return np.float64 if prec == "f64" else np.float32


def min_space_sampling(lay: GridLayout, samp: Sampling):
    """Grid::getMinSpaceSampling: min over the used axes, stored as Myfloat."""
    T = _T(lay.prec)
    m = T(samp.d[0])
    if lay.dim >= 2:
        m = T(min(float(m), samp.d[1]))
    if lay.dim >= 3:
        m = T(min(float(m), samp.d[2]))
    return m


@dataclass(frozen=True)
class EigenSetup:
    """Everything Propagator_Ac2::initialize(EIGEN_MODE) fixes."""
    samp: Sampling
    cfl: float
    stable_dt: float
    dt: float
    nt: int
    tmax: float
    snap_inc: int
    coef: float                 # v^2 dt^2 with v = 1 (src/propagator_Ac2.cpp:234)
    modes: Tuple[int, int, int]
    gamma: float
    freq_max: float

    def params(self, lay: GridLayout) -> Tuple[float, float, float]:
        """(val1, val2, val3) of initializeGrid (src/propagator_Ac2.cpp:462-530)."""
        m = self.modes
        vals = [PI * m[0], PI * m[1] if lay.dim >= 2 else 1.0, PI * m[2] if lay.dim >= 3 else 1.0]
        return tuple(vals)

    def amplitude(self, time_sec) -> float:
        """sin(PI * timeSec * gamma) (src/propagator_Ac2.cpp:533)."""
        return math.sin(PI * float(time_sec) * self.gamma)

    def time_of_step(self, it: int, prec: str):
        """Myfloat timeSec = it * dt (src/testCase_Propa.cpp:141)."""
        T = _T(prec)
        return T(T(it) * T(self.dt))


def eigen_setup(lay: GridLayout, ratio_cfl: float = 1.0, tmax: Optional[float] = None,
                nt: int = 20, dt: float = 0.0, snap_inc: int = 1,
                modes: Tuple[float, float, float] = (0.8, 0.9, 1.0)) -> EigenSetup:
    """Propagator_Ac2::initialize(EIGEN_MODE) for one rank.

    Defaults are the reference's Config defaults (src/config.cpp:33-83):
    ratioCFL 1, nt 20, dt 0 (= stable dt), snapInc 1, param1..3 = 0.8, 0.9, 1.0
    (the number of modes is ceil(param))."""
    T = _T(lay.prec)
    samp = unit_sampling(lay)
    vp = T(1.0)
    c = T(fdm.cfl(lay.order, lay.dim, T))
    stable = T(T(c * min_space_sampling(lay, samp)) / vp)
    if dt > 0.0:
        dt_v = T(dt)
    else:
        dt_v = T(float(stable) * ratio_cfl)
    if tmax is not None:
        tmax_v = T(tmax)
        nt_v = int(T(T(tmax_v / dt_v) + T(1)))
    else:
        nt_v = int(nt)
        tmax_v = T(T(nt_v - 1) * dt_v)
    coef = T(T(T(vp * vp) * dt_v) * dt_v)
    m = tuple(int(math.ceil(p)) for p in modes)
    if lay.dim == 1:
        gamma = float(m[0])
    elif lay.dim == 2:
        gamma = math.sqrt(m[0] * m[0] + m[1] * m[1])
    else:
        gamma = math.sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2])
    return EigenSetup(samp=samp, cfl=float(c), stable_dt=float(stable), dt=float(dt_v), nt=nt_v,
                      tmax=float(tmax_v), snap_inc=int(snap_inc), coef=float(coef), modes=m,
                      gamma=gamma, freq_max=gamma / 2.0)


def init_times(setup: EigenSetup, prec: str):
    """Times of the two initial fields: prn at -2 dt, prc at -dt
    (src/propagator_Ac2.cpp:272-285; Myfloat timeSec = -2.0 * dt)."""
    T = _T(prec)
    return T(-2.0 * setup.dt), T(-T(setup.dt))


EIGEN_FUNCS = (FUNC_SINE, FUNC_SINE, FUNC_SINE)
