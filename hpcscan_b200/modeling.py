"""Batched acoustic modelling and adjoint-state gradients on the B200 engine.

The reference's propagator step (computePressureWithFD, src/grid.cpp:4612-5113; coef = (v dt)^2,
src/propagator_Ac2.cpp:234) with an absorbing sponge, a Ricker point source and point receivers,
for many shots of different grid sizes at once, plus the adjoint and the gradient of the
receiver-data misfit with respect to the squared slowness, with checkpointing. The reference has
no adjoint and runs one shot per process (TestCase_Modeling, src/testCase_Modeling.cpp:33-282);
its Ricker source follows DataAcquisition (src/data_Acquisition.cpp:58-352): f0 = freqMax / 2.5,
t0 = 1.5 sqrt(6) / (pi f0).

Every operation on the wavefields is a hpcscan_b200 kernel (b200_batch_*); torch allocates the
device memory and provides the stream (and, for the velocity models, generates the synthetic
inputs). A schedule of batch calls neither allocates nor synchronises, so it can be captured in a
CUDA graph (`graph=True`).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib, fdm
from .grid import init_device
from .layout import GridLayout, b200_layout


# ---- inputs -------------------------------------------------------------------------------------

def ricker(f0: float, dt: float, nt: int, t0: Optional[float] = None) -> np.ndarray:
    """Ricker wavelet (1 - 2 (pi f0 tau)^2) exp(-(pi f0 tau)^2), tau = n dt - t0 (FP32)."""
    if t0 is None:
        t0 = 1.5 * math.sqrt(6.0) / (math.pi * f0)
    tau = np.arange(nt, dtype=np.float64) * dt - t0
    a = (math.pi * f0 * tau) ** 2
    return ((1.0 - 2.0 * a) * np.exp(-a)).astype(np.float32)


def sponge_table(n: int, s: int, e: int, width: int, strength: float = 0.015) -> np.ndarray:
    """Damping factor along one axis: 1 inside, exp(-(strength (width - d))^2) on the `width`
    inner points nearest each edge (d = distance to the edge point), 0 in the halos."""
    g = np.zeros(n, dtype=np.float64)
    g[s:e + 1] = 1.0
    for d in range(min(width, (e - s + 1) // 2)):
        f = math.exp(-(strength * (width - d)) ** 2)
        g[s + d] = f
        g[e - d] = f
    return g.astype(np.float32)


def stable_dt(order: int, dx: float, vmax: float, ratio_cfl: float = 0.8) -> float:
    """dt = ratioCFL * CFL * dx / vmax with the reference's CFL number
    (Propagator_Ac2::getCFL, src/propagator_Ac2.cpp:410-439)."""
    return ratio_cfl * fdm.cfl(order, 3, np.float64) * dx / vmax


def grf_velocity(shape: Tuple[int, int, int], sigma: float, seed: int, vmin: float = 1500.0,
                 vmax: float = 4500.0, device: int = 0) -> torch.Tensor:
    """Smooth Gaussian random field (white noise, seeded, convolved with a Gaussian of
    `sigma` points along each axis) mapped affinely onto [vmin, vmax]. Shape (n3, n2, n1)."""
    g = torch.Generator().manual_seed(seed)
    x = torch.randn(shape, generator=g, dtype=torch.float32).to(f"cuda:{device}")
    r = int(math.ceil(3 * sigma))
    k = torch.exp(-0.5 * (torch.arange(-r, r + 1, dtype=torch.float32, device=x.device) / sigma) ** 2)
    k = (k / k.sum()).view(1, 1, -1)
    for axis in range(3):
        y = x.movedim(axis, -1)
        sh = y.shape
        y = y.reshape(-1, 1, sh[-1])
        y = torch.nn.functional.pad(y, (r, r), mode="replicate")
        y = torch.nn.functional.conv1d(y, k).reshape(sh)
        x = y.movedim(-1, axis).contiguous()
    lo, hi = x.min(), x.max()
    return (vmin + (x - lo) * ((vmax - vmin) / (hi - lo))).contiguous()


# ---- one shot -----------------------------------------------------------------------------------

@dataclass
class Shot:
    """One shot on its own grid: inner size n, model (velocity, inner points, (n3, n2, n1)),
    source and receivers (inner coordinates i1, i2, i3)."""
    n: Tuple[int, int, int]
    dx: float
    vel: torch.Tensor
    src: Tuple[int, int, int]
    rec: np.ndarray                       # (nrec, 3) inner coordinates
    amp: float = 1.0
    sponge: int = 20
    dobs: Optional[torch.Tensor] = None   # (nt, nrec) observed data, for the gradient


@dataclass
class _ShotState:
    lay: GridLayout
    coef: torch.Tensor
    sponge: List[torch.Tensor]
    wavelet: torch.Tensor
    rec: torch.Tensor
    traces: torch.Tensor
    dobs: Optional[torch.Tensor]
    wave: torch.Tensor
    adj: Optional[torch.Tensor]
    grad: Optional[torch.Tensor]
    ckpt: Optional[torch.Tensor] = None
    src_flat: int = 0


def _flat(lay: GridLayout, i1, i2, i3):
    return (lay.a1.inner_start + np.asarray(i1)) + (lay.a2.inner_start + np.asarray(i2)) * lay.n1 + \
        (lay.a3.inner_start + np.asarray(i3)) * lay.n1 * lay.n2


def embed(lay: GridLayout, inner: torch.Tensor) -> torch.Tensor:
    """Inner-point array (n3, n2, n1) -> full grid (flat, halos and padding zero)."""
    full = torch.zeros((lay.n3, lay.n2, lay.n1), dtype=torch.float32, device=inner.device)
    full[lay.a3.inner_start:lay.a3.inner_end + 1, lay.a2.inner_start:lay.a2.inner_end + 1,
         lay.a1.inner_start:lay.a1.inner_end + 1] = inner
    return full.reshape(-1)


def inner_of(lay: GridLayout, flat: torch.Tensor) -> torch.Tensor:
    return flat.view(lay.n3, lay.n2, lay.n1)[lay.a3.inner_start:lay.a3.inner_end + 1,
                                             lay.a2.inner_start:lay.a2.inner_end + 1,
                                             lay.a1.inner_start:lay.a1.inner_end + 1]


# ---- a batch ------------------------------------------------------------------------------------

class Batch:
    """Shots stepped in lockstep with one launch per stencil pass for all of them.

    `checkpoint` = k: the forward pass keeps (p[n-1], p[n]) every k steps and the backward pass
    recomputes each segment into a ring of k + 1 forward grids (memory per shot about
    (2 nt / k + k + 5) grids).

    `survey` (shots on one grid size, gradient=True): the backward pass accumulates the survey
    gradient (the sum over the shots) into one grid, one pass per step over all shots without a
    stencil (b200_batch_survey_gradient: C Lap p[n] from p[n+1], p[n], p[n-1], which the segment
    recompute keeps, one step further); the shots' own gradients are then not formed."""

    def __init__(self, shots: Sequence[Shot], order: int, dt: float, nt: int, f0: float,
                 gradient: bool = False, checkpoint: int = 45, device: int = 0,
                 survey: bool = False):
        init_device(device)
        self.order, self.dt, self.nt, self.device = order, float(dt), int(nt), device
        self.gradient = gradient
        self.survey = bool(survey)
        if self.survey:
            if not gradient:
                raise ValueError("survey=True needs gradient=True")
            if len({tuple(sh.n) for sh in shots}) != 1:
                raise ValueError("survey=True needs every shot on the same grid size")
        self.k = max(1, min(int(checkpoint), self.nt)) if gradient else 1
        # the survey gradient reads p[n+1] at the segment's last step: one more slot
        self.nslot = (self.k + 2 if self.survey else self.k + 1) if gradient else 2
        self.nckpt = (self.nt + self.k - 1) // self.k if gradient else 0
        dev = f"cuda:{device}"
        wav = torch.from_numpy(ricker(f0, dt, nt)).to(dev)
        self.states: List[_ShotState] = []
        c_shots = (_lib.Shot * len(shots))()
        for i, sh in enumerate(shots):
            lay = b200_layout(3, *sh.n, order=order, prec="f32")
            npt = lay.npoint
            coef = embed(lay, (sh.vel.to(dev) * self.dt) ** 2)
            sp = [torch.from_numpy(sponge_table(ax.n, ax.inner_start, ax.inner_end, sh.sponge)).to(dev)
                  for ax in (lay.a1, lay.a2, lay.a3)]
            rec = torch.from_numpy(_flat(lay, sh.rec[:, 0], sh.rec[:, 1], sh.rec[:, 2])
                                   .astype(np.int64)).to(dev)
            if len(torch.unique(rec)) != len(rec):
                raise ValueError("receivers of a shot must be distinct points")
            st = _ShotState(
                lay=lay, coef=coef, sponge=sp, wavelet=wav, rec=rec,
                traces=torch.zeros((nt, len(rec)), dtype=torch.float32, device=dev),
                dobs=None if sh.dobs is None else sh.dobs.to(dev).float().contiguous(),
                wave=torch.zeros((self.nslot, npt), dtype=torch.float32, device=dev),
                adj=torch.zeros((2, npt), dtype=torch.float32, device=dev) if gradient else None,
                grad=torch.zeros(npt, dtype=torch.float32, device=dev)
                if gradient and not self.survey else None,
                src_flat=int(_flat(lay, *sh.src)))
            if gradient:
                if st.dobs is None:
                    raise ValueError("the gradient needs observed data (Shot.dobs)")
                st.ckpt = torch.zeros((self.nckpt, 2, npt), dtype=torch.float32, device=dev)
            self.states.append(st)
            c = c_shots[i]
            c.lay = _lib.Layout(*lay.c_struct_fields())
            for a, d in enumerate((sh.dx, sh.dx, sh.dx)):
                c.inv2[a] = float(np.float32(1.0 / d) * np.float32(1.0 / d))
            c.coef = coef.data_ptr()
            for a in range(3):
                c.sponge[a] = sp[a].data_ptr()
            c.src = st.src_flat
            c.amp = float(sh.amp)
            c.wavelet = wav.data_ptr()
            c.nrec = len(rec)
            c.rec = rec.data_ptr()
            c.traces = st.traces.data_ptr()
            c.dobs = st.dobs.data_ptr() if st.dobs is not None else None
            c.wave = st.wave.data_ptr()
            c.adj = st.adj.data_ptr() if st.adj is not None else None
            c.grad = st.grad.data_ptr() if st.grad is not None else None
        self._c_shots = c_shots
        self.survey_grad = torch.zeros(self.states[0].lay.npoint, dtype=torch.float32,
                                       device=dev) if self.survey else None
        self.handle = ctypes.c_void_p()
        flags = ((_lib.B200_BATCH_ADJOINT if self.survey else
                  _lib.B200_BATCH_ADJOINT | _lib.B200_BATCH_GRADIENT) if gradient else 0)
        _lib.call("b200_batch_create", ctypes.byref(self.handle), order, self.nslot, len(shots),
                  c_shots, self.dt, flags)
        n = ctypes.c_int()
        _lib.call("b200_batch_info", self.handle, ctypes.byref(n))
        self.ctas_per_pass = n.value
        self.launches = 0

    def close(self):
        if self.handle:
            _lib.call("b200_batch_destroy", self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- schedule pieces (enqueue only) ---------------------------------------------------------
    def _s(self, stream):
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        return ctypes.c_void_p(s.cuda_stream)

    def _fwd(self, n, scur, sprev, sout, stream):
        _lib.call("b200_batch_forward_step", self.handle, n, scur, sprev, sout, self._s(stream))
        self.launches += 2

    def _copy(self, dst: torch.Tensor, src: torch.Tensor, stream):
        _lib.call("b200_memcpy_d2d", ctypes.c_void_p(dst.data_ptr()), ctypes.c_void_p(src.data_ptr()),
                  src.numel() * 4, self._s(stream))

    def _zero(self, t: torch.Tensor, stream):
        _lib.call("b200_memset", ctypes.c_void_p(t.data_ptr()), 0, t.numel() * 4, self._s(stream))

    def forward(self, stream=None) -> None:
        """nt forward steps of every shot from rest; traces filled; checkpoints when the batch
        computes gradients."""
        for st in self.states:
            self._zero(st.wave[0], stream)
            self._zero(st.wave[1], stream)
        for n in range(self.nt):
            cur, prev = (n + 1) % 2, n % 2          # slot of p[n], of p[n-1] (and of p[n+1])
            if self.gradient and n % self.k == 0:
                c = n // self.k
                for st in self.states:
                    self._copy(st.ckpt[c, 0], st.wave[prev], stream)
                    self._copy(st.ckpt[c, 1], st.wave[cur], stream)
            self._fwd(n, cur, prev, prev, stream)

    def backward(self, stream=None) -> None:
        """Adjoint and gradient of every shot, segment by segment from the checkpoints."""
        assert self.gradient
        if self.survey:
            return self._backward_survey(stream)
        for st in self.states:
            self._zero(st.adj, stream)
            self._zero(st.grad, stream)
        sv = ctypes.c_void_p
        for c in range(self.nckpt - 1, -1, -1):
            n0 = c * self.k
            end = min(n0 + self.k, self.nt)
            for st in self.states:                   # slot j holds p[n0 - 1 + j]
                self._copy(st.wave[0], st.ckpt[c, 0], stream)
                self._copy(st.wave[1], st.ckpt[c, 1], stream)
            for n in range(n0, end - 1):
                j = n - n0 + 1
                self._fwd(n, j, j - 1, j + 1, stream)
            for k in range(end, n0, -1):
                scur = (self.nt - k) % 2             # slot of w[k+1]
                _lib.call("b200_batch_adjoint_step", self.handle, k, scur, self._s(stream))
                _lib.call("b200_batch_gradient", self.handle, k - n0, 1 - scur, self._s(stream))
                self.launches += 3

    def _backward_survey(self, stream) -> None:
        """backward() with the survey gradient: the segment's recompute runs one step further
        (slot j holds p[n0 - 1 + j], j = 0 .. end - n0 + 1), and after adjoint step k the survey
        pass adds w[k] (C Lap p[k - 1]) of every shot."""
        for st in self.states:
            self._zero(st.adj, stream)
        self._zero(self.survey_grad, stream)
        gptr = ctypes.c_void_p(self.survey_grad.data_ptr())
        for c in range(self.nckpt - 1, -1, -1):
            n0 = c * self.k
            end = min(n0 + self.k, self.nt)
            for st in self.states:
                self._copy(st.wave[0], st.ckpt[c, 0], stream)
                self._copy(st.wave[1], st.ckpt[c, 1], stream)
            for n in range(n0, end):
                j = n - n0 + 1
                self._fwd(n, j, j - 1, j + 1, stream)
            for k in range(end, n0, -1):
                scur = (self.nt - k) % 2             # slot of w[k+1]
                _lib.call("b200_batch_adjoint_step", self.handle, k, scur, self._s(stream))
                j = k - n0                           # slot of p[k - 1]
                _lib.call("b200_batch_survey_gradient", self.handle, k - 1, j + 1, j, j - 1,
                          1 - scur, gptr, self._s(stream))
                self.launches += 3

    # ---- results --------------------------------------------------------------------------------
    def traces(self, i: int) -> torch.Tensor:
        return self.states[i].traces

    def gradient_of(self, i: int) -> torch.Tensor:
        """dJ/dm of shot i on its inner points, (n3, n2, n1)."""
        if self.survey:
            raise ValueError("a survey batch forms the sum over its shots only (survey_gradient_of)")
        return inner_of(self.states[i].lay, self.states[i].grad)

    def survey_gradient_of(self) -> torch.Tensor:
        """The sum over the shots of dJ/dm on the common inner points (survey batches)."""
        if not self.survey:
            raise ValueError("not a survey batch")
        return inner_of(self.states[0].lay, self.survey_grad)

    def misfit(self, i: int) -> float:
        st = self.states[i]
        r = (st.traces.double() - st.dobs.double()).cpu().numpy()
        return 0.5 * float((r * r).sum())


def run_graph(fn, stream: Optional[torch.cuda.Stream] = None):
    """Capture fn(stream) once into a CUDA graph and return the graph (replay() to run)."""
    s = stream if stream is not None else torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        fn(s)
    return g
