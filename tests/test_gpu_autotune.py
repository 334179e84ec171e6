"""Tuning on first use (b200_set_autotune): the first launch of the pressure, Laplacian and
fused-step kernels on a grid of at least 2^24 inner points times the tile-shape and z-chunk
candidates for that grid size and keeps the fastest. Every candidate evaluates the same
expressions in the same order, so the tuned launch is bit-identical to the oracle; and it is
not slower than the untuned default beyond timing noise."""
import ctypes
import statistics

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from hpcscan_b200 import layout as L  # noqa: E402


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hpcscan_b200 import _lib
    from hpcscan_b200.grid import init_device
    init_device(0)
    _lib.call("b200_set_autotune", 1)
    return torch


def _dev(lay, arr, samp):
    from hpcscan_b200.grid import Grid
    g = Grid(lay, samp)
    g.initializeGrid()
    g.from_numpy(arr)
    return g


def _launch_ms(torch, fn, reps=10):
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(reps)]
    for a, b in ev:
        a.record()
        fn()
        b.record()
    torch.cuda.synchronize()
    return statistics.median(a.elapsed_time(b) for a, b in ev)


def test_tuned_pressure_bitexact_and_not_slower(gpu, oracle):
    from hpcscan_b200 import _lib
    from hpcscan_b200.grid import tuned_config
    lay = L.b200_layout(3, 256, 256, 256, order=8, prec="f32")      # 2^24 inner points
    rng = np.random.default_rng(5)
    prc = rng.uniform(-1, 1, lay.npoint).astype(np.float32)
    prn = rng.uniform(-1, 1, lay.npoint).astype(np.float32)
    coef = (np.abs(rng.uniform(-1, 1, lay.npoint)) * 1e-3).astype(np.float32)
    samp = L.Sampling((0.02, 0.03, 0.025), (0.0, 0.0, 0.0))
    Prc, Prn, Coef = _dev(lay, prc, samp), _dev(lay, prn, samp), _dev(lay, coef, samp)
    assert Prn.computePressureWithFD(Prc, Coef, 8) == 0           # first use: tunes, then runs
    t = tuned_config(Prn, _lib.OP_PRESSURE)
    assert t["measured"], t
    oracle.compute_pressure(lay, prn, prc, coef, L.inv2_spacing(samp, "f32"))
    assert np.array_equal(Prn.to_numpy().view(np.uint32), prn.view(np.uint32))
    # the tuned launch against the untuned default (forced), interleaved
    P2 = _dev(lay, prn, samp)
    tuned, default = [], []
    for _ in range(3):
        tuned.append(_launch_ms(gpu, lambda: P2.computePressureWithFD(Prc, Coef, 8)))
        _lib.call("b200_set_stencil_config", _lib.B200_F32, 8, _lib.OP_PRESSURE, 1, 0)
        try:
            default.append(_launch_ms(gpu, lambda: P2.computePressureWithFD(Prc, Coef, 8)))
        finally:
            _lib.call("b200_set_stencil_config", _lib.B200_F32, 8, _lib.OP_PRESSURE, -1, 0)
    print(f"tuned {t}: {min(tuned):.4f} ms, default shape 1: {min(default):.4f} ms")
    assert min(tuned) <= 1.05 * min(default), (tuned, default)


def test_tuned_step_and_laplacian_bitexact(gpu, oracle):
    """The fused-or-separate choice of the propagator step and the tuned Laplacian: prn and
    prc's inner points after b200_propagate_step, and the Laplacian, bit-identical to the
    oracle's boundary condition + pressure update and Laplacian."""
    from hpcscan_b200 import _lib
    from hpcscan_b200.grid import Grid, tuned_config
    lay = L.b200_layout(3, 256, 256, 256, order=12, prec="f32")
    rng = np.random.default_rng(6)
    prc = rng.uniform(-1, 1, lay.npoint).astype(np.float32)
    prn = rng.uniform(-1, 1, lay.npoint).astype(np.float32)
    coef = (np.abs(rng.uniform(-1, 1, lay.npoint)) * 1e-3).astype(np.float32)
    samp = L.Sampling((0.02, 0.03, 0.025), (0.0, 0.0, 0.0))
    inv2 = L.inv2_spacing(samp, "f32")
    Prc, Prn, Coef = _dev(lay, prc, samp), _dev(lay, prn, samp), _dev(lay, coef, samp)
    W = Grid(lay, samp)
    W.initializeGrid()
    assert Prc.FD_LAPLACIAN(L.INNER_POINTS, W, 12) == 0
    assert tuned_config(Prc, _lib.OP_LAPLACIAN)["measured"]
    w = np.zeros(lay.npoint, dtype=np.float32)
    oracle.laplacian(lay, prc, w, inv2)
    assert np.array_equal(W.to_numpy().view(np.uint32), w.view(np.uint32))
    assert Prn.propagateStep(Prc, Coef, 12) == 0
    step = tuned_config(Prn, _lib.OP_STEP)
    assert step["measured"], step
    oracle.apply_bc(lay, prc)
    oracle.compute_pressure(lay, prn, prc, coef, inv2)
    assert np.array_equal(lay.inner(Prn.to_numpy()).view(np.uint32), lay.inner(prn).view(np.uint32))
    assert np.array_equal(lay.inner(Prc.to_numpy()).view(np.uint32), lay.inner(prc).view(np.uint32))
    print(f"step at 256^3 O12: {step}")
    st = ctypes.c_int()
    _lib.call("b200_device_status", ctypes.byref(st), 1)
    assert st.value == 0
