"""Mixed precision: FP16 / BF16 wavefields (power-of-two per-field scale), FP32 or 16-bit coef,
FP32 stencil arithmetic in the z-marching pressure kernel; error against the FP64 oracle and
against the analytic eigen-mode solution (the reference's own Propa check)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from hpcscan_b200 import layout as L  # noqa: E402

NT, SNAP = 80, 20


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hpcscan_b200.grid import init_device
    init_device(0)
    return torch


def route(lay):
    import ctypes
    from hpcscan_b200 import _lib
    r = ctypes.c_int()
    _lib.call("b200_stencil_route", ctypes.byref(_lib.Layout(*lay.c_struct_fields())), lay.order,
              _lib.DTYPE_CODE[lay.prec], ctypes.byref(r))
    return r.value


@pytest.mark.parametrize("prec,coef_prec,scale,tol", [
    ("f16", "f16", 2.0 ** -3, 1e-2), ("f16", "f32", 1.0, 1e-2),
    ("bf16", "bf16", 1.0, 4e-2), ("bf16", "f32", 2.0 ** 4, 4e-2)])
def test_16bit_wavefields_against_fp64_oracle(gpu, prec, coef_prec, scale, tol):
    from hpcscan_b200.propa_setup import eigen_setup
    from hpcscan_b200.propagator import run_propa
    from oracle import oracle
    n = (72, 56, 48)
    lay = L.b200_layout(3, *n, order=8, prec=prec)
    assert route(lay) == 1                       # the z-marching TMA kernel
    got = {}
    res = run_propa(lay, ratio_cfl=0.8, nt=NT, snap_inc=SNAP, modes=(1, 1, 1), coef_prec=coef_prec,
                    wave_scale=scale,
                    on_check=lambda it, prn, ref: got.__setitem__(it, lay.inner(prn.to_numpy()).astype(np.float64)))
    # FP64 oracle with the same time step and coefficient
    lay64 = L.b200_layout(3, *n, order=8, prec="f64")
    setup = eigen_setup(lay, ratio_cfl=0.8, nt=NT, snap_inc=SNAP, modes=(1, 1, 1))
    want = {}
    _, _, err64 = oracle.propagate(lay64, setup, on_check=lambda it, prn, ref: want.__setitem__(it, lay64.inner(prn).copy()))
    # errors relative to the wavefield's peak norm over the run (the first check is at t = 0,
    # where the eigen mode passes through zero and relative errors mean nothing)
    peak = max(np.linalg.norm(w) for w in want.values())
    for it in want:
        e = np.linalg.norm(got[it] - want[it]) / peak
        print(f"{prec}/{coef_prec} step {it}: relative L2 error vs FP64 oracle {e:.3e}")
        assert e < tol, (it, e)
    # the reference's analytic check stays within its own threshold (src/testCase_Propa.cpp:91)
    print(f"{prec}/{coef_prec} errTestCase {res.err_test_case:.4e} (FP64 oracle {err64:.4e})")
    assert res.err_test_case < 2e-2


@pytest.mark.parametrize("order", [10, 12, 14, 16])
@pytest.mark.parametrize("prec,scale,tol", [("f16", 2.0 ** 4, 1e-2), ("bf16", 1.0, 4e-2)])
def test_16bit_wavefields_high_orders_against_fp64_oracle(gpu, order, prec, scale, tol):
    """The 16-bit pressure kernels of the high orders (22-row tiles at O10-O12, the deeper
    9-warp tile at O14-O16), FP32 coef: 40 eigen-mode steps within the same bounds of the FP64
    oracle as at O8."""
    from hpcscan_b200.propa_setup import eigen_setup
    from hpcscan_b200.propagator import run_propa
    from oracle import oracle
    n, nt, snap = (72, 56, 48), 40, 20
    lay = L.b200_layout(3, *n, order=order, prec=prec)
    assert route(lay) == 1
    got = {}
    run_propa(lay, ratio_cfl=0.8, nt=nt, snap_inc=snap, modes=(1, 1, 1), coef_prec="f32",
              wave_scale=scale,
              on_check=lambda it, prn, ref: got.__setitem__(it, lay.inner(prn.to_numpy()).astype(np.float64)))
    # the FP64 oracle on the same array geometry (the grid origin follows the layout's first
    # inner index, which the 16-bit and FP64 layouts place differently at some orders)
    import dataclasses
    lay64 = dataclasses.replace(lay, prec="f64")
    setup = eigen_setup(lay, ratio_cfl=0.8, nt=nt, snap_inc=snap, modes=(1, 1, 1))
    want = {}
    oracle.propagate(lay64, setup, on_check=lambda it, prn, ref: want.__setitem__(it, lay64.inner(prn).copy()))
    peak = max(np.linalg.norm(w) for w in want.values())
    for it in want:
        e = np.linalg.norm(got[it] - want[it]) / peak
        print(f"{prec} O{order} step {it}: relative L2 error vs FP64 oracle {e:.3e}")
        assert e < tol, (it, e)


def _last_inner_field(torch, prec, coef_prec, scale, n, order, nt):
    """nt steps of the eigen-mode Propa test (boundary condition + pressure update per step) on
    the GPU; the last wavefield's inner points as physical FP64 values on the device."""
    from hpcscan_b200.propagator import Propagator_Ac2
    lay = L.b200_layout(3, n, n, n, order=order, prec=prec)
    p = Propagator_Ac2(lay, coef_prec=coef_prec, wave_scale=scale)
    p.initialize(ratio_cfl=0.8, nt=nt, snap_inc=nt, modes=(1, 1, 1))
    prn, prc = p.prnGrid, p.prcGrid
    for _ in range(nt):
        p.computeWavefieldNextTimeStep(prn, prc)
        prn, prc = prc, prn
    out = lay.inner(prc.data.detach()).to(torch.float64) * prc.scale
    del p, prn, prc
    torch.cuda.empty_cache()
    return out


def test_fp16_wavefields_512_cubed_1000_steps_within_one_percent_of_fp64(gpu):
    """The mixed-precision configuration's 512^3 O8 case at its stated length: FP16 wavefields
    (scale 2^4) with FP32 coef and FP32 arithmetic stay within 1 % (relative L2 of the last
    wavefield) of the FP64 run of the same 1000 steps, which is itself bit-identical to the
    reference's FP64 build."""
    torch = gpu
    ref = _last_inner_field(torch, "f64", "f64", 1.0, 512, 8, 1000)
    got = _last_inner_field(torch, "f16", "f32", 2.0 ** 4, 512, 8, 1000)
    rel = float(torch.linalg.vector_norm((got - ref).flatten()) /
                torch.linalg.vector_norm(ref.flatten()))
    print(f"FP16 512^3 O8, 1000 steps: relative L2 to FP64 {rel:.3e}")
    assert rel < 1e-2, rel
