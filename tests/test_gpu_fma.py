"""The FMA arithmetic mode (b200_set_arith_mode(B200_ARITH_FMA)): the z-marching Laplacian and
pressure update with fused multiply-adds. Not bit-identical to the reference CPU path, so it is
held to the FP32 noise floor instead: its error against the FP64 evaluation of the same inputs
stays within max(1e-5, 2 x the error of the reference's own FP32 arithmetic), the bound that the
FP32 build of hpcscan itself meets against its FP64 build.

Inputs are the FD_D2 test case's smooth field sin(4 pi x1) sin(6 pi x2) sin(8 pi x3) on the unit
cube (cancellation against 1/d^2 is what makes FP32 lose digits here) and, for the pressure
update, a second smooth field and a constant coef as the eigen-mode test sets them."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from hpcscan_b200 import layout as L  # noqa: E402

B200_ARITH_EXACT, B200_ARITH_FMA = 0, 1


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hpcscan_b200.grid import init_device
    init_device(0)
    return torch


@pytest.fixture
def fma_mode(gpu):
    from hpcscan_b200 import _lib
    _lib.call("b200_set_arith_mode", B200_ARITH_FMA)
    m = ctypes.c_int()
    _lib.call("b200_get_arith_mode", ctypes.byref(m))
    assert m.value == B200_ARITH_FMA
    yield
    _lib.call("b200_set_arith_mode", B200_ARITH_EXACT)


def _sine_grid(lay, params, amp):
    from hpcscan_b200.grid import Grid
    g = Grid(lay)
    g.initializeGrid()
    g.defineUnitGrid()
    g.fill(L.ALL_POINTS, L.FUNC_SINE, L.FUNC_SINE, L.FUNC_SINE, *params, amp)
    return g


def _rel(a, ref, lay):
    a, ref = lay.inner(a).astype(np.float64), lay.inner(ref)
    return float(np.linalg.norm((a - ref).ravel()) / np.linalg.norm(ref.ravel()))


def _f64(lay):
    """The same array geometry with FP64 arithmetic in the oracle (the FP32 grid's padding)."""
    import dataclasses
    return dataclasses.replace(lay, prec="f64")


@pytest.mark.parametrize("order", [4, 8, 12, 16])
@pytest.mark.parametrize("op", ["laplacian", "pressure"])
def test_fma_mode_within_fp32_noise_floor(gpu, oracle, fma_mode, order, op):
    from hpcscan_b200.grid import Grid
    lay = L.b200_layout(3, 130, 96, 80, order=order, prec="f32")
    lay64 = _f64(lay)
    a = (L.PI * 4, L.PI * 6, L.PI * 8)
    U = _sine_grid(lay, a, 1.0)
    u32 = U.to_numpy()
    inv2 = U.inv2()
    inv2_64 = L.inv2_spacing(U.sampling, "f64")
    if op == "laplacian":
        W = Grid(lay, U.sampling)
        W.initializeGrid()
        assert U.FD_LAPLACIAN(L.INNER_POINTS, W, order) == 0
        got = W.to_numpy()
        ref32 = oracle.alloc(lay)
        oracle.laplacian(lay, u32, ref32, inv2)
        ref64 = oracle.alloc(lay64)
        oracle.laplacian(lay64, u32.astype(np.float64), ref64, inv2_64)
    else:
        P = _sine_grid(lay, (L.PI, L.PI, L.PI), 0.9)
        C = Grid(lay, U.sampling)
        C.initializeGrid()
        coef = 2.1e-6                      # (v dt)^2 of the unit-cube eigen-mode test at this size
        C.fill(L.INNER_POINTS, coef)
        p32, c32 = P.to_numpy(), C.to_numpy()
        assert P.computePressureWithFD(U, C, order) == 0
        got = P.to_numpy()
        ref32 = p32.copy()
        oracle.compute_pressure(lay, ref32, u32, c32, inv2)
        ref64 = p32.astype(np.float64)
        oracle.compute_pressure(lay64, ref64, u32.astype(np.float64), c32.astype(np.float64),
                                inv2_64)
    floor = _rel(ref32, ref64, lay)
    err = _rel(got, ref64, lay)
    print(f"{op} O{order}: FMA {err:.3e}, reference FP32 {floor:.3e}")
    assert err <= max(1e-5, 2.0 * floor), (err, floor)
    # FMA arithmetic really ran: the exact mode is bit-identical to the oracle, this one is not
    assert not np.array_equal(lay.inner(got), lay.inner(ref32))
