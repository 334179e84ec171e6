"""GPU parity of the hpcscan_b200 kernels against the oracle (oracle/oracle.c, itself
pinned to the reference) and against the reference-written golden grids.

Elementwise results (fills, FD_D2, Laplacian, pressure update, boundary condition)
must be BIT-IDENTICAL in FP32 and FP64: the kernels evaluate the reference's
expressions in its order with separately rounded operations. FP64 norms are
compared at 1e-12 relative (summation order differs).
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from hpcscan_b200 import layout as L  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MANIFEST = json.load(open(os.path.join(GOLDEN, "manifest.json")))
ORDERS = (2, 4, 6, 8, 10, 12, 14, 16)


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hpcscan_b200.grid import init_device
    init_device(0)
    return torch


def dev(lay, arr=None, samp=None):
    from hpcscan_b200.grid import Grid
    g = Grid(lay, samp)
    g.initializeGrid()
    if arr is not None:
        g.from_numpy(arr)
    return g


def rand_field(lay, seed):
    rng = np.random.default_rng(seed)
    t = np.float32 if lay.prec == "f32" else np.float64
    return rng.uniform(-1.0, 1.0, lay.npoint).astype(t)


def bits(a):
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def layouts():
    """3-D layouts exercising both kernel families (the B200 layout goes to the z-marching
    TMA kernel; the reference layout, whose row pitch is not a multiple of 16 bytes, to
    the direct kernel), with several tiles and z-chunks and partial edge tiles, plus 1-D
    and 2-D."""
    out = []
    for prec in ("f32", "f64"):
        for o in ORDERS:
            out.append(L.b200_layout(3, 37, 20, 23, order=o, prec=prec))
        out.append(L.b200_layout(3, 130, 37, 150, order=8, prec=prec))
        out.append(L.b200_layout(3, 70, 33, 41, order=16, prec=prec))
        out.append(L.b200_layout(3, 77, 45, 70, order=2, prec=prec))
        out.append(L.reference_layout(3, 29, 21, 20, order=6, prec=prec))
        out.append(L.reference_layout(3, 31, 21, 20, order=8, prec=prec))
        out.append(L.reference_layout(2, 40, 33, order=12, prec=prec))
        out.append(L.reference_layout(1, 57, order=16, prec=prec))
    return out


def lay_id(lay):
    return f"d{lay.dim}_o{lay.order}_{lay.prec}_{lay.n1}x{lay.n2}x{lay.n3}"


def route(lay):
    import ctypes
    from hpcscan_b200 import _lib
    r = ctypes.c_int()
    cl = _lib.Layout(*lay.c_struct_fields())
    _lib.call("b200_stencil_route", ctypes.byref(cl), lay.order, _lib.DTYPE_CODE[lay.prec],
              ctypes.byref(r))
    return r.value


def device_status():
    import ctypes
    from hpcscan_b200 import _lib
    st = ctypes.c_int()
    _lib.call("b200_device_status", ctypes.byref(st), 1)
    return st.value


def test_routes(gpu):
    """The B200 layout of every 3-D FP32/FP64 grid takes the z-marching TMA kernel."""
    for prec in ("f32", "f64"):
        for o in ORDERS:
            assert route(L.b200_layout(3, 37, 20, 23, order=o, prec=prec)) == 1
        assert route(L.b200_layout(2, 37, 20, order=8, prec=prec)) == 2
    # row pitch not a multiple of 16 bytes: direct kernel
    assert route(L.reference_layout(3, 29, 21, 20, order=6, prec="f64")) == 2
    assert route(L.reference_layout(3, 31, 21, 20, order=8)) == 2


@pytest.mark.parametrize("lay", layouts(), ids=lay_id)
def test_fd_operators_bitexact(gpu, oracle, lay):
    u = rand_field(lay, 1)
    samp = L.Sampling((0.013, 0.011, 0.017), (0.0, 0.0, 0.0))
    inv2 = L.inv2_spacing(samp, lay.prec)
    U = dev(lay, u, samp)
    for axis in range(0, lay.dim + 1):
        W = dev(lay, None, samp)
        w_ref = oracle.alloc(lay)
        if axis == 0:
            assert U.FD_LAPLACIAN(L.INNER_POINTS, W, lay.order) == 0
            oracle.laplacian(lay, u, w_ref, inv2)
        else:
            assert getattr(U, f"FD_D2_N{axis}")(L.INNER_POINTS, W, lay.order) == 0
            oracle.fd_d2(lay, axis, u, w_ref, inv2)
        got = W.to_numpy()
        assert np.array_equal(bits(got), bits(w_ref)), (axis, np.abs(got - w_ref).max())
    assert device_status() == 0


@pytest.mark.parametrize("lay", layouts() + [L.b200_layout(3, 45, 130, 29, order=10),
                                     L.b200_layout(3, 33, 17, 300, order=4, prec="f64")],
                         ids=lay_id)
def test_fd_d1_bitexact(gpu, oracle, lay):
    """FD_D1_N1/N2/N3 (staggered first derivative) against the oracle, bit for bit; the
    layouts cover partial x tiles and marched chunks of every remainder."""
    u = rand_field(lay, 2)
    samp = L.Sampling((0.013, 0.011, 0.017), (0.0, 0.0, 0.0))
    inv = L.inv_spacing(samp, lay.prec)
    U = dev(lay, u, samp)
    for axis in range(1, lay.dim + 1):
        W = dev(lay, None, samp)
        assert getattr(U, f"FD_D1_N{axis}")(L.INNER_POINTS, W, lay.order) == 0
        w_ref = oracle.alloc(lay)
        oracle.fd_d1(lay, axis, u, w_ref, inv)
        got = W.to_numpy()
        assert np.array_equal(bits(got), bits(w_ref)), (axis, np.abs(got - w_ref).max())
        # the halos and the outer points stay as they were (zero)
        outside = lay.view3(got.copy())
        outside[lay.box_slices(L.INNER_POINTS)] = 0
        assert not outside.any()


def test_fd_d1_fp16_storage_matches_fp32_oracle(gpu, oracle):
    """16-bit storage, FP32 arithmetic: the FP32 oracle on the widened inputs, rounded once to
    FP16, gives the same bits."""
    import dataclasses
    lay = L.b200_layout(3, 40, 21, 26, order=8, prec="f16")
    lay32 = dataclasses.replace(lay, prec="f32")
    u16 = rand_field(lay32, 3).astype(np.float16)
    samp = L.Sampling((0.5, 0.25, 0.125), (0.0, 0.0, 0.0))
    inv = L.inv_spacing(samp, "f32")
    U = dev(lay, u16, samp)
    for axis in (1, 2, 3):
        W = dev(lay, None, samp)
        assert getattr(U, f"FD_D1_N{axis}")(L.INNER_POINTS, W, 8) == 0
        w_ref = oracle.alloc(lay32)
        oracle.fd_d1(lay32, axis, u16.astype(np.float32), w_ref, inv)
        got = lay.inner(W.to_numpy()).astype(np.float16)
        want = lay32.inner(w_ref).astype(np.float16)
        assert np.array_equal(got.view(np.uint16), want.view(np.uint16)), axis


def test_fd_d1_rejects_bad_arguments(gpu):
    import ctypes
    from hpcscan_b200 import _lib
    lay = L.b200_layout(2, 40, 33, order=8)
    U, W = dev(lay), dev(lay)
    cl = _lib.Layout(*lay.c_struct_fields())
    for axis, order in ((3, 8), (0, 8), (1, 18), (1, 7)):
        rc = _lib.load().b200_fd_d1(ctypes.byref(cl), axis, order, U.c_field(), W.c_field(),
                                   1.0, 1.0, 1.0, None)
        assert rc != 0, (axis, order)
    rc = _lib.load().b200_fd_d1(ctypes.byref(cl), 1, 8, U.c_field(), U.c_field(), 1.0, 1.0, 1.0, None)
    assert rc != 0
    narrow = L.b200_layout(2, 40, 33, order=4)     # halo 2 < 16 / 2
    cn = _lib.Layout(*narrow.c_struct_fields())
    V, X = dev(narrow), dev(narrow)
    assert _lib.load().b200_fd_d1(ctypes.byref(cn), 1, 16, V.c_field(), X.c_field(), 1.0, 1.0,
                                 1.0, None) != 0


@pytest.mark.parametrize("lay", layouts(), ids=lay_id)
def test_compute_pressure_bitexact(gpu, oracle, lay):
    prc, prn, coef = rand_field(lay, 2), rand_field(lay, 3), np.abs(rand_field(lay, 4)) * 1e-3
    samp = L.Sampling((0.02, 0.03, 0.025), (0.0, 0.0, 0.0))
    inv2 = L.inv2_spacing(samp, lay.prec)
    Prc, Prn, Coef = dev(lay, prc, samp), dev(lay, prn, samp), dev(lay, coef, samp)
    assert Prn.computePressureWithFD(Prc, Coef, lay.order) == 0
    ref = prn.copy()
    oracle.compute_pressure(lay, ref, prc, coef, inv2)
    got = Prn.to_numpy()
    assert np.array_equal(bits(got), bits(ref)), np.abs(got - ref).max()
    assert device_status() == 0
    # the input is untouched
    assert np.array_equal(bits(Prc.to_numpy()), bits(prc))


@pytest.mark.parametrize("lay", layouts(), ids=lay_id)
def test_update_pressure_bitexact(gpu, oracle, lay):
    a = [rand_field(lay, s) for s in (5, 6, 7, 8)]
    G = [dev(lay, x) for x in a]
    assert G[0].updatePressure(L.INNER_POINTS, G[1], G[2], G[3]) == 0
    ref = a[0].copy()
    oracle.update_pressure(lay, ref, a[1], a[2], a[3])
    assert np.array_equal(bits(G[0].to_numpy()), bits(ref))


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_array_ops_bitexact(gpu, prec):
    """Grid::fillArray / copyArray / addArray / multiplyArray / addUpdateArray over every point
    (src/grid.cpp:1828-1918): IEEE operations in the storage type, so numpy gives the bits."""
    lay = L.b200_layout(3, 30, 21, 22, order=4, prec=prec)
    t = np.float32 if prec == "f32" else np.float64
    a, b, c = rand_field(lay, 21), rand_field(lay, 22), rand_field(lay, 23)
    A, B, C, W = dev(lay, a), dev(lay, b), dev(lay, c), dev(lay)
    W.fillArray(0.3)
    assert np.array_equal(bits(W.to_numpy()), bits(np.full(lay.npoint, 0.3, dtype=t)))
    W.copyArray(A)
    assert np.array_equal(bits(W.to_numpy()), bits(a))
    W.addArray(A, B)
    assert np.array_equal(bits(W.to_numpy()), bits(a + b))
    W.multiplyArray(A, B)
    assert np.array_equal(bits(W.to_numpy()), bits(a * b))
    W.addUpdateArray(C)
    assert np.array_equal(bits(W.to_numpy()), bits(a * b + c))


BC_LAYOUTS = [L.b200_layout(3, 30, 21, 22, order=8), L.reference_layout(3, 25, 20, 21, order=16),
              L.b200_layout(3, 12, 9, 10, order=16, prec="f64"),      # small: sequential faces
              L.reference_layout(2, 33, 20, order=4, prec="f64"), L.reference_layout(1, 40, order=6),
              # the one-launch form at the other halo widths, several i1 runs, ny != nz
              L.b200_layout(3, 300, 17, 40, order=2), L.reference_layout(3, 37, 26, 19, order=6),
              L.b200_layout(3, 40, 33, 27, order=10, prec="f64"), L.b200_layout(3, 35, 30, 31, order=14),
              L.b200_layout(3, 530, 18, 19, order=12)]


@pytest.mark.parametrize("lay", BC_LAYOUTS, ids=lay_id)
def test_boundary_condition_bitexact(gpu, oracle, lay):
    """Anti-mirror BC: same bits as the reference's sequential faces, signs of zero included."""
    u = rand_field(lay, 9)
    U = dev(lay, u)
    assert U.applyBoundaryCondition() == 0
    ref = u.copy()
    oracle.apply_bc(lay, ref)
    assert np.array_equal(bits(U.to_numpy()), bits(ref))


@pytest.mark.parametrize("lay", BC_LAYOUTS[:2] + [L.b200_layout(3, 41, 33, 20, order=8, prec="f64")],
                         ids=lay_id)
def test_norms(gpu, oracle, lay):
    u1, u2 = rand_field(lay, 10), rand_field(lay, 11)
    A, B = dev(lay, u1), dev(lay, u2)
    for pt in (L.INNER_POINTS, L.ALL_POINTS, L.I1HALO1, L.I3INNERHALO2):
        box = lay.box(pt)
        np.testing.assert_allclose(A.getSumAbs(pt), oracle.sum_abs(lay, u1, box), rtol=1e-12)
        np.testing.assert_allclose(A.getSumAbsDiff(pt, B), oracle.sum_abs_diff(lay, u1, u2, box),
                                   rtol=1e-12)
        np.testing.assert_allclose(A.maxErr(pt, B), oracle.max_err(lay, u1, u2, box), rtol=1e-15)
        mn, mx = oracle.min_max(lay, u1, box)
        assert A.getMin(pt) == mn and A.getMax(pt) == mx
    np.testing.assert_allclose(A.L1Err(L.INNER_POINTS, B),
                               oracle.l1_err(lay, u1, u2, lay.box(L.INNER_POINTS)), rtol=1e-12)


def test_size_mismatch_and_bad_arguments(gpu):
    from hpcscan_b200 import _lib
    a = dev(L.b200_layout(3, 20, 20, 20, order=8))
    b = dev(L.b200_layout(3, 20, 21, 20, order=8))
    assert a.FD_LAPLACIAN(L.INNER_POINTS, b, 8) == -1            # RTN_CODE_KO
    assert a.getSumAbsDiff(L.INNER_POINTS, b) == -1.0
    assert a.L1Err(L.INNER_POINTS, b) == -1.0
    assert a.applyBoundaryCondition(7) == -1
    with pytest.raises(_lib.B200Error):
        a.FD_LAPLACIAN(L.INNER_POINTS, dev(a.layout), 6)        # halo/order mismatch
    with pytest.raises(ValueError):
        a.FD_D2_N1(L.INNER_POINTS, dev(a.layout), 5)


# ---- golden fixtures written by the reference ---------------------------------------------------

FD_FIXTURES = sorted(k for k, v in MANIFEST.items() if v["kind"] == "FD_D2")
PROPA_FIXTURES = sorted(k for k, v in MANIFEST.items() if v["kind"] == "Propa")


def flag_value(flags, name, default):
    return float(flags[flags.index(name) + 1]) if name in flags else default


@pytest.mark.parametrize("fixture", FD_FIXTURES)
def test_fd_golden_on_gpu(gpu, fixture):
    """Unchanged FD_D2 test-case inputs in the B200 layout: fill and every operator give the
    reference's inner values bit for bit."""
    meta = MANIFEST[fixture]
    gold = np.load(os.path.join(GOLDEN, fixture))
    flags = meta["flags"]
    lay = L.b200_layout(meta["dim"], *meta["n"], order=meta["order"], prec=meta["prec"])
    ref_lay = L.reference_layout(meta["dim"], *meta["n"], order=meta["order"], prec=meta["prec"])
    p = [flag_value(flags, f"-param{i + 1}", (0.8, 0.9, 1.0, 1.1)[i]) for i in range(4)]
    U = dev(lay)
    U.defineUnitGrid()
    U.fill(L.ALL_POINTS, L.FUNC_SINE, L.FUNC_SINE, L.FUNC_SINE, L.PI * p[0], L.PI * p[1],
           L.PI * p[2], p[3])
    if "U" in gold and not any("Pad" in f for f in flags):
        # the fill is independent of padding: compare the inner points
        assert np.array_equal(lay.inner(U.to_numpy()), ref_lay.inner(gold["U"]))
    for case in meta["cases"]:
        W = dev(lay)
        W.defineUnitGrid()
        if case.startswith("Axis"):
            getattr(U, f"FD_D2_N{case[-1]}")(L.INNER_POINTS, W, meta["order"])
        else:
            U.FD_LAPLACIAN(L.INNER_POINTS, W, meta["order"])
        assert np.array_equal(lay.inner(W.to_numpy()), gold[case]), case


FDD1_FIXTURES = sorted(k for k, v in MANIFEST.items() if v["kind"] == "FD_D1")


@pytest.mark.parametrize("fixture", FDD1_FIXTURES)
def test_fd_d1_golden_on_gpu(gpu, fixture):
    """Unchanged FD_D1 test-case inputs in the B200 layout give the reference's inner values
    of every axis bit for bit."""
    meta = MANIFEST[fixture]
    gold = np.load(os.path.join(GOLDEN, fixture))
    flags = meta["flags"]
    lay = L.b200_layout(meta["dim"], *meta["n"], order=meta["order"], prec=meta["prec"])
    p = [flag_value(flags, f"-param{i + 1}", (0.8, 0.9, 1.0, 1.1)[i]) for i in range(4)]
    U = dev(lay)
    U.defineUnitGrid()
    U.fill(L.ALL_POINTS, L.FUNC_SINE, L.FUNC_SINE, L.FUNC_SINE, L.PI * p[0], L.PI * p[1],
           L.PI * p[2], p[3])
    for case in meta["cases"]:
        W = dev(lay)
        W.defineUnitGrid()
        assert getattr(U, f"FD_D1_N{case[-1]}")(L.INNER_POINTS, W, meta["order"]) == 0
        assert np.array_equal(lay.inner(W.to_numpy()), gold[case]), case


@pytest.mark.parametrize("fixture", PROPA_FIXTURES)
def test_propa_golden_on_gpu(gpu, fixture):
    """The Propa test case (standard and split propagators) on the GPU reproduces the
    reference's wavefields bit for bit at every check, and its errTestCase."""
    from hpcscan_b200.propagator import run_propa
    meta = MANIFEST[fixture]
    gold = np.load(os.path.join(GOLDEN, fixture))
    flags = meta["flags"]
    lay = L.b200_layout(meta["dim"], *meta["n"], order=meta["order"], prec=meta["prec"])
    got = []
    res = run_propa(lay, propagator=meta["propagator"],
                    ratio_cfl=flag_value(flags, "-ratioCFL", 1.0),
                    nt=int(flag_value(flags, "-nt", 20)),
                    snap_inc=int(flag_value(flags, "-snapInc", 1)),
                    modes=tuple(flag_value(flags, f"-param{i + 1}", (0.8, 0.9, 1.0)[i])
                                for i in range(3)),
                    on_check=lambda it, prn, ref: got.append(lay.inner(prn.to_numpy())))
    assert res.nt == meta["nt"]
    for i, g in enumerate(got):
        assert np.array_equal(g, gold[f"prn_{i}"]), i
    assert abs(res.err_test_case - meta["err_test_case"]) <= 2e-5 * abs(meta["err_test_case"])


def test_fused_check_equals_materialised_reference(gpu):
    """b200_l1_sums_separable gives the sums of fill + getSumAbsDiff + getSumAbs."""
    from hpcscan_b200.propagator import run_propa
    lay = L.b200_layout(3, 40, 36, 33, order=8)
    a = run_propa(lay, nt=12, snap_inc=3, fused_check=True)
    b = run_propa(lay, nt=12, snap_inc=3, fused_check=False)
    for (ia, s1a, s2a), (ib, s1b, s2b) in zip(a.checks, b.checks):
        assert ia == ib
        np.testing.assert_allclose([s1a, s2a], [s1b, s2b], rtol=1e-12)
    assert a.err_test_case == b.err_test_case


# ---- the fused propagator step (boundary condition inside the pressure kernel) -----------------

STEP_LAYOUTS = [L.b200_layout(3, 37, 20, 23, order=8), L.b200_layout(3, 70, 33, 41, order=16),
                L.b200_layout(3, 130, 37, 150, order=8), L.b200_layout(3, 66, 49, 35, order=4),
                L.b200_layout(3, 21, 22, 20, order=2), L.b200_layout(3, 45, 27, 29, order=6),
                L.b200_layout(3, 52, 31, 40, order=12, prec="f64"),
                L.b200_layout(3, 37, 20, 23, order=8, prec="f64"),
                L.b200_layout(3, 33, 40, 22, order=14), L.b200_layout(3, 29, 21, 25, order=10),
                # tiles and z-chunks clear of every boundary (the fused step's unpatched CTAs)
                L.b200_layout(3, 200, 60, 50, order=8),
                L.b200_layout(3, 120, 60, 50, order=12, prec="f64")]


def propagate_step(lay, prn, prc, coef, samp):
    import ctypes
    from hpcscan_b200 import _lib
    cl = _lib.Layout(*lay.c_struct_fields())
    i1, i2, i3 = L.inv2_spacing(samp, lay.prec)
    _lib.call("b200_propagate_step", ctypes.byref(cl), lay.order, prn.c_field(), prc.c_field(),
              coef.c_field(), i1, i2, i3, 1, None)


@pytest.mark.parametrize("lay", STEP_LAYOUTS, ids=lay_id)
@pytest.mark.parametrize("shape,chunk", [(0, 0), (1, 16), (2, 7)])
def test_fused_step_bitexact(gpu, oracle, lay, shape, chunk):
    """b200_propagate_step (BC fused into the pressure kernel) == applyBoundaryCondition +
    computePressureWithFD of the oracle, bit for bit, over several steps; prc's inner points
    (with the zeroed boundary planes) too. Every tile shape, with z-chunks that put chunk
    edges next to the boundary planes."""
    from hpcscan_b200 import _lib
    _lib.call("b200_set_stencil_config", _lib.DTYPE_CODE[lay.prec], lay.order, _lib.OP_STEP,
              shape, chunk)
    try:
        prc, prn, coef = rand_field(lay, 12), rand_field(lay, 13), np.abs(rand_field(lay, 14)) * 1e-3
        samp = L.Sampling((0.02, 0.03, 0.025), (0.0, 0.0, 0.0))
        inv2 = L.inv2_spacing(samp, lay.prec)
        Prc, Prn, Coef = dev(lay, prc, samp), dev(lay, prn, samp), dev(lay, coef, samp)
        a, b = prn.copy(), prc.copy()
        for it in range(3):
            propagate_step(lay, Prn, Prc, Coef, samp)
            oracle.apply_bc(lay, b)
            oracle.compute_pressure(lay, a, b, coef, inv2)
            assert np.array_equal(bits(lay.inner(Prn.to_numpy())), bits(lay.inner(a))), it
            assert np.array_equal(bits(lay.inner(Prc.to_numpy())), bits(lay.inner(b))), it
            Prn, Prc = Prc, Prn
            a, b = b, a
        assert device_status() == 0
    finally:
        _lib.call("b200_set_stencil_config", _lib.DTYPE_CODE[lay.prec], lay.order, _lib.OP_STEP, -1, 0)


def test_fused_step_small_grid_falls_back(gpu, oracle):
    """Fewer than halo + 2 inner points on an axis: the two operators run back to back."""
    lay = L.b200_layout(3, 30, 9, 25, order=16)
    prc, prn, coef = rand_field(lay, 15), rand_field(lay, 16), np.abs(rand_field(lay, 17)) * 1e-3
    samp = L.Sampling((0.02, 0.03, 0.025), (0.0, 0.0, 0.0))
    Prc, Prn, Coef = dev(lay, prc, samp), dev(lay, prn, samp), dev(lay, coef, samp)
    propagate_step(lay, Prn, Prc, Coef, samp)
    oracle.apply_bc(lay, prc)
    oracle.compute_pressure(lay, prn, prc, coef, L.inv2_spacing(samp, lay.prec))
    assert np.array_equal(bits(Prn.to_numpy()), bits(prn))
    assert np.array_equal(bits(Prc.to_numpy()), bits(prc))


@pytest.mark.parametrize("lay", [L.b200_layout(3, 70, 33, 41, order=10), L.b200_layout(3, 45, 30, 37, order=16),
                                 L.b200_layout(3, 37, 20, 23, order=8), L.b200_layout(3, 41, 30, 26, order=12, prec="f64"),
                                 L.b200_layout(3, 36, 22, 19, order=16, prec="f64")], ids=lay_id)
@pytest.mark.parametrize("shape", [0, 1, 2])
def test_pressure_and_laplacian_every_shape(gpu, oracle, lay, shape):
    """computePressureWithFD and FD_LAPLACIAN through every tile shape of the z-marching kernel
    (two- and four-plane prefetch, 8- and 9-warp tiles), bit for bit."""
    from hpcscan_b200 import _lib
    dt = _lib.DTYPE_CODE[lay.prec]
    for op in (_lib.OP_PRESSURE, _lib.OP_LAPLACIAN):
        _lib.call("b200_set_stencil_config", dt, lay.order, op, shape, 0)
    try:
        prc, prn, coef = rand_field(lay, 21), rand_field(lay, 22), np.abs(rand_field(lay, 23)) * 1e-3
        samp = L.Sampling((0.02, 0.03, 0.025), (0.0, 0.0, 0.0))
        inv2 = L.inv2_spacing(samp, lay.prec)
        Prc, Prn, Coef, W = dev(lay, prc, samp), dev(lay, prn, samp), dev(lay, coef, samp), dev(lay, None, samp)
        assert Prn.computePressureWithFD(Prc, Coef, lay.order) == 0
        assert Prc.FD_LAPLACIAN(L.INNER_POINTS, W, lay.order) == 0
        oracle.compute_pressure(lay, prn, prc, coef, inv2)
        w = oracle.alloc(lay)
        oracle.laplacian(lay, prc, w, inv2)
        assert np.array_equal(bits(Prn.to_numpy()), bits(prn))
        assert np.array_equal(bits(W.to_numpy()), bits(w))
        assert device_status() == 0
    finally:
        for op in (_lib.OP_PRESSURE, _lib.OP_LAPLACIAN):
            _lib.call("b200_set_stencil_config", dt, lay.order, op, -1, 0)
