"""ORACLE — test infrastructure, not product code.

ctypes front end of liboracle.so, the plain-C restatement of the hpcscan CPU
reference hot path (oracle.c; see its header for the reference citations and
for how its parity is pinned against the reference's own outputs).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")


class _Layout(ctypes.Structure):
    _fields_ = [("n1", ctypes.c_int64), ("n2", ctypes.c_int64), ("n3", ctypes.c_int64),
                ("s1", ctypes.c_int64), ("e1", ctypes.c_int64), ("s2", ctypes.c_int64),
                ("e2", ctypes.c_int64), ("s3", ctypes.c_int64), ("e3", ctypes.c_int64),
                ("dim", ctypes.c_int32), ("halo", ctypes.c_int32)]


class _Box(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("i1s", "i1e", "i2s", "i2e", "i3s", "i3e")]


# where the build recipes look for the hpcscan sources when REF_SRC is not set: the read-only
# checkout of the build container (absent on the GPU machines, which use the built files)
_REF_CHECKOUT_SRC = "/root/reference/src"


def reference_sources():
    """The src/ directory of the hpcscan checkout the recipes compile from (REF_SRC, else the
    build container's checkout), or None when neither exists."""
    for d in (os.environ.get("REF_SRC"), _REF_CHECKOUT_SRC):
        if d and os.path.isdir(d):
            return os.path.abspath(d)
    return None


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and, when the reference sources are present, the
    reference binaries in _ref/)."""
    targets = ["oracle"]
    ref_src = reference_sources()
    if ref_src:
        targets.append("ref")
    make = ["make", "-C", HERE, "-j8"] + ([f"REF_SRC={ref_src}"] if ref_src else [])
    subprocess.run(make + targets, check=True, stdout=subprocess.DEVNULL if quiet else None)
    if ref_src:
        # the reference's own CUDA modes, a comparison point only: a failure here leaves the
        # checker intact
        r = subprocess.run(make + ["ref-cuda"], stdout=subprocess.DEVNULL if quiet else None)
        if r.returncode != 0:
            print("oracle: the reference's CUDA modes did not build (comparison only)")


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        for suf, ct in (("f32", ctypes.c_float), ("f64", ctypes.c_double)):
            vp = ctypes.c_void_p
            getattr(_lib, f"oracle_fd_d2_{suf}").argtypes = [P(_Layout), ctypes.c_int, ctypes.c_int,
                                                             vp, vp, ct, ct, ct]
            getattr(_lib, f"oracle_fd_d1_{suf}").argtypes = [P(_Layout), ctypes.c_int, ctypes.c_int,
                                                             vp, vp, ct, ct, ct]
            getattr(_lib, f"oracle_laplacian_{suf}").argtypes = [P(_Layout), ctypes.c_int, vp, vp,
                                                                 ct, ct, ct]
            getattr(_lib, f"oracle_update_pressure_{suf}").argtypes = [P(_Layout), vp, vp, vp, vp]
            getattr(_lib, f"oracle_compute_pressure_{suf}").argtypes = [P(_Layout), ctypes.c_int,
                                                                        vp, vp, vp, ct, ct, ct]
            getattr(_lib, f"oracle_apply_bc_{suf}").argtypes = [P(_Layout), vp]
            getattr(_lib, f"oracle_fill_const_{suf}").argtypes = [P(_Layout), vp, P(_Box),
                                                                  ctypes.c_double]
            getattr(_lib, f"oracle_fill_sep_{suf}").argtypes = [P(_Layout), vp, P(_Box), vp, vp, vp,
                                                                ctypes.c_double]
            for name in ("sum_abs",):
                f = getattr(_lib, f"oracle_{name}_{suf}")
                f.argtypes = [P(_Layout), vp, P(_Box)]
                f.restype = ctypes.c_double
            for name in ("sum_abs_diff", "max_err"):
                f = getattr(_lib, f"oracle_{name}_{suf}")
                f.argtypes = [P(_Layout), vp, vp, P(_Box)]
                f.restype = ctypes.c_double
            getattr(_lib, f"oracle_min_max_{suf}").argtypes = [P(_Layout), vp, P(_Box),
                                                               P(ctypes.c_double),
                                                               P(ctypes.c_double)]
        d, vp, i64 = ctypes.c_double, ctypes.c_void_p, ctypes.c_int64
        _lib.oracle_model_forward_f64.argtypes = [P(_Layout), ctypes.c_int, vp, vp, i64, d, vp,
                                                  ctypes.c_int, ctypes.c_int, vp, d, d, d, vp, vp]
        _lib.oracle_model_adjoint_f64.argtypes = [P(_Layout), ctypes.c_int, vp, vp, ctypes.c_int,
                                                  ctypes.c_int, vp, d, d, d, vp, i64, vp, vp, d, vp]
        _lib.oracle_model_gradient_f64.argtypes = [P(_Layout), ctypes.c_int, vp, vp, i64, d, vp,
                                                   ctypes.c_int, ctypes.c_int, vp, d, d, d, vp, d,
                                                   vp, P(ctypes.c_double)]
    return _lib


# ---- FP64 modelling / adjoint (oracle_model.c) ----------------------------------------------------

def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(ctypes.c_void_p)


def model_forward(lay, C, G, src, amp, wavelet, rec, inv2, snapshots=False):
    """Traces (nt x nrec) of the damped leapfrog with a point source; with snapshots also
    p[0..nt] as an (nt + 1, npoint) array."""
    C, pc = _d(C)
    G, pg = _d(G)
    w, pw = _d(wavelet)
    rec = np.ascontiguousarray(rec, dtype=np.int64)
    nt, nrec = len(wavelet), len(rec)
    tr = np.zeros((nt, nrec))
    snap = np.zeros((nt + 1, lay.npoint)) if snapshots else None
    rc = lib().oracle_model_forward_f64(_L(lay), lay.order, pc, pg, int(src), float(amp), pw, nt,
                                        nrec, rec.ctypes.data_as(ctypes.c_void_p), *inv2,
                                        tr.ctypes.data_as(ctypes.c_void_p),
                                        None if snap is None else snap.ctypes.data_as(ctypes.c_void_p))
    assert rc == 0
    return (tr, snap) if snapshots else tr


def model_adjoint(lay, C, G, res, rec, src, inv2):
    """The adjoint wavefield w[n+1] at the source point, n = 0..nt-1, driven by res."""
    C, pc = _d(C)
    G, pg = _d(G)
    res, pr = _d(res)
    rec = np.ascontiguousarray(rec, dtype=np.int64)
    nt, nrec = res.shape
    w_src = np.zeros(nt)
    rc = lib().oracle_model_adjoint_f64(_L(lay), lay.order, pc, pg, nt, nrec,
                                        rec.ctypes.data_as(ctypes.c_void_p), *inv2, pr, int(src),
                                        w_src.ctypes.data_as(ctypes.c_void_p), None, 1.0, None)
    assert rc == 0
    return w_src


def model_gradient(lay, C, G, src, amp, wavelet, rec, inv2, dobs, dt):
    """(misfit, dJ/dm) for the squared slowness m (C = dt^2 / m)."""
    C, pc = _d(C)
    G, pg = _d(G)
    w, pw = _d(wavelet)
    dobs, po = _d(dobs)
    rec = np.ascontiguousarray(rec, dtype=np.int64)
    grad = np.zeros(lay.npoint)
    J = ctypes.c_double()
    rc = lib().oracle_model_gradient_f64(_L(lay), lay.order, pc, pg, int(src), float(amp), pw,
                                         len(wavelet), len(rec),
                                         rec.ctypes.data_as(ctypes.c_void_p), *inv2, po,
                                         float(dt) ** 2, grad.ctypes.data_as(ctypes.c_void_p),
                                         ctypes.byref(J))
    assert rc == 0
    return J.value, grad


def _suf(lay):
    if lay.prec not in ("f32", "f64"):
        raise ValueError("the oracle computes in the reference's FP32 or FP64 builds only")
    return lay.prec


def _np_t(lay):
    return np.float32 if lay.prec == "f32" else np.float64


def _L(lay):
    return _Layout(*lay.c_struct_fields())


def _B(b):
    return _Box(*b)


def _p(a, lay):
    assert a.dtype == _np_t(lay) and a.flags.c_contiguous and a.size == lay.npoint, \
        (a.dtype, a.size, lay.npoint)
    return a.ctypes.data_as(ctypes.c_void_p)


def alloc(lay, value=0.0):
    return np.full(lay.npoint, value, dtype=_np_t(lay))


def fd_d2(lay, axis, u, w, inv2):
    rc = getattr(lib(), f"oracle_fd_d2_{_suf(lay)}")(_L(lay), axis, lay.order, _p(u, lay),
                                                      _p(w, lay), *inv2)
    assert rc == 0


def fd_d1(lay, axis, u, w, inv):
    """Grid::FD_D1_N<axis> (src/grid.cpp:3401, 3735, 4069); inv = (1/d1, 1/d2, 1/d3)."""
    rc = getattr(lib(), f"oracle_fd_d1_{_suf(lay)}")(_L(lay), axis, lay.order, _p(u, lay),
                                                      _p(w, lay), *inv)
    assert rc == 0


def laplacian(lay, u, w, inv2):
    rc = getattr(lib(), f"oracle_laplacian_{_suf(lay)}")(_L(lay), lay.order, _p(u, lay),
                                                          _p(w, lay), *inv2)
    assert rc == 0


def update_pressure(lay, prn, prc, coef, lapla):
    getattr(lib(), f"oracle_update_pressure_{_suf(lay)}")(_L(lay), _p(prn, lay), _p(prc, lay),
                                                          _p(coef, lay), _p(lapla, lay))


def compute_pressure(lay, prn, prc, coef, inv2):
    rc = getattr(lib(), f"oracle_compute_pressure_{_suf(lay)}")(_L(lay), lay.order, _p(prn, lay),
                                                                _p(prc, lay), _p(coef, lay), *inv2)
    assert rc == 0


def apply_bc(lay, u):
    getattr(lib(), f"oracle_apply_bc_{_suf(lay)}")(_L(lay), _p(u, lay))


def fill_const(lay, u, box, val):
    getattr(lib(), f"oracle_fill_const_{_suf(lay)}")(_L(lay), _p(u, lay), _B(box), float(val))


def fill_sep(lay, u, box, tables, amp):
    t = [np.ascontiguousarray(x, dtype=np.float64) for x in tables]
    getattr(lib(), f"oracle_fill_sep_{_suf(lay)}")(
        _L(lay), _p(u, lay), _B(box), *[x.ctypes.data_as(ctypes.c_void_p) for x in t], float(amp))


def sum_abs(lay, u, box):
    return getattr(lib(), f"oracle_sum_abs_{_suf(lay)}")(_L(lay), _p(u, lay), _B(box))


def sum_abs_diff(lay, u1, u2, box):
    return getattr(lib(), f"oracle_sum_abs_diff_{_suf(lay)}")(_L(lay), _p(u1, lay), _p(u2, lay),
                                                              _B(box))


def max_err(lay, u1, u2, box):
    return getattr(lib(), f"oracle_max_err_{_suf(lay)}")(_L(lay), _p(u1, lay), _p(u2, lay), _B(box))


def l1_err(lay, u1, u2, box):
    """Grid::L1Err (src/grid.cpp:2058-2110): sum|u1-u2| / sum|u2|, with sum2
    replaced by npoint when it is below MAX_ERR_FLOAT."""
    s1 = sum_abs_diff(lay, u1, u2, box)
    s2 = sum_abs(lay, u2, box)
    if s2 < (1e-5 if lay.prec == "f32" else 1e-11):
        s2 = 1.0 * lay.npoint
    return s1 / s2


def min_max(lay, u, box):
    mn, mx = ctypes.c_double(), ctypes.c_double()
    getattr(lib(), f"oracle_min_max_{_suf(lay)}")(_L(lay), _p(u, lay), _B(box), ctypes.byref(mn),
                                                  ctypes.byref(mx))
    return mn.value, mx.value


def ref_binary(prec: str) -> str:
    """Path of the reference CPU binary built unchanged from the reference sources."""
    return os.path.join(REF_DIR, f"hpcscan_{'fp64' if prec == 'f64' else 'fp32'}")


def ref_gpu_binary() -> str:
    """Path of the reference built with its own CUDA test modes (CUDA, CUDA_Opt, CUDA_Ref), FP32,
    unchanged sources, for sm_100a."""
    return os.path.join(REF_DIR, "hpcscan_cuda_fp32")


def eigen_fields(lay, setup, point_type_all=True):
    """Initial fields of Propagator_Ac2::initialize(EIGEN_MODE): coef on INNER,
    prn at t = -2 dt and prc at t = -dt on ALL_POINTS."""
    from hpcscan_b200.layout import ALL_POINTS, INNER_POINTS, fill_tables
    from hpcscan_b200.propa_setup import EIGEN_FUNCS, init_times
    coef = alloc(lay)
    fill_const(lay, coef, lay.box(INNER_POINTS), setup.coef)
    tabs = fill_tables(lay, setup.samp, ALL_POINTS, EIGEN_FUNCS, setup.params(lay))
    t_prn, t_prc = init_times(setup, lay.prec)
    prn = alloc(lay)
    prc = alloc(lay)
    fill_sep(lay, prn, lay.box(ALL_POINTS), tabs, setup.amplitude(t_prn))
    fill_sep(lay, prc, lay.box(ALL_POINTS), tabs, setup.amplitude(t_prc))
    return prn, prc, coef, tabs


def propagate(lay, setup, nsteps=None, split=False, on_check=None):
    """TestCase_Propa time loop (src/testCase_Propa.cpp:111-161) with the
    Ac2Standard (computePressureWithFD) or Ac2SplitComp (Laplacian +
    updatePressure) kernel. Returns (prn, prc, errTestCase) with the reference's
    FP32 accumulation of the per-check sums."""
    from hpcscan_b200.layout import ALL_POINTS, INNER_POINTS, inv2_spacing
    prn, prc, coef, tabs = eigen_fields(lay, setup)
    inv2 = inv2_spacing(setup.samp, lay.prec)
    nt = setup.nt if nsteps is None else nsteps
    ref = alloc(lay)
    lapla = alloc(lay) if split else None
    acc = np.float32 if lay.prec == "f32" else np.float64
    sum1 = np.float32(0.0)
    sum2 = np.float32(0.0)
    inner = lay.box(INNER_POINTS)
    for it in range(nt):
        apply_bc(lay, prc)
        if split:
            laplacian(lay, prc, lapla, inv2)
            update_pressure(lay, prn, prc, coef, lapla)
        else:
            compute_pressure(lay, prn, prc, coef, inv2)
        if it % setup.snap_inc == 0:
            t = setup.time_of_step(it, lay.prec)
            fill_sep(lay, ref, lay.box(ALL_POINTS), tabs, setup.amplitude(t))
            s1 = acc(sum_abs_diff(lay, prn, ref, inner))
            s2 = acc(sum_abs(lay, ref, inner))
            sum1 = np.float32(sum1 + np.float32(s1))
            sum2 = np.float32(sum2 + np.float32(s2))
            if on_check is not None:
                on_check(it, prn, ref)
        prn, prc = prc, prn
    err = float(np.float32(sum1 / sum2)) if sum2 != 0 else float("nan")
    # after the last swap, the newest field is prc
    return prc, prn, err
