"""ctypes binding of libhpcscan_b200.so (the C ABI declared in include/hpcscan_b200.h).

The library is built in-tree by hpcscan_b200/csrc/Makefile (see build()). There is
no fallback: if the shared library is missing or cannot be loaded, every entry
point raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhpcscan_b200.so")

B200_OK = 0
B200_F32, B200_F64, B200_F16, B200_BF16 = 0, 1, 2, 3
DTYPE_CODE = {"f32": B200_F32, "f64": B200_F64, "f16": B200_F16, "bf16": B200_BF16}
B200_NO_BOUND_COND, B200_BOUND_COND_ANTI_MIRROR = 0, 1


class B200Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"hpcscan_b200 error {code}: {msg}")
        self.code = code


class Layout(ctypes.Structure):
    _fields_ = [("n1", ctypes.c_int64), ("n2", ctypes.c_int64), ("n3", ctypes.c_int64),
                ("s1", ctypes.c_int64), ("e1", ctypes.c_int64), ("s2", ctypes.c_int64),
                ("e2", ctypes.c_int64), ("s3", ctypes.c_int64), ("e3", ctypes.c_int64),
                ("dim", ctypes.c_int32), ("halo", ctypes.c_int32)]


class Box(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("i1s", "i1e", "i2s", "i2e", "i3s", "i3e")]


class Field(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("dtype", ctypes.c_int32), ("scale", ctypes.c_float)]


class Shot(ctypes.Structure):
    _fields_ = [("lay", Layout), ("inv2", ctypes.c_double * 3), ("coef", ctypes.c_void_p),
                ("sponge", ctypes.c_void_p * 3), ("src", ctypes.c_int64), ("amp", ctypes.c_float),
                ("wavelet", ctypes.c_void_p), ("nrec", ctypes.c_int), ("rec", ctypes.c_void_p),
                ("traces", ctypes.c_void_p), ("dobs", ctypes.c_void_p), ("wave", ctypes.c_void_p),
                ("adj", ctypes.c_void_p), ("grad", ctypes.c_void_p)]


def build(quiet: bool = True) -> None:
    """Compile every CUDA source of hpcscan_b200/csrc for sm_100a into libhpcscan_b200.so."""
    subprocess.run(["make", "-C", os.path.join(HERE, "csrc"), "-j8"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


_VP = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_PL = ctypes.POINTER(Layout)
_PB = ctypes.POINTER(Box)
_PD = ctypes.POINTER(ctypes.c_double)

# name -> argtypes (all return int status unless listed in _RESTYPE)
SIGNATURES = {
    "b200_init": [_I],
    "b200_last_error": [],
    "b200_device_count": [ctypes.POINTER(_I)],
    "b200_malloc": [ctypes.POINTER(_VP), ctypes.c_size_t],
    "b200_free": [_VP],
    "b200_memcpy_h2d": [_VP, _VP, ctypes.c_size_t, _VP],
    "b200_memcpy_d2h": [_VP, _VP, ctypes.c_size_t, _VP],
    "b200_memcpy_d2d": [_VP, _VP, ctypes.c_size_t, _VP],
    "b200_memset": [_VP, _I, ctypes.c_size_t, _VP],
    "b200_stream_sync": [_VP],
    "b200_copy_box_d2h": [_PL, _I, _VP, _VP, _PB, _VP],
    "b200_copy_box_h2d": [_PL, _I, _VP, _VP, _PB, _VP],
    "b200_fill_const": [_PL, Field, _PB, _D, _VP],
    "b200_fill_separable": [_PL, Field, _PB, _VP, _VP, _VP, _D, _VP],
    "b200_array_op": [_I, ctypes.c_int64, Field, Field, Field, _D, _VP],
    "b200_gather_points": [Field, _VP, ctypes.c_int64, _VP, ctypes.c_int64, _VP],
    "b200_set_point": [Field, ctypes.c_int64, _D, _VP],
    "b200_fd_d2": [_PL, _I, _I, Field, Field, _D, _D, _D, _VP],
    "b200_fd_d1": [_PL, _I, _I, Field, Field, _D, _D, _D, _VP],
    "b200_laplacian": [_PL, _I, Field, Field, _D, _D, _D, _VP],
    "b200_update_pressure": [_PL, Field, Field, Field, Field, _VP],
    "b200_compute_pressure": [_PL, _I, Field, Field, Field, _D, _D, _D, _VP],
    "b200_apply_boundary": [_PL, Field, _I, _I, _VP],
    "b200_propagate_step": [_PL, _I, Field, Field, Field, _D, _D, _D, _I, _VP],
    "b200_sum_abs": [_PL, Field, _PB, _PD, _VP],
    "b200_sum_abs_diff": [_PL, Field, Field, _PB, _PD, _VP],
    "b200_l1_sums": [_PL, Field, Field, _PB, _PD, _PD, _VP],
    "b200_max_err": [_PL, Field, Field, _PB, _D, _PD, _VP],
    "b200_min_max": [_PL, Field, _PB, _PD, _PD, _VP],
    "b200_l1_sums_separable": [_PL, Field, _PB, _VP, _VP, _VP, _D, _I, _PD, _PD, _VP],
    "b200_l1_sums_separable_noalloc": [_PL, Field, _PB, _VP, _VP, _VP, _D, _I, _PD, _PD, _VP],
    "b200_device_status": [ctypes.POINTER(_I), _I],
    "b200_stencil_route": [_PL, _I, _I, ctypes.POINTER(_I)],
    "b200_batch_create": [ctypes.POINTER(_VP), _I, _I, _I, ctypes.POINTER(Shot), _D, _I],
    "b200_batch_destroy": [_VP],
    "b200_batch_forward_step": [_VP, _I, _I, _I, _I, _VP],
    "b200_batch_adjoint_step": [_VP, _I, _I, _VP],
    "b200_batch_gradient": [_VP, _I, _I, _VP],
    "b200_batch_survey_gradient": [_VP, _I, _I, _I, _I, _I, _VP, _VP],
    "b200_batch_info": [_VP, ctypes.POINTER(_I)],
    "b200_set_autotune": [_I],
    "b200_get_autotune": [ctypes.POINTER(_I)],
    "b200_prepare_stencil": [_PL, _I, _I, _I, _I],
    "b200_get_tuned_config": [_PL, _I, _I, _I, ctypes.POINTER(_I), ctypes.POINTER(_I),
                              ctypes.POINTER(_I), ctypes.POINTER(_I)],
    "b200_set_arith_mode": [_I],
    "b200_get_arith_mode": [ctypes.POINTER(_I)],
    "b200_set_stencil_config": [_I, _I, _I, _I, _I],
    "b200_get_stencil_config": [_I, _I, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)],
    "b200_autotune_stencil": [_PL, _I, _I, _I, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), _PD],
}
B200_ARITH_EXACT, B200_ARITH_FMA = 0, 1
B200_BATCH_ADJOINT, B200_BATCH_GRADIENT = 1, 2
B200_ARRAY_FILL, B200_ARRAY_COPY, B200_ARRAY_ADD, B200_ARRAY_MUL, B200_ARRAY_ADD_UPDATE = range(5)
OP_FD_D2_N1, OP_FD_D2_N2, OP_FD_D2_N3, OP_LAPLACIAN, OP_PRESSURE, OP_STEP = 1, 2, 3, 4, 5, 6
_RESTYPE = {"b200_last_error": ctypes.c_char_p}

_lib = None


def load() -> ctypes.CDLL:
    """Load the in-tree library once; raise if it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise B200Error(-3, f"{LIB_PATH} is not built; run hpcscan_b200._lib.build() "
                                "(or __graft_entry__.build())")
        lib = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = lib
    return _lib


def last_error() -> str:
    return load().b200_last_error().decode(errors="replace")


def check(rc: int) -> None:
    if rc != B200_OK:
        raise B200Error(rc, last_error())


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))
