"""b200_l1_sums_separable_noalloc, the variant of b200_l1_sums_separable that works on scratch
compiled into the library instead of allocating: the same sums as the allocating entry point on
consecutive calls, and boxes beyond its table capacity rejected with a clear error.

Kept in its own file, collected last, so that it runs both alone in a fresh process (where its
first call is the one that does the set-up) and after every other GPU test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from hpcscan_b200 import layout as L  # noqa: E402

TABLE_MAX = 16384      # table entries (nx + ny + nz) of the preallocated scratch


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hpcscan_b200.grid import init_device
    init_device(0)
    return torch


def _grid(lay, seed):
    from hpcscan_b200.grid import Grid
    g = Grid(lay)
    g.initializeGrid()
    rng = np.random.default_rng(seed)
    t = np.float32 if lay.prec == "f32" else np.float64
    g.from_numpy(rng.uniform(-1.0, 1.0, lay.npoint).astype(t))
    return g


def _tables(lay, seed):
    b = lay.box(L.INNER_POINTS)
    rng = np.random.default_rng(seed)
    return [np.ascontiguousarray(rng.uniform(-1.0, 1.0, b[2 * a + 1] - b[2 * a] + 1))
            for a in range(3)]


def _sums(entry, grid, tabs, amp):
    from hpcscan_b200 import _lib
    s1, s2 = ctypes.c_double(), ctypes.c_double()
    cl, box = grid.c_layout(), grid.c_box(L.INNER_POINTS)
    ref_dtype = _lib.DTYPE_CODE["f64" if grid.layout.prec == "f64" else "f32"]
    _lib.call(entry, ctypes.byref(cl), grid.c_field(), ctypes.byref(box),
              *[t.ctypes.data_as(ctypes.c_void_p) for t in tabs], float(amp), ref_dtype,
              ctypes.byref(s1), ctypes.byref(s2), None)
    return s1.value, s2.value


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_noalloc_matches_allocating_entry_on_consecutive_calls(gpu, prec):
    lay = L.b200_layout(3, 70, 45, 38, order=8, prec=prec)
    cases = [(_grid(lay, 1), _tables(lay, 2), 0.7), (_grid(lay, 3), _tables(lay, 4), 1.9)]
    for grid, tabs, amp in cases:          # two calls in a row, the no-alloc entry first
        got = _sums("b200_l1_sums_separable_noalloc", grid, tabs, amp)
        want = _sums("b200_l1_sums_separable", grid, tabs, amp)
        np.testing.assert_allclose(got, want, rtol=1e-12)
        assert got[0] > 0.0 and got[1] > 0.0


def test_noalloc_rejects_boxes_beyond_its_scratch(gpu):
    from hpcscan_b200 import _lib
    lay = L.b200_layout(1, TABLE_MAX, order=2)        # nx + ny + nz = TABLE_MAX + 2
    grid = _grid(lay, 5)
    with pytest.raises(_lib.B200Error) as e:
        _sums("b200_l1_sums_separable_noalloc", grid, _tables(lay, 6), 1.0)
    assert e.value.code == -3 and str(TABLE_MAX) in str(e.value)


def test_noalloc_calls_leave_free_device_memory_unchanged(gpu):
    """The property the entry point exists for: once its first call on the device has set it up,
    further calls take no device memory. Only no-alloc calls run between the two readings."""
    lay = L.b200_layout(3, 64, 48, 40, order=8, prec="f32")
    grid, tabs = _grid(lay, 7), _tables(lay, 8)
    first = _sums("b200_l1_sums_separable_noalloc", grid, tabs, 1.3)     # set-up call
    gpu.cuda.synchronize()
    free0, _ = gpu.cuda.mem_get_info()
    for _ in range(5):
        assert _sums("b200_l1_sums_separable_noalloc", grid, tabs, 1.3) == first
    gpu.cuda.synchronize()
    free1, _ = gpu.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
