"""Finite-difference operator tables of hpcscan (host side).

Restates, for host logic only, what src/fdm.h of vetienne74/hpcscan defines:
the centred second-derivative coefficients A0..A8 per order
(src/fdm.h:277-545), the halo width (src/fdm.h:770), the per-axis operation
counts `_NOP` (src/fdm.h:870-922) and the CFL coefficient sum
(src/fdm.h:743-756). The device kernels get the same numbers from
hpcscan_b200/csrc/b200_fdm.cuh.
"""
from __future__ import annotations

import math

import numpy as np

# A0..AR for orders 2..16 (src/fdm.h:277-545); exact rational values in FP64.
D2_COEF = {
    2: (-2.0, 1.0),
    4: (-5.0 / 2.0, 4.0 / 3.0, -1.0 / 12.0),
    6: (-49.0 / 18.0, 3.0 / 2.0, -3.0 / 20.0, 1.0 / 90.0),
    8: (-205.0 / 72.0, 8.0 / 5.0, -1 / 5.0, 8.0 / 315.0, -1 / 560.0),
    10: (-5269.0 / 1800.0, 5.0 / 3.0, -5.0 / 21.0, 5.0 / 126.0, -5.0 / 1008.0, 1.0 / 3150.0),
    12: (-5369.0 / 1800.0, 12.0 / 7.0, -15.0 / 56.0, 10.0 / 189.0, -1.0 / 112.0, 2.0 / 1925.0,
         -1.0 / 16632.0),
    14: (-266681.0 / 88200.0, 7.0 / 4.0, -7.0 / 24.0, 7.0 / 108.0, -7.0 / 528.0, 7.0 / 3300.0,
         -7.0 / 30888.0, 1.0 / 84084.0),
    16: (-1077749.0 / 352800.0, 16.0 / 9.0, -14.0 / 45.0, 112.0 / 1485.0, -7.0 / 396.0,
         112.0 / 32175.0, -2.0 / 3861.0, 16.0 / 315315.0, -1.0 / 411840.0),
}

# FD_D2_Ox_NOP: flops of one axis derivative (src/fdm.h:277-545)
D2_NOP = {2: 4, 4: 8, 6: 11, 8: 14, 10: 17, 12: 20, 14: 23, 16: 26}

ORDERS = tuple(sorted(D2_COEF))


def check_order(order: int) -> None:
    if order not in D2_COEF:
        raise ValueError(f"FD order {order} not supported (orders 2..16, even)")


def halo_width(order: int) -> int:
    """getFD_haloWidth (src/fdm.h:770)."""
    return order // 2


def coef_vector(order: int, compute_dtype=np.float32) -> np.ndarray:
    """getFD_D2coefVector (src/fdm.h:690-741): outermost-first A_R..A0..A_R,
    each value rounded to the compute type (Myfloat2)."""
    check_order(order)
    c = D2_COEF[order]
    v = list(reversed(c[1:])) + [c[0]] + list(c[1:])
    return np.array(v, dtype=compute_dtype)


def sum_abs_coef(order: int, compute_dtype=np.float32) -> float:
    """getSumAbsFD_D2Coef (src/fdm.h:743-756): FP64 sum of |coef| where each
    coefficient is first rounded to the compute type."""
    s = 0.0
    for c in coef_vector(order, compute_dtype):
        s += abs(float(c))
    return s


def sum_coef(order: int, compute_dtype=np.float32) -> float:
    """getSumFD_D2Coef (src/fdm.h:789-800): expected to be ~0."""
    s = 0.0
    for c in coef_vector(order, compute_dtype):
        s += float(c)
    return s


def flop_per_pt_d2(order: int) -> int:
    return D2_NOP[order]


def flop_per_pt_laplacian(order: int, dim: int) -> int:
    """Grid::getFlopPerPtFD_LAPLACIAN (src/grid.cpp:2408-2424)."""
    n = D2_NOP[order]
    return {1: n, 2: 2 * n + 1, 3: 3 * n + 2}[dim]


def pt_per_stencil_laplacian(order: int, dim: int) -> int:
    """Grid::getPtPerStencilFD_LAPLACIAN."""
    h = order // 2
    return {1: 2 * h + 1, 2: 4 * h + 1, 3: 6 * h + 1}[dim]


def cfl(order: int, dim: int, compute_dtype=np.float32) -> float:
    """Propagator_Ac2::getCFL (src/propagator_Ac2.cpp:410-439):
    sqrt(sum|A_O2| / (dim * sum|A_order|)), returned as Myfloat."""
    a1 = sum_abs_coef(2, compute_dtype)
    a2 = sum_abs_coef(order, compute_dtype) * dim
    return float(np.dtype(compute_dtype).type(math.sqrt(a1 / a2)))
