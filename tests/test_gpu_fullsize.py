"""Parity at the benchmark's full size (512^3 inner points, O8, FP32 and FP64): the time step
of the bench (boundary condition + pressure update) on the GPU against the C oracle, bit for
bit over every point of the array, and properties that hold at any size (power-of-two scaling,
which every separately rounded operation carries exactly) at 1000^3.

The oracle runs on the host cores (OpenMP); one step at 512^3 takes it a few seconds."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from hpcscan_b200 import layout as L  # noqa: E402


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hpcscan_b200.grid import init_device
    init_device(0)
    return torch


def raw_bits(a):
    return a.view({4: np.uint32, 8: np.uint64}[a.dtype.itemsize])


@pytest.mark.parametrize("prec,nsteps", [("f32", 2), ("f64", 1)])
def test_bench_step_512_bitexact(gpu, oracle, prec, nsteps):
    """The bench workload itself: eigen mode (1, 1, 1), ratioCFL 0.8, 512^3, O8; nsteps steps of
    applyBoundaryCondition + computePressureWithFD with the swap, on the GPU and in the oracle."""
    from hpcscan_b200.propagator import Propagator_Ac2
    lay = L.b200_layout(3, 512, 512, 512, order=8, prec=prec)
    p = Propagator_Ac2(lay)
    p.initialize(ratio_cfl=0.8, nt=nsteps, snap_inc=nsteps, modes=(1, 1, 1))
    prn, prc, coef = p.prnGrid.to_numpy(), p.prcGrid.to_numpy(), p.coefGrid.to_numpy()
    inv2 = L.inv2_spacing(p.setup.samp, prec)
    g_prn, g_prc = p.prnGrid, p.prcGrid
    for _ in range(nsteps):
        p.computeWavefieldNextTimeStep(g_prn, g_prc)
        oracle.apply_bc(lay, prc)
        oracle.compute_pressure(lay, prn, prc, coef, inv2)
        g_prn, g_prc = g_prc, g_prn
        prn, prc = prc, prn
    gpu.cuda.synchronize()
    # every inner point (the halo points of a grid whose boundary condition the library built
    # inside the fused step's tiles keep their earlier values, which no later read uses)
    for got, want in ((g_prc.to_numpy(), prc), (g_prn.to_numpy(), prn)):
        got, want = lay.inner(got), lay.inner(want)
        same = raw_bits(got) == raw_bits(want)
        assert same.all(), (int((~same).sum()), float(np.abs(got - want).max()))


def _sub_block(lay, big_flat, corner, m):
    """The values of the big grid around an m^3 block of its inner points (inner corner
    (i1, i2, i3)), laid out as a small grid of the same order: its inner points are the block,
    its halos the big grid's values next to the block."""
    small = L.b200_layout(3, m, m, m, order=lay.order, prec=lay.prec)
    R = lay.halo
    big = big_flat.view(lay.n3, lay.n2, lay.n1)
    x0 = lay.a1.inner_start + corner[0] - R
    y0 = lay.a2.inner_start + corner[1] - R
    z0 = lay.a3.inner_start + corner[2] - R
    blk = big[z0:z0 + m + 2 * R, y0:y0 + m + 2 * R, x0:x0 + m + 2 * R].cpu().numpy()
    out = np.zeros((small.n3, small.n2, small.n1), dtype=blk.dtype)
    s1, s2, s3 = small.a1.inner_start - R, small.a2.inner_start - R, small.a3.inner_start - R
    out[s3:s3 + m + 2 * R, s2:s2 + m + 2 * R, s1:s1 + m + 2 * R] = blk
    return small, out.reshape(-1)


@pytest.mark.parametrize("order", [12, 16])
def test_pressure_1000_blocks_bitexact(gpu, oracle, order):
    """At 1000^3 (the mixed-precision configuration's size), O12 and O16, FP32: the pressure
    update on the GPU, bit for bit against the oracle on blocks of the grid (each block's
    update depends only on the values within R of it): a corner block touching three
    boundaries, an edge block, a block in the middle, and a block astride tile and z-chunk
    seams."""
    torch = gpu
    from hpcscan_b200.grid import Grid
    lay = L.b200_layout(3, 1000, 1000, 1000, order=order, prec="f32")
    samp = L.Sampling((0.002, 0.002, 0.002), (0.0, 0.0, 0.0))
    g = torch.Generator(device="cuda").manual_seed(9)
    prn, prc, coef = (Grid(lay, samp) for _ in range(3))
    for G in (prn, prc, coef):
        G.initializeGrid()
    prc.data.uniform_(-1.0, 1.0, generator=g)
    prn.data.uniform_(-1.0, 1.0, generator=g)
    coef.data.uniform_(0.0, 1e-3, generator=g)
    before = {"prn": prn.data.clone()}
    assert prn.computePressureWithFD(prc, coef, order) == 0
    torch.cuda.synchronize()
    inv2 = L.inv2_spacing(samp, "f32")
    m = 40
    for corner in ((0, 0, 0), (1000 - m, 500, 0), (480, 480, 480), (60, 10, 120)):
        small, u = _sub_block(lay, prc.data, corner, m)
        _, p_old = _sub_block(lay, before["prn"], corner, m)
        _, c = _sub_block(lay, coef.data, corner, m)
        _, got = _sub_block(lay, prn.data, corner, m)
        oracle.compute_pressure(small, p_old, u, c, inv2)
        a, b = small.inner(got), small.inner(p_old)
        same = raw_bits(a) == raw_bits(b)
        assert same.all(), (corner, int((~same).sum()), float(np.abs(a - b).max()))
    del prn, prc, coef, before
    torch.cuda.empty_cache()


def test_power_of_two_scaling_1000(gpu):
    """At 1000^3 O12 FP32 (the mixed-precision configuration's size): the pressure update of
    4 prc, 4 prn equals 4 times the update of prc, prn bit for bit, and FD_D1 / FD_D2 of 4 u
    equal 4 times those of u (scaling by a power of two is exact in every operation)."""
    torch = gpu
    from hpcscan_b200.grid import Grid
    lay = L.b200_layout(3, 1000, 1000, 1000, order=12, prec="f32")
    samp = L.Sampling((0.002, 0.002, 0.002), (0.0, 0.0, 0.0))
    g = torch.Generator(device="cuda").manual_seed(5)
    grids = []
    for _ in range(4):
        G = Grid(lay, samp)
        G.initializeGrid()
        grids.append(G)
    prn, prc, coef, out = grids
    prc.data.uniform_(-1.0, 1.0, generator=g)
    prn.data.uniform_(-1.0, 1.0, generator=g)
    coef.data.uniform_(0.0, 1e-3, generator=g)
    ref = prn.data.clone()
    prn.computePressureWithFD(prc, coef, lay.order)
    once = prn.data.clone()
    prn.data.copy_(ref * 4)
    prc.data.mul_(4)
    prn.computePressureWithFD(prc, coef, lay.order)
    assert torch.equal(prn.data, once * 4)
    del ref, once
    for op in ("FD_D1_N1", "FD_D1_N3", "FD_D2_N2"):
        getattr(prc, op)(L.INNER_POINTS, out, lay.order)
        a = out.data.clone()
        prc.data.mul_(0.25)
        getattr(prc, op)(L.INNER_POINTS, out, lay.order)
        assert torch.equal(out.data * 4, a), op
        prc.data.mul_(4)
        del a
    del grids, prn, prc, coef, out
    torch.cuda.empty_cache()
