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
    for got, want in ((g_prc.to_numpy(), prc), (g_prn.to_numpy(), prn)):
        same = raw_bits(got) == raw_bits(want)
        assert same.all(), (int((~same).sum()), float(np.abs(got - want).max()))


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
