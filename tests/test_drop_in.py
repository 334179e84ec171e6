"""hpcscan's own test cases, unchanged, on -testMode B200.

hpcscan_b200/host/bin/hpcscan_b200_fp{32,64} are hpcscan's drivers (main, test cases,
propagators, factories, the Grid base class) compiled from the hpcscan sources with Grid_B200
registered in the factories. The same test case on the reference CPU build (oracle/_ref, modes
Baseline / CacheBlk) is the yardstick: every "Test PASSED / ... err." line and the Propa
errTestCase must agree.

CPU tests check that the wrapped factories leave the CPU modes untouched; GPU tests run B200.
"""
import os
import re
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
B200_BIN = {p: os.path.join(REPO, "hpcscan_b200", "host", "bin", f"hpcscan_b200_{p}")
            for p in ("fp32", "fp64")}
REF_BIN = {p: os.path.join(REPO, "oracle", "_ref", f"hpcscan_{p}") for p in ("fp32", "fp64")}

RESULT = re.compile(r"Test (PASSED|FAILED)!? / (\w+) err\.\s+(\S+)")
PROPA_ERR = re.compile(r"errTestCase2\s+(\S+)")


def run(binary, args, tmp_path):
    if not os.path.exists(binary):
        pytest.skip(f"{os.path.relpath(binary, REPO)} not built")
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "4"))
    p = subprocess.run([binary] + args, cwd=tmp_path, capture_output=True, text=True, timeout=900,
                       env=env)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    assert "TERMINATED SUCCESSFULLY" in p.stdout, p.stdout[-3000:]
    assert "No test case was executed" not in p.stdout, p.stdout[-3000:]
    return p.stdout


def results(out):
    return [(s, k, float(v)) for s, k, v in RESULT.findall(out)]


def propa_err(out):
    m = PROPA_ERR.findall(out)
    assert m and "Test PASSED" in out, out[-3000:]
    return float(m[-1])


def same_results(got, want, rtol, atol):
    assert len(got) == len(want) > 0, (got, want)
    for (sg, kg, vg), (sw, kw, vw) in zip(got, want):
        assert (sg, kg) == (sw, kw), (got, want)
        assert abs(vg - vw) <= atol + rtol * abs(vw), (kg, vg, vw)


GRID_ARGS = ["-n1", "40", "-n2", "40", "-n3", "40", "-ntry", "1"]


# ---- CPU: the factory wrapping leaves the hpcscan CPU modes as they are ------------------------

@pytest.mark.parametrize("case", ["Grid", "FD_D2", "FD_D1", "Propa"])
def test_cpu_modes_unchanged_by_b200_registration(tmp_path, case):
    args = ["-testCase", case, "-testMode", "CacheBlk"] + GRID_ARGS
    got = run(B200_BIN["fp32"], args, tmp_path)
    want = run(REF_BIN["fp32"], args, tmp_path)
    if case == "Propa":
        assert propa_err(got) == propa_err(want)
    else:
        assert results(got) == results(want)


# ---- GPU: the unchanged test cases on the B200 path ---------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("prec,order,propagator", [
    ("fp32", 8, "Ac2Standard"), ("fp32", 2, "Ac2Standard"), ("fp32", 16, "Ac2Standard"),
    ("fp32", 8, "Ac2SplitComp"), ("fp64", 8, "Ac2Standard"), ("fp64", 12, "Ac2SplitComp")])
def test_propa_b200_equals_reference(tmp_path, prec, order, propagator):
    """Eigen-mode propagation (TestCase_Propa) with the reference's check every step: the
    errTestCase of B200 equals the reference CPU build's (wavefields are bit-identical; only the
    FP64 summation order of the norms differs)."""
    args = ["-testCase", "Propa", "-propagator", propagator, "-fdOrder", str(order),
            "-n1", "70", "-n2", "61", "-n3", "53", "-ratioCFL", "0.8", "-nt", "60", "-ntry", "1"]
    got = propa_err(run(B200_BIN[prec], args + ["-testMode", "B200"], tmp_path))
    want = propa_err(run(REF_BIN[prec], args + ["-testMode", "Baseline"], tmp_path))
    assert abs(got - want) <= 1e-5 * abs(want), (got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("fused", ["1", "0"])
@pytest.mark.parametrize("prec,order", [("fp32", 8), ("fp32", 16), ("fp64", 4)])
def test_propa_fused_propagator_equals_reference(tmp_path, monkeypatch, fused, prec, order):
    """-propagator Ac2Fused (registered for -testMode B200): the boundary condition deferred by
    the grids and built inside the pressure kernel's tiles (HPCSCAN_B200_FUSED_STEP=1) or run as
    its own kernel in the same library call (0); errTestCase equal to the reference CPU build's
    Ac2Standard, the analytic check every step."""
    monkeypatch.setenv("HPCSCAN_B200_FUSED_STEP", fused)
    args = ["-testCase", "Propa", "-fdOrder", str(order), "-n1", "70", "-n2", "61", "-n3", "53",
            "-ratioCFL", "0.8", "-nt", "60", "-ntry", "1"]
    out = run(B200_BIN[prec], args + ["-testMode", "B200", "-propagator", "Ac2Fused"], tmp_path)
    assert "Boundary condition fused" in out
    got = propa_err(out)
    want = propa_err(run(REF_BIN[prec], args + ["-testMode", "Baseline", "-propagator",
                                                "Ac2Standard"], tmp_path))
    assert abs(got - want) <= 1e-5 * abs(want), (got, want)


@pytest.mark.gpu
def test_modeling_fused_propagator_traces_equal_reference(tmp_path, monkeypatch):
    """TestCase_Modeling with -propagator Ac2Fused on B200 (fused kernel forced): the traces of
    the reference CPU build's Ac2Standard (FP32, 1e-6 relative)."""
    import numpy as np
    monkeypatch.setenv("HPCSCAN_B200_FUSED_STEP", "1")
    n = (48, 40, 44)
    rng = np.random.default_rng(8)
    vel = (2000.0 + 400.0 * np.tanh(rng.standard_normal((n[2], n[1], n[0])))).astype(np.float32)
    runs = {}
    for mode, binary, propa in (("B200", B200_BIN["fp32"], "Ac2Fused"),
                                ("Baseline", REF_BIN["fp32"], "Ac2Standard")):
        d = tmp_path / mode
        d.mkdir()
        vel.tofile(d / "vp.bin")
        args = ["-testCase", "Modeling", "-testMode", mode, "-propagator", propa,
                "-n1", str(n[0]), "-n2", str(n[1]), "-n3", str(n[2]), "-modelVpFile", "vp.bin",
                "-nt", "160", "-ntry", "1"]
        run(binary, args, d)
        runs[mode] = np.fromfile(d / "ModelingForwardPrn.trace.bin", dtype=np.float32)
    got, want = runs["B200"], runs["Baseline"]
    assert got.shape == want.shape and np.abs(want).max() > 0
    assert np.abs(got - want).max() / np.abs(want).max() <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("order", [2, 4, 6, 8, 10, 12, 14, 16])
def test_fd_d2_b200_equals_reference(tmp_path, prec, order):
    """TestCase_FD_D2: D2 along each axis and the Laplacian of sin(a1 x1) sin(a2 x2) sin(a3 x3)
    against the analytic derivatives; the same L1 errors and verdicts as the reference CPU
    build (at this size O2 misses the 1e-3 threshold on both)."""
    args = ["-testCase", "FD_D2", "-fdOrder", str(order), "-n1", "50", "-n2", "44", "-n3", "38",
            "-param1", "4", "-param2", "6", "-param3", "8", "-param4", "1", "-ntry", "1"]
    got = results(run(B200_BIN[prec], args + ["-testMode", "B200"], tmp_path))
    want = results(run(REF_BIN[prec], args + ["-testMode", "Baseline"], tmp_path))
    same_results(got, want, rtol=1e-5, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("order,dim", [(2, 3), (4, 3), (8, 3), (12, 3), (16, 3), (6, 2), (10, 1)])
def test_fd_d1_b200_equals_reference(tmp_path, prec, order, dim):
    """TestCase_FD_D1: the staggered first derivative along each axis against the analytic
    derivative on the grid shifted by half a cell; the same L1 errors and verdicts as the
    reference CPU build."""
    args = ["-testCase", "FD_D1", "-dim", str(dim), "-fdOrder", str(order), "-n1", "50",
            "-n2", "44", "-n3", "38", "-param1", "3", "-param2", "5", "-param3", "7", "-ntry", "1"]
    got = results(run(B200_BIN[prec], args + ["-testMode", "B200"], tmp_path))
    want = results(run(REF_BIN[prec], args + ["-testMode", "Baseline"], tmp_path))
    assert len(got) == dim
    same_results(got, want, rtol=1e-5, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["Grid", "Memory"])
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_grid_and_memory_cases_pass_on_b200(tmp_path, case, prec):
    """TestCase_Grid (fill, norms, min/max, updatePressure, boundary condition) and
    TestCase_Memory (whole-array operations): every check passes on B200, with the reference's
    tolerance, and reports what the reference CPU build reports."""
    args = ["-testCase", case] + GRID_ARGS
    got = results(run(B200_BIN[prec], args + ["-testMode", "B200"], tmp_path))
    want = results(run(REF_BIN[prec], args + ["-testMode", "Baseline"], tmp_path))
    same_results(got, want, rtol=1e-4, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("boundary", ["FreeSurf", "None"])
def test_modeling_b200_traces_equal_reference(tmp_path, prec, boundary):
    """TestCase_Modeling (velocity read from file, Ricker source one point below the top,
    receiver plane): the B200 traces (source and receivers on the device, DataAcquisition_B200)
    equal those of the reference CPU build."""
    import numpy as np
    n = (48, 40, 44)
    t = np.float32 if prec == "fp32" else np.float64
    rng = np.random.default_rng(7)
    vel = (2000.0 + 400.0 * np.tanh(rng.standard_normal((n[2], n[1], n[0])))).astype(t)
    runs = {}
    for mode, binary in (("B200", B200_BIN[prec]), ("Baseline", REF_BIN[prec])):
        d = tmp_path / mode
        d.mkdir()
        vel.tofile(d / "vp.bin")
        args = ["-testCase", "Modeling", "-testMode", mode, "-n1", str(n[0]), "-n2", str(n[1]),
                "-n3", str(n[2]), "-modelVpFile", "vp.bin", "-nt", "160", "-boundary", boundary,
                "-ntry", "1"]
        run(binary, args, d)
        runs[mode] = np.fromfile(d / "ModelingForwardPrn.trace.bin", dtype=t)
    got, want = runs["B200"], runs["Baseline"]
    assert got.shape == want.shape and np.abs(want).max() > 0
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err <= (1e-6 if prec == "fp32" else 1e-13), err


# ---- the stated sizes of the benchmarked configurations ----------------------------------------

@pytest.mark.gpu
def test_propa_config_200_cubed_one_period_equals_reference(tmp_path):
    """The plain Propa configuration at its stated size: Ac2Standard, O8, FP32, 200^3 inner
    points of the unit cube, ratioCFL 0.8, one period of the (1, 1, 1) eigen mode (tmax =
    2 / sqrt(3), 635 time steps), the analytic check every step. The B200 errTestCase equals the
    reference CPU build's (the CacheBlk mode, the reference's optimised CPU path) within 1e-5
    relative; both pass the reference's own 2e-2 bar (src/testCase_Propa.cpp:91)."""
    args = ["-testCase", "Propa", "-propagator", "Ac2Standard", "-fdOrder", "8",
            "-n1", "200", "-n2", "200", "-n3", "200", "-ratioCFL", "0.8", "-tmax", "1.1547005",
            "-ntry", "1"]
    out_b200 = run(B200_BIN["fp32"], args + ["-testMode", "B200"], tmp_path)
    out_ref = run(REF_BIN["fp32"], args + ["-testMode", "CacheBlk"], tmp_path)
    got, want = propa_err(out_b200), propa_err(out_ref)
    for out in (out_b200, out_ref):
        assert re.findall(r"No\. time steps\s+(\d+)", out)[-1] == "635", out[-3000:]
    assert abs(got - want) <= 1e-5 * abs(want), (got, want)
    assert 3.0e-4 < got < 4.5e-4, got          # the reference's 3.737e-4 at this configuration


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("order", [2, 4, 8, 12, 16])
def test_fd_d2_sweep_128_cubed_equals_reference(tmp_path, prec, order):
    """The FD_D2 sweep's smallest cube (128^3, u = sin(4 pi x1) sin(6 pi x2) sin(8 pi x3)) for
    every order of the sweep: the same four L1 errors against the analytic derivatives and the
    same verdicts as the reference CPU build (src/testCase_FD_D2.cpp:65-74)."""
    args = ["-testCase", "FD_D2", "-fdOrder", str(order), "-n1", "128", "-n2", "128",
            "-n3", "128", "-param1", "4", "-param2", "6", "-param3", "8", "-param4", "1",
            "-ntry", "1"]
    got = results(run(B200_BIN[prec], args + ["-testMode", "B200"], tmp_path))
    want = results(run(REF_BIN[prec], args + ["-testMode", "CacheBlk"], tmp_path))
    assert len(got) == 4
    same_results(got, want, rtol=1e-5, atol=1e-12)
