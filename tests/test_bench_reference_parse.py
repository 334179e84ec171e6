"""The bench's reference runners (CPU): the command lines they build and how they read the
reference's own timers and verdict, against a stand-in executable that prints the reference's
report lines (no reference build, no GPU)."""
import os
import stat

import pytest

import bench
from oracle import oracle

REPORT = """ Check at time\t0
 Bound. cond. time (s)\t0.0190412
 Compute pres. time (s)\t0.238038
 Best Gpoint/s in FD\t112.77
 errTestCase2\t4.21244e-05
 Test PASSED
"""


@pytest.fixture
def fake_ref(tmp_path, monkeypatch):
    args_file = tmp_path / "args.txt"
    exe = tmp_path / "hpcscan_fake"
    exe.write_text("#!/bin/sh\n"
                   f"echo \"$@\" > {args_file}\n"
                   f"cat <<'EOF'\n{REPORT}EOF\n")
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    monkeypatch.setattr(oracle, "ref_binary", lambda prec: str(exe))
    monkeypatch.setattr(oracle, "ref_gpu_binary", lambda: str(exe))
    return args_file


def test_cpu_runner_reads_the_reference_timers(fake_ref):
    v, det = bench.run_reference_cpu(512, 8, 200, 4)
    assert v == pytest.approx(512 ** 3 * 200 / (0.0190412 + 0.238038) / 1e9)
    assert det["passed"] and det["err_test_case"] == pytest.approx(4.21244e-05)
    args = fake_ref.read_text().split()
    assert args[args.index("-testMode") + 1] == "CacheBlk"
    assert args[args.index("-nt") + 1] == "200" and args[args.index("-snapInc") + 1] == "100"


def test_gpu_runner_passes_block_sizes(fake_ref):
    v, det = bench.run_reference_gpu(512, 8, 200, "CUDA_Opt", (64, 8, 32))
    assert det["mode"] == "CUDA_Opt" and det["passed"]
    args = fake_ref.read_text().split()
    assert args[args.index("-testMode") + 1] == "CUDA_Opt"
    assert [args[args.index(f"-cb{i}") + 1] for i in (1, 2, 3)] == ["64", "8", "32"]


def test_missing_timers_are_an_error(tmp_path, monkeypatch):
    exe = tmp_path / "hpcscan_silent"
    exe.write_text("#!/bin/sh\necho nothing\n")
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    monkeypatch.setattr(oracle, "ref_gpu_binary", lambda: str(exe))
    with pytest.raises(RuntimeError):
        bench.run_reference_gpu(64, 8, 10, "CUDA", None)


def test_missing_binary(monkeypatch, tmp_path):
    monkeypatch.setattr(oracle, "ref_gpu_binary", lambda: os.path.join(str(tmp_path), "absent"))
    with pytest.raises(FileNotFoundError):
        bench.run_reference_gpu(64, 8, 10, "CUDA", None)


def test_reference_gpu_arm_reports_unavailable(monkeypatch, tmp_path, capsys):
    import json
    import types
    monkeypatch.setattr(oracle, "ref_gpu_binary", lambda: os.path.join(str(tmp_path), "absent"))
    bench.reference_gpu_arm(types.SimpleNamespace(steps=10, size=64, order=8))
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference-gpu" and "unavailable" in line
    assert len(line["runs"]) == 4 and all("failed" in r for r in line["runs"])


def test_reference_gpu_arm_picks_the_fastest(fake_ref, capsys):
    import json
    import types
    bench.reference_gpu_arm(types.SimpleNamespace(steps=200, size=512, order=8))
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference-gpu" and line["metric"] == bench.METRIC
    assert line["value"] == max(r["value"] for r in line["runs"])
    assert line["config"]["test_mode"].startswith("CUDA_Opt")      # first of equal times
