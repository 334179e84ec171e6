"""Benchmark of the hpcscan B200 hot path: the Propa acoustic propagator step.

Workload (the headline configuration): Propa Ac2Standard, FD order 8, FP32,
n1 = n2 = n3 = 512 inner points (520^3 with halos), eigen mode (1, 1, 1), ratioCFL 0.8.
A step is one time step of Propagator_Ac2::computeWavefieldNextTimeStep:
applyBoundaryCondition(prc) then computePressureWithFD(prn, prc), then the swap.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--size 512]

One JSON line on stdout (rank 0). Under torchrun every rank runs its own replica of the
workload on its GPU (the propagator does not shard on one grid: "replicas only"), the
device time is the max over ranks, and value = all points updated / that time.

  value          GPoint/s with the grids resident in HBM (device time, CUDA events)
  e2e            GPoint/s of one whole Propa job through the Python Grid/propagator API:
                 host eigen-mode fields (pinned) -> device, nt time steps with the
                 reference's periodic analytic checks, final wavefield -> host
  roofline       the fused pressure kernel: 16 algorithmic bytes per inner point
                 (prc, prn, coef read once, prn written once) / its mean launch time,
                 against the measured HBM copy bandwidth
  cpu_baseline   the reference CPU path itself (oracle/_ref/hpcscan_fp32, test mode
                 CacheBlk, all host threads) on a bounded number of steps of the same grid
--impl reference prints the same line for the reference CPU implementation; --impl
reference-gpu for the reference's own CUDA modes (built unchanged for sm_100a) on this GPU, a
comparison only.

The other workloads (--workload) print their own line: adjoint and modeling split their
fixed survey of shots over the ranks under torchrun (one GPU per rank, the adjoint's survey
gradient summed by one all-reduce); mixed, fd and sustained run on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

METRIC = "Propa GPoint/s (O8 FP32 acoustic leapfrog step, 512^3)"
UNIT = "GPoint/s"
ALG_BYTES_PER_POINT = 16     # FP32: read prc, prn, coef; write prn (computePressureWithFD)
KERNEL_NAME = "k_zmarch (computePressureWithFD, TMA z-marching)"
KERNEL_STEP_NAME = ("k_zmarch MODE_STEP (boundary condition built in the tiles of "
                    "computePressureWithFD) + k_bc_planes")


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference", "reference-gpu"],
                   help="b200 (this library), reference (the reference CPU path, the baseline) "
                        "or reference-gpu (the reference's own CUDA modes on this GPU)")
    p.add_argument("--size", type=int, default=None,
                   help="inner points per axis (default 512; the adjoint workload 256)")
    p.add_argument("--order", type=int, default=8)
    p.add_argument("--e2e-steps", type=int, default=0,
                   help="time steps of the end-to-end job (default: one period of the mode)")
    p.add_argument("--cpu-steps", type=int, default=200,
                   help="time steps of the bounded reference CPU sample")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--workload", default="propa",
                   choices=["propa", "adjoint", "modeling", "mixed", "fd", "fdsweep", "dropin",
                            "launches", "sustained"],
                   help="propa (default, the headline), adjoint (batched checkpointed gradients), "
                        "modeling (batched uneven forward shots), mixed (16-bit wavefields), "
                        "fd (the FD_D1 / FD_D2 operator test cases), fdsweep (the FD_D2 test "
                        "case over orders, cubes and precisions), dropin (hpcscan's own Propa "
                        "driver on -testMode B200), launches (one launch of each hot kernel, for "
                        "a profiler) or sustained (the headline step back to back for --nt "
                        "steps, with clocks and power per bin)")
    p.add_argument("--shots", type=int, default=0, help="shots (adjoint: 16, modeling: 64)")
    p.add_argument("--nt", type=int, default=0, help="time steps (adjoint: 2000, modeling: 1500)")
    p.add_argument("--checkpoint", type=int, default=45, help="adjoint checkpoint interval")
    p.add_argument("--sizes", default="", help="fdsweep: cubes, comma-separated (128,256,512,800)")
    p.add_argument("--orders", default="", help="fdsweep: orders, comma-separated (2,4,8,12,16)")
    p.add_argument("--snap", type=int, default=0, help="dropin: steps between analytic checks (50)")
    p.add_argument("--propagator", default="Ac2Standard",
                   help="dropin: hpcscan propagator (Ac2Standard, Ac2SplitComp, Ac2Fused)")
    p.add_argument("--survey", type=int, default=1,
                   help="adjoint: 1 = the batch accumulates the survey gradient in one pass per step "
                        "(b200_batch_survey_gradient), 0 = each shot's gradient by its own stencil "
                        "pass, summed after")
    a = p.parse_args()
    if a.size is None:
        a.size = 256 if a.workload == "adjoint" else 512
    return a


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), \
        int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(dist, values, device):
    """Per-rank timings -> their maxima over all ranks (one all-reduce that every rank takes);
    the values themselves on a single process."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def job_gpoints(world, points_per_rank, steps, seconds):
    """Whole-job throughput of `world` replicas, each updating points_per_rank x steps."""
    return world * points_per_rank * steps / seconds / 1e9


def measured_peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, copy)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s"


def profiled_traffic():
    """DRAM bytes per launch of the pressure kernel from the committed ncu summary."""
    path = os.path.join(REPO, "profiles", "zmarch_pressure_o8_f32_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d
    except Exception:
        return None


class ClockSampler:
    """SM clock and throttle reasons sampled in-process through NVML every 20 ms; start it
    before the warm-up so that no NVML start-up falls into the timed region, and mark the
    timed region with begin()/end()."""
    PERIOD_S = 0.02

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []          # (t, sm_mhz, reasons bitmask, power_w)
        self.window = None
        self.ok = False
        self.stop_ev = threading.Event()

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
            time.sleep(0.2)
        except Exception:
            self.ok = False
        return self

    def _run(self):
        nv = self.nv
        while not self.stop_ev.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                self.samples.append((time.perf_counter(), sm, rs, pw))
            except Exception:
                pass
            time.sleep(self.PERIOD_S)

    def begin(self):
        self.t0 = time.perf_counter()

    def end(self):
        self.window = (self.t0, time.perf_counter())
        time.sleep(self.PERIOD_S * 2)

    def __exit__(self, *a):
        self.stop_ev.set()

    def _reasons(self, sel):
        nv = self.nv
        names = {"hw_slowdown": getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
                 "hw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
                 "sw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
                 "sw_power_cap": getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4)}
        return sorted({n for x in sel for n, bit in names.items() if x[2] & bit})

    def summary(self):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        t0, t1 = self.window
        sel = [x for x in self.samples if t0 - self.PERIOD_S <= x[0] <= t1 + self.PERIOD_S]
        if not sel:
            sel = self.samples[-3:]
        return {"sm_mhz": statistics.median([x[1] for x in sel]), "sm_max_mhz": self.max_mhz,
                "reasons": self._reasons(sel), "samples": len(sel)}

    def between(self, t0, t1):
        """Median SM clock, mean board power (NVML's own running average) and the reasons
        seen in the samples taken between host times t0 and t1."""
        sel = [x for x in self.samples if t0 <= x[0] <= t1] if self.ok else []
        if not sel:
            return {"sm_mhz": None, "power_w": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median([x[1] for x in sel]),
                "power_w": round(statistics.mean([x[3] for x in sel]), 1),
                "reasons": self._reasons(sel), "samples": len(sel)}


# ---- reference CPU path -------------------------------------------------------------------------

def run_reference_cpu(n: int, order: int, nt: int, threads: int):
    """Run the reference Propa test case (CacheBlk) for nt steps and return its own
    timers: (GPoint/s over BC + pressure time, details)."""
    from oracle import oracle
    exe = oracle.ref_binary("f32")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    args = [exe, "-testCase", "Propa", "-testMode", "CacheBlk", "-propagator", "Ac2Standard",
            "-fdOrder", str(order), "-n1", str(n), "-n2", str(n), "-n3", str(n),
            "-ratioCFL", "0.8", "-param1", "1", "-param2", "1", "-param3", "1",
            "-nt", str(nt), "-snapInc", str(max(1, nt // 2)), "-ntry", "1"]
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close")
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        out = subprocess.run(args, cwd=d, capture_output=True, text=True, env=env, timeout=900)
        wall = time.perf_counter() - t0
    if out.returncode != 0:
        raise RuntimeError(out.stdout[-2000:] + out.stderr[-2000:])
    txt = out.stdout

    def grab(pat):
        m = re.search(pat + r"\s+(\S+)", txt)
        return float(m.group(1)) if m else None
    t_bc = grab(r"Bound\. cond\. time \(s\)")
    t_p = grab(r"Compute pres\. time \(s\)")
    pts = float(n) ** 3 * nt
    value = pts / (t_bc + t_p) / 1e9
    return value, {"bc_s": t_bc, "pressure_s": t_p, "gpoint_fd": grab(r"Best Gpoint/s in FD"),
                   "wall_s": wall, "nt": nt, "passed": "Test PASSED" in txt,
                   "err_test_case": grab(r"errTestCase2")}


def run_reference_gpu(n: int, order: int, nt: int, mode: str, cb=None):
    """Run the reference Propa test case in one of its own GPU test modes (CUDA, CUDA_Opt), built
    unchanged from its sources for sm_100a, and return its own timers like run_reference_cpu.
    cb: the reference's block sizes (-cb1, -cb2, -cb3), which size CUDA_Opt's tiles."""
    from oracle import oracle
    exe = oracle.ref_gpu_binary()
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    args = [exe, "-testCase", "Propa", "-testMode", mode, "-propagator", "Ac2Standard",
            "-fdOrder", str(order), "-n1", str(n), "-n2", str(n), "-n3", str(n),
            "-ratioCFL", "0.8", "-param1", "1", "-param2", "1", "-param3", "1",
            "-nt", str(nt), "-snapInc", str(max(1, nt // 2)), "-ntry", "1"]
    if cb is not None:
        args += ["-cb1", str(cb[0]), "-cb2", str(cb[1]), "-cb3", str(cb[2])]
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        out = subprocess.run(args, cwd=d, capture_output=True, text=True, timeout=600)
        wall = time.perf_counter() - t0
    if out.returncode != 0:
        raise RuntimeError((out.stdout[-1500:] + out.stderr[-1500:]).strip())
    txt = out.stdout

    def grab(pat):
        m = re.search(pat + r"\s+(\S+)", txt)
        return float(m.group(1)) if m else None
    t_bc = grab(r"Bound\. cond\. time \(s\)")
    t_p = grab(r"Compute pres\. time \(s\)")
    if t_bc is None or t_p is None:
        raise RuntimeError("no timers in the reference's output: " + txt[-800:])
    return n ** 3 * nt / (t_bc + t_p) / 1e9, {
        "mode": mode, "cb": cb, "bc_s": t_bc, "pressure_s": t_p,
        "gpoint_fd": grab(r"Best Gpoint/s in FD"), "wall_s": round(wall, 2), "nt": nt,
        "passed": "Test PASSED" in txt, "err_test_case": grab(r"errTestCase2")}


def reference_gpu_arm(a):
    """The reference's own GPU path on this GPU: its CUDA_Opt mode (2.5-D shared-memory tiles with
    a register z-queue, one kernel per order) at its default block sizes and at two larger ones,
    and its plain CUDA mode; the line reports the fastest, every run in `runs`. Not the driver's
    reference arm (the reference CPU path, --impl reference): a comparison on the same GPU."""
    rank, world, _ = dist_env()
    if world > 1 and rank != 0:
        return
    nt = max(a.steps, 1)
    runs, best = [], None
    for mode, cb in (("CUDA_Opt", None), ("CUDA_Opt", (64, 16, 64)), ("CUDA_Opt", (64, 8, 32)),
                     ("CUDA", None)):
        try:
            v, det = run_reference_gpu(a.size, a.order, nt, mode, cb)
            runs.append({"value": round(v, 4), **det})
            if best is None or v > best[0]:
                best = (v, det)
        except Exception as e:
            runs.append({"mode": mode, "cb": cb, "failed": str(e)[:300]})
    if best is None:
        print(json.dumps({"impl": "reference-gpu", "unavailable": "the reference's CUDA modes "
                          "did not run", "runs": runs}))
        return
    v, det = best
    print(json.dumps({
        "impl": "reference-gpu", "metric": METRIC, "value": round(v, 4), "unit": UNIT,
        "n_gpus": 1, "steps": nt, "warmup": 0,
        "ms_per_step": round((det["bc_s"] + det["pressure_s"]) / nt * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (eigen mode, the reference's own Propa initialisation)",
        "config": {"workload": f"Propa Ac2Standard O{a.order} FP32 {a.size}^3 eigen mode",
                   "n": a.size, "order": a.order, "ratio_cfl": 0.8,
                   "test_mode": f"{det['mode']} (reference GPU path, unchanged source, sm_100a)",
                   "timers": "the reference's own boundary-condition + compute-pressure timers "
                             "(each call ends with a device synchronisation)"},
        "runs": runs}))


def propa_config(a, layout_n1, l2, tuning, parallelism):
    """The config object of the Propa lines, the same keys for this library's arm and the
    reference arm."""
    return {"workload": f"Propa Ac2Standard O{a.order} FP32 {a.size}^3 eigen mode "
                        "(boundary condition + pressure update per step)",
            "n": a.size, "order": a.order, "ratio_cfl": 0.8, "layout_n1": layout_n1, "l2": l2,
            "tuning": tuning, "parallelism": parallelism}


def reference_arm(a):
    rank, world, _ = dist_env()
    if world > 1 and rank != 0:
        return
    threads = os.cpu_count() or 1
    nt = max(a.steps, 1)
    try:
        value, det = run_reference_cpu(a.size, a.order, nt, threads)
    except Exception as e:   # the reference binary is built by build(); report why not
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU run failed: {e}"[:300]}))
        return
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
        "n_gpus": a.gpus, "steps": nt, "warmup": 0,
        "ms_per_step": round((det["bc_s"] + det["pressure_s"]) / nt * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (eigen mode, the reference's own Propa initialisation)",
        "config": propa_config(a, layout_n1=a.size + 2 * (a.order // 2),
                               l2="inputs larger than L2 (the host's caches)",
                               tuning="CacheBlk (reference CPU, unchanged source), its default "
                                      "cache blocks",
                               parallelism=f"OpenMP x{threads} host threads"),
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads,
                         "kind": "reference",
                         "sample": f"{nt} time steps of {a.size}^3, timed by the reference's own "
                                   "boundary-condition + compute-pressure timers"},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "details": det,
    }
    print(json.dumps(line))


# ---- B200 arm ------------------------------------------------------------------------------------

def b200_arm(a):
    import ctypes

    import numpy as np
    import torch

    from hpcscan_b200 import _lib
    from hpcscan_b200 import layout as L
    from hpcscan_b200.grid import Grid, init_device
    from hpcscan_b200.propagator import Propagator_Ac2, run_propa

    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device(f"cuda:{local}"))
    init_device(local)
    lay = L.b200_layout(3, a.size, a.size, a.size, order=a.order, prec="f32")

    propa = Propagator_Ac2(lay, device=local)
    propa.initialize(ratio_cfl=0.8, nt=1, snap_inc=1, modes=(1, 1, 1))
    prn, prc = propa.prnGrid, propa.prcGrid
    stream = torch.cuda.current_stream()

    # events around every pressure-kernel launch of the timed region (same stream)
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(a.steps)]

    fused = False

    def step(i=None):
        # Propagator_Ac2::computeWavefieldNextTimeStep: the boundary condition and the pressure
        # update, or the fused kernel where the tuner measured it faster for this grid (events
        # then bracket the fused kernel and its boundary-plane kernel)
        nonlocal prn, prc
        if fused:
            if i is not None:
                kev[i][0].record(stream)
            propa.computeWavefieldNextTimeStep(prn, prc)
        else:
            prc.applyBoundaryCondition()
            if i is not None:
                kev[i][0].record(stream)
            propa.computePressureWithFD(prn, prc)
        if i is not None:
            kev[i][1].record(stream)
        prn, prc = prc, prn

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # tuning on first use (b200_set_autotune): the first propagator step times the kernel
    # candidates for this grid; untimed, before the warm-up
    propa.computeWavefieldNextTimeStep(prn, prc)
    prn, prc = prc, prn
    torch.cuda.synchronize()
    tuning = propa.step_config()
    fused = tuning["step"]["fused"]
    with ClockSampler(torch.cuda.current_device()) as clk:
        for _ in range(a.warmup):
            step()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        clk.begin()
        e0.record(stream)
        for i in range(a.steps):
            step(i)
        e1.record(stream)
        torch.cuda.synchronize()
        clk.end()
    ms = e0.elapsed_time(e1)
    kern_ms = [s.elapsed_time(e) for s, e in kev]
    st = ctypes.c_int()
    _lib.call("b200_device_status", ctypes.byref(st), 1)
    if st.value:
        raise RuntimeError(f"device-side error word {st.value}")
    ms, kmean = max_over_ranks(dist, [ms, statistics.mean(kern_ms)], "cuda")
    pts = lay.inner_points
    value = job_gpoints(world, pts, a.steps, ms * 1e-3)

    # error of the benchmarked field against the analytic solution at the last step
    del kev
    peak, peak_src = measured_peak()
    achieved = ALG_BYTES_PER_POINT * pts / (kmean * 1e-3) / 1e9
    traffic = profiled_traffic()
    if traffic is not None and (traffic.get("workload", {}).get("n") != a.size or
                                traffic.get("workload", {}).get("order") != a.order):
        traffic = None          # the committed capture covers another workload
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": peak_src,
            "kernel": KERNEL_STEP_NAME if fused else KERNEL_NAME, "kernel_ms": round(kmean, 5),
            "alg_bytes_per_point": ALG_BYTES_PER_POINT, "points_per_launch": pts,
            "traffic": None if traffic is None else traffic.get("dram_bytes_per_launch"),
            "traffic_unit": "bytes per launch",
            "traffic_note": None if traffic is None else traffic.get("note")}
    # free the timed grids before the end-to-end job
    del propa, prn, prc
    torch.cuda.empty_cache()

    e2e = e2e_job(a, lay, local)
    if dist is not None:
        (sec,) = max_over_ranks(dist, [e2e["seconds"]], "cuda")
        e2e["value"] = round(job_gpoints(world, e2e["points"], 1, sec), 4)

    cpu = None
    if rank == 0 and not a.no_cpu:
        threads = os.cpu_count() or 1
        try:
            v, det = run_reference_cpu(a.size, a.order, a.cpu_steps, threads)
            cpu = {"value": round(v, 4), "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"{a.cpu_steps} time steps of the same {a.size}^3 O{a.order} FP32 "
                             "Propa grid, reference CacheBlk, timed by its own BC + pressure timers",
                   "details": det}
        except Exception as e:
            cpu = {"value": None, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"unavailable: {e}"[:200]}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (eigen mode sin(pi x) sin(pi y) sin(pi z), the reference's Propa "
                "initialisation; no dataset involved)",
        "config": propa_config(a, layout_n1=lay.n1,
                               l2="inputs larger than L2 (3 x %.0f MB grids vs 126 MB L2)"
                                  % (lay.nbytes / 1e6),
                               tuning=tuning, parallelism=f"replicas x{world}"),
        # per step: the boundary condition (one launch when every axis has 2 halo + 2 inner
        # points, else halos + planes) and the pressure kernel
        "gpu_launches": (2 if (fused or min(lay.n_inner) >= 2 * lay.halo + 2) else 3) * a.steps,
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": {k: e2e[k] for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step",
                                    "job_steps", "err_test_case", "note")},
        "clocks": clocks,
    }
    print(json.dumps(line))


def e2e_job(a, lay, device):
    """One Propa job through the public API from host memory: the initial fields are
    built on the host (as a caller holding its own arrays would), copied from pinned
    memory into the grids, the time loop runs with the reference's analytic checks
    (every snapInc steps, fused norm), and the final wavefield comes back to the host."""
    import numpy as np
    import torch

    from hpcscan_b200 import layout as L
    from hpcscan_b200.propagator import Propagator_Ac2, l1_sums_eigen
    from hpcscan_b200.propa_setup import EIGEN_FUNCS, eigen_setup, init_times

    setup = eigen_setup(lay, ratio_cfl=0.8, tmax=2.0 / np.sqrt(3.0), modes=(1, 1, 1))
    nt = a.e2e_steps if a.e2e_steps > 0 else setup.nt
    snap = max(1, nt // 10)
    # host inputs (pinned): prn(-2dt), prc(-dt), coef
    samp = setup.samp
    tabs = L.fill_tables(lay, samp, L.ALL_POINTS, EIGEN_FUNCS, setup.params(lay))
    t_prn, t_prc = init_times(setup, "f32")
    sh = lay.shape3
    b = lay.box(L.ALL_POINTS)

    def host_field(amp):
        h = torch.zeros(lay.npoint, dtype=torch.float32).pin_memory()
        v = h.numpy().reshape(sh)
        sl = lay.box_slices(L.ALL_POINTS)
        # (((amp * v1) * v2) * v3) per point, the order of Grid::fill
        v[sl] = (((amp * tabs[0][None, None, :]) * tabs[1][None, :, None]) *
                 tabs[2][:, None, None]).astype(np.float32)
        return h
    h_prn = host_field(setup.amplitude(t_prn))
    h_prc = host_field(setup.amplitude(t_prc))
    h_coef = torch.zeros(lay.npoint, dtype=torch.float32).pin_memory()
    h_coef.numpy().reshape(sh)[lay.box_slices(L.INNER_POINTS)] = np.float32(setup.coef)
    h_out = torch.empty(lay.npoint, dtype=torch.float32).pin_memory()

    propa = Propagator_Ac2(lay, device=device)
    propa.initialize(ratio_cfl=0.8, tmax=2.0 / np.sqrt(3.0), modes=(1, 1, 1))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    prn, prc = propa.prnGrid, propa.prcGrid
    prn.data.copy_(h_prn, non_blocking=True)
    prc.data.copy_(h_prc, non_blocking=True)
    propa.coefGrid.data.copy_(h_coef, non_blocking=True)
    sum1 = np.float32(0)
    sum2 = np.float32(0)
    for it in range(nt):
        propa.computeWavefieldNextTimeStep(prn, prc)
        if it % snap == 0:
            s1, s2 = l1_sums_eigen(prn, propa, setup.amplitude(setup.time_of_step(it, "f32")))
            sum1 = np.float32(sum1 + np.float32(s1))
            sum2 = np.float32(sum2 + np.float32(s2))
        prn, prc = prc, prn
    h_out.copy_(prc.data, non_blocking=True)
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    pts = lay.inner_points * nt
    h2d = 3 * lay.nbytes
    d2h = lay.nbytes + (nt // snap + 1) * 16
    return {"value": round(pts / sec / 1e9, 4), "unit": UNIT, "seconds": sec, "points": pts,
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "job_steps": nt,
            "err_test_case": float(np.float32(sum1 / sum2)),
            "note": "one e2e step = one whole Propa job of job_steps time steps from pinned "
                    "host arrays (H2D of prn, prc, coef; D2H of the final wavefield and of "
                    "the periodic analytic-check norms)"}


# ---- batched modelling and adjoint workloads ------------------------------------------------------

def _shot_dist():
    """Process group of the shot-parallel workloads under torchrun (NCCL, one GPU per rank):
    (dist or None, rank, world, local rank)."""
    rank, world, local = dist_env()
    if world == 1:
        return None, rank, world, local
    import datetime

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                            device_id=torch.device(f"cuda:{local}"))
    return dist, rank, world, local


def sum_over_ranks(dist, values, device):
    """Per-rank counts -> their sums over all ranks (one all-reduce); the values themselves on
    a single process."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.tolist()


def _surface_shots(n, nshot, seed):
    """Distinct seeded source positions on the surface plane i1 = 1, off the receiver lattice."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out, seen = [], set()
    while len(out) < nshot:
        j, k = (int(v) for v in rng.integers(n // 8, n - n // 8, size=2))
        if j % 4 == 0 and k % 4 == 0:
            j += 1
        if (j, k) not in seen:
            seen.add((j, k))
            out.append((1, j, k))
    return out


def _timed(fn, reps=1):
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def _graph_timed(fn, reps):
    """Device seconds per call of fn(stream): reps calls captured in one CUDA graph, the replay
    timed with CUDA events (after one untimed replay)."""
    import torch
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        for _ in range(reps):
            fn(s)
    g.replay()
    torch.cuda.synchronize()
    sec = _timed(g.replay)
    del g
    return sec / reps


def adjoint_arm(a):
    """Batched checkpointed adjoint gradients vs the plain one-shot-per-launch form.

    16 shots on one 256^3 grid (dx 10 m), O8 FP32, 2000 steps, Ricker f0 10 Hz, 20-point
    sponge, receivers on the surface plane i1 = 1 every 4th point in i2 and i3, sources at seeded
    surface positions; observed data from the background model with a 5 % Gaussian anomaly of
    the squared slowness (sigma 10 points, centre); gradient of 1/2 |d - dobs|^2 with respect to
    the squared slowness at the background; checkpoints every 45 steps. Batched: all shots in
    each launch, the whole gradient (forward, then segment-wise recompute, adjoint and
    gradient) replayed from one CUDA graph, then the survey gradient (the sum over the shots).
    Plain: the same kernels one shot per launch, from the host, no graph. Both give
    bit-identical per-shot gradients (checked).

    Under torchrun the survey is split over the ranks (hpcscan_b200.shots: one GPU per rank,
    its shots in one batch, nothing exchanged in the time loop) and the survey gradient ends
    with one sum all-reduce, inside the timed region; the time is the max over ranks (strong
    scaling: the survey is fixed). The plain form runs on a single process only."""
    import numpy as np
    import torch

    from hpcscan_b200.grid import init_device
    from hpcscan_b200.modeling import Batch, Shot, grf_velocity, run_graph, stable_dt
    from hpcscan_b200.shots import my_shots, survey_gradient

    dist, rank, world, local = _shot_dist()
    n = a.size
    nshot = a.shots or 16
    if nshot < world:
        raise SystemExit(f"{nshot} shots for {world} ranks: every rank needs a shot")
    nt = a.nt or 2000
    order, dx, f0 = a.order, 10.0, 10.0
    init_device(local)
    dev = f"cuda:{local}"
    mine = my_shots([1.0] * nshot, rank, world)
    vel0 = grf_velocity((n, n, n), sigma=20.0, seed=1234, device=local)
    c = (n - 1) / 2.0
    ax = torch.arange(n, device=dev, dtype=torch.float32)
    r2 = (ax[:, None, None] - c) ** 2 + (ax[None, :, None] - c) ** 2 + (ax[None, None, :] - c) ** 2
    vel_true = vel0 / torch.sqrt(1.0 + 0.05 * torch.exp(-r2 / (2 * 10.0 ** 2)))
    del r2
    rec = np.array([(1, j, k) for j in range(0, n, 4) for k in range(0, n, 4)])
    srcs = _surface_shots(n, nshot, 4321)
    dt = stable_dt(order, dx, 4500.0)

    def shots(vel, dobs=None):
        return [Shot(n=(n, n, n), dx=dx, vel=vel, src=srcs[i], rec=rec, amp=1.0, sponge=20,
                     dobs=None if dobs is None else dobs[j]) for j, i in enumerate(mine)]

    obs = Batch(shots(vel_true), order, dt, nt, f0, device=local)
    obs.forward()
    torch.cuda.synchronize()
    dobs = [obs.traces(j).clone() for j in range(len(mine))]
    obs.close()
    del obs
    torch.cuda.empty_cache()

    # batched: one graph for the whole gradient of this rank's shots; the shots share one grid,
    # so the backward pass accumulates the survey gradient itself (one stencil-free pass per step
    # over all shots, survey=True), and the CTAs of one tile of every shot run side by side (the
    # model tiles then come from DRAM once)
    bat = Batch(shots(vel0, dobs), order, dt, nt, f0, gradient=True, checkpoint=a.checkpoint,
                device=local, survey=bool(a.survey))
    gsum = torch.empty((n, n, n), dtype=torch.float32, device=dev)
    mem_batched = torch.cuda.memory_allocated() / 1e9
    ctas = bat.ctas_per_pass
    g = run_graph(lambda s: (bat.forward(s), bat.backward(s)))

    def job():
        g.replay()
        survey_gradient(bat, out=gsum)

    _timed(job)                                    # warm-up replay
    t_batched = _timed(job)
    (t_batched,) = max_over_ranks(dist, [t_batched], dev)
    launches, jsum = sum_over_ranks(dist, [bat.launches, sum(bat.misfit(j) for j in range(len(mine)))], dev)
    gnorm = float(gsum.double().norm())
    del g
    bat.close()
    del bat
    torch.cuda.empty_cache()

    plain = None
    if world == 1:
        # plain: one shot per launch, eager, shot after shot, each shot's gradient by its own
        # stencil pass per step; each shot's set-up (allocation, tensor maps) stays outside the
        # timed part, which is its forward + backward pass; the survey gradient is the sum of
        # the shots' gradients (timed too)
        def plain_one(i):
            b = Batch(shots(vel0, dobs)[i:i + 1], order, dt, nt, f0, gradient=True,
                      checkpoint=a.checkpoint, device=local)
            sec = _timed(lambda: (b.forward(), b.backward()))
            out = b.gradient_of(0).clone()
            b.close()
            return sec, out
        plain_one(0)                                   # warm-up
        t_plain = 0.0
        gplain = torch.zeros_like(gsum)
        for i in range(nshot):
            sec, gi = plain_one(i)
            t_plain += sec
            t_plain += _timed(lambda: gplain.add_(gi))
        d = (gsum.double() - gplain.double()).norm() / gplain.double().norm()
        plain = (t_plain, float(d))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    pts = n ** 3
    k = a.checkpoint
    nck = (nt + k - 1) // k
    # algorithmic bytes per shot: forward 16 B/pt-step, recompute 16 B (one step per segment
    # more for the survey pass), adjoint 16 B, and either the survey gradient (16 B per shot + the
    # gradient's read and write shared by the shots) or each shot's gradient pass (20 B);
    # checkpoint save (8 B/pt written) and restore (8 B read + 8 B written) per checkpoint
    if a.survey:
        alg = pts * ((16 * nt + 16 * nt + 16 * nt + 16 * nt + 24 * nck) * nshot + 8 * nt * world)
    else:
        alg = pts * (16 * nt + 16 * (nt - nck) + 16 * nt + 20 * nt + 24 * nck) * nshot
    peak, peak_src = measured_peak()
    peak_job = peak * world
    line = {
        "metric": f"adjoint gradient shots/s ({n}^3, O{order} FP32, {nt} steps, checkpoint {k})",
        "value": round(nshot / t_batched, 4), "unit": "shots/s", "n_gpus": world, "steps": nt,
        "warmup": 1, "ms_per_step": round(t_batched / nt * 1e3, 4), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian-random-field velocity 1500-4500 m/s, 5 % Gaussian "
                "anomaly of the squared slowness, Ricker 10 Hz sources); no dataset involved",
        "config": {"workload": "batched checkpointed adjoint gradients", "n": n, "shots": nshot,
                   "order": order, "dx_m": dx, "receivers": len(rec), "sponge": 20,
                   "checkpoint_every": k, "ctas_per_pass": ctas,
                   "parallelism": f"shots over {world} rank(s), one gradient all-reduce",
                   "device_memory_gb": round(mem_batched, 1)},
        "misfit_mean": jsum / nshot,
        "survey_gradient_norm": gnorm,
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": round(alg / t_batched / 1e9, 1),
                     "peak": peak_job, "unit": "GB/s",
                     "frac": round(alg / t_batched / 1e9 / peak_job, 4),
                     "peak_source": peak_src + (f" x {world} GPUs" if world > 1 else ""),
                     "alg_bytes": ("per shot-step: 16 forward + 16 recompute + 16 adjoint + 16 "
                                   "survey gradient, plus 8 per step for the gradient grid and "
                                   "the checkpoint save/restore") if a.survey else
                                  ("per shot-step: 16 forward + 16 recompute + 16 adjoint + 20 "
                                   "gradient, plus the checkpoint save/restore")},
        "seconds": round(t_batched, 3),
        "batched_form": "all shots in every launch, the whole gradient in one CUDA graph, CTAs of "
                        "one tile of every shot side by side, " +
                        ("the survey gradient accumulated over the shots in one stencil-free pass "
                         "per step" if a.survey else
                         "each shot's gradient by a stencil pass per step, summed after") +
                        " (timed, with the final all-reduce under torchrun)",
    }
    if plain is not None:
        t_plain, d = plain
        line["plain"] = {"value": round(nshot / t_plain, 4), "unit": "shots/s",
                         "form": "one shot per launch, eager host loop, no CUDA graph, each "
                                 "shot's gradient by a stencil pass per step, the survey "
                                 "gradient summed from the shots' gradients (timed); per-shot "
                                 "set-up (allocation, tensor maps) not timed",
                         "seconds": round(t_plain, 3)}
        line["speedup_vs_plain"] = round(t_plain / t_batched, 3)
        line["survey_gradient_rel_diff_vs_plain"] = d
    print(json.dumps(line))


def modeling_arm(a):
    """Batched multi-shot forward modelling: 64 shots on uneven cubes N_s = 128 + round(192 s /
    63) (128 .. 320), dx 10 m, Gaussian-random-field velocity 1500-4500 m/s (seed 1234 + s,
    Gaussian kernel sigma 20 points), Ricker 10 Hz point source at the surface centre (i1 = 1),
    20-point sponge, O8 FP32, 1500 steps; every step of every shot in one launch, the time loop
    in one CUDA graph; against the same kernels one shot per launch without a graph.

    Under torchrun the survey is split over the ranks by work (hpcscan_b200.shots: points per
    shot, longest first to the least-loaded rank), each rank's shots in one batch on its GPU,
    nothing exchanged; the time is the max over ranks (strong scaling: the survey is fixed).
    The plain form runs on a single process only."""
    import numpy as np
    import torch

    from hpcscan_b200.grid import init_device
    from hpcscan_b200.modeling import Batch, Shot, grf_velocity, run_graph, stable_dt
    from hpcscan_b200.shots import my_shots

    dist, rank, world, local = _shot_dist()
    nshot = a.shots or 64
    if nshot < world:
        raise SystemExit(f"{nshot} shots for {world} ranks: every rank needs a shot")
    nt = a.nt or 1500
    order, dx, f0 = a.order, 10.0, 10.0
    init_device(local)
    sizes = [128 + round(192 * s / max(nshot - 1, 1)) for s in range(nshot)]
    mine = my_shots([float(n) ** 3 for n in sizes], rank, world)
    dt = stable_dt(order, dx, 4500.0)
    shots = []
    for s in mine:
        n = sizes[s]
        vel = grf_velocity((n, n, n), sigma=20.0, seed=1234 + s, device=local)
        rec = np.array([(1, j, n // 2) for j in range(0, n, 2)])
        shots.append(Shot(n=(n, n, n), dx=dx, vel=vel, src=(1, n // 2, n // 2), rec=rec,
                          amp=1.0, sponge=20))
    bat = Batch(shots, order, dt, nt, f0, device=local)
    g = run_graph(lambda st: bat.forward(st))
    _timed(g.replay)
    t_batched = _timed(g.replay)
    dev = f"cuda:{local}"
    (t_batched,) = max_over_ranks(dist, [t_batched], dev)
    (launches,) = sum_over_ranks(dist, [bat.launches // 2], dev)
    traces = [bat.traces(j).clone() for j in range(len(mine))] if world == 1 else []
    del g
    bat.close()
    del bat
    torch.cuda.empty_cache()
    plain = None
    if world == 1:
        same, t_plain = True, 0.0
        for i in range(nshot):
            b = Batch(shots[i:i + 1], order, dt, nt, f0, device=local)
            t_plain += _timed(b.forward)
            same = same and bool(torch.equal(b.traces(0), traces[i]))
            b.close()
        plain = (t_plain, same)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    pts = sum(n ** 3 for n in sizes) * nt
    peak, peak_src = measured_peak()
    peak_job = peak * world
    line = {
        "metric": f"batched modelling GPoint/s ({nshot} shots 128^3..320^3, O{order} FP32, {nt} steps)",
        "value": round(pts / t_batched / 1e9, 4), "unit": "GPoint/s", "n_gpus": world, "steps": nt,
        "warmup": 1, "ms_per_step": round(t_batched / nt * 1e3, 4), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian-random-field velocities); no dataset involved",
        "config": {"workload": "batched multi-shot modelling, one CUDA graph", "shots": nshot,
                   "sizes": [sizes[0], sizes[-1]], "order": order, "dx_m": dx, "sponge": 20,
                   "parallelism": f"shots over {world} rank(s) by work, nothing exchanged"},
        "shots_per_s": round(nshot / t_batched, 4),
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": round(16 * pts / t_batched / 1e9, 1),
                     "peak": peak_job, "unit": "GB/s",
                     "frac": round(16 * pts / t_batched / 1e9 / peak_job, 4),
                     "peak_source": peak_src + (f" x {world} GPUs" if world > 1 else "")},
        "seconds": round(t_batched, 3),
        "batched_form": "all shots in every launch (a CTA range per shot), the time loop in one "
                        "CUDA graph",
    }
    if plain is not None:
        t_plain, same = plain
        line["plain"] = {"value": round(pts / t_plain / 1e9, 4), "unit": "GPoint/s",
                         "form": "same kernels, one shot per launch, eager host loop, no CUDA "
                                 "graph (per-shot set-up not timed)",
                         "seconds": round(t_plain, 3)}
        line["speedup_vs_plain"] = round(t_plain / t_batched, 3)
        line["traces_identical_to_plain"] = same
    print(json.dumps(line))


def mixed_arm(a):
    """Mixed-precision Propa: the eigen-mode test (ratioCFL 0.8, modes (1, 1, 1)) at 512^3 (or
    --size), O8 (or --order), 1000 steps (or --nt), wavefields in FP16 and in BF16 with a
    power-of-two per-field scale, FP32 coef and FP32 stencil arithmetic; against the FP64 run
    of the same steps (bit-identical to the reference's FP64 build) and the analytic solution.
    A step = boundary condition + pressure update, as in the headline workload."""
    import numpy as np
    import torch

    from hpcscan_b200 import layout as L
    from hpcscan_b200.grid import init_device
    from hpcscan_b200.propagator import Propagator_Ac2, l1_sums_eigen

    n, order = a.size, a.order
    nt = a.nt or 1000
    init_device(0)
    results = {}
    finals = {}
    ref_dev = None
    for prec, coef_prec, scale in (("f64", "f64", 1.0), ("f32", "f32", 1.0), ("f16", "f32", 2.0 ** 4),
                                   ("bf16", "f32", 1.0)):
        lay = L.b200_layout(3, n, n, n, order=order, prec=prec)
        propa = Propagator_Ac2(lay, coef_prec=coef_prec, wave_scale=scale)
        propa.initialize(ratio_cfl=0.8, nt=nt, snap_inc=max(1, nt // 10), modes=(1, 1, 1))
        s = propa.setup
        prn, prc = propa.prnGrid, propa.prcGrid
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sum1 = sum2 = np.float32(0.0)
        kernel_ms = 0.0
        for it in range(nt):
            if it == 3:
                torch.cuda.synchronize()
                e0.record(stream)
            propa.computeWavefieldNextTimeStep(prn, prc)
            if it % s.snap_inc == 0:
                amp = s.amplitude(s.time_of_step(it, "f64" if prec == "f64" else "f32"))
                s1, s2 = l1_sums_eigen(prn, propa, amp)
                sum1 = np.float32(sum1 + np.float32(s1))
                sum2 = np.float32(sum2 + np.float32(s2))
            prn, prc = prc, prn
        e1.record(stream)
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        steps = nt - 3
        bpp = {"f64": 32, "f32": 16, "f16": 10, "bf16": 10}[prec]
        # the last wavefield's inner points as physical values, kept on the device (FP64)
        fin = lay.inner(prc.data.detach()).to(torch.float64) * prc.scale
        if prec == "f64":
            ref_dev = fin
        else:
            d = (fin - ref_dev).flatten()
            rel = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(ref_dev.flatten()))
            finals[prec] = rel
        del fin
        results[prec] = {"gpoint_s": round(lay.inner_points * steps / sec / 1e9, 3),
                         "ms_per_step": round(sec / steps * 1e3, 4),
                         "alg_gb_s": round(bpp * lay.inner_points * steps / sec / 1e9, 1),
                         "bytes_per_point": bpp,
                         "err_test_case": float(sum1 / sum2), "wave_scale": scale,
                         "coef": coef_prec}
        del propa, prn, prc
        torch.cuda.empty_cache()
    for prec, rel in finals.items():
        results[prec]["rel_l2_vs_fp64"] = rel
        results[prec]["meets_1pct_vs_fp64"] = rel < 1e-2
    del ref_dev
    pk, pk_src = measured_peak()
    line = {
        "metric": f"mixed-precision Propa GPoint/s (O{order}, FP16 wavefields, FP32 coef and "
                  f"arithmetic, {n}^3, {nt} steps)",
        "value": results["f16"]["gpoint_s"], "unit": "GPoint/s", "n_gpus": 1, "steps": nt - 3,
        "warmup": 3, "ms_per_step": results["f16"]["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f16 storage, f32 compute",
        "data": "synthetic (eigen mode, the reference's Propa initialisation)",
        "config": {"workload": "mixed-precision Propa (BC + pressure update per step)", "n": n,
                   "order": order, "ratio_cfl": 0.8, "steps": nt,
                   "accuracy": "rel_l2_vs_fp64: relative L2 distance of the last wavefield's inner "
                               "points to the FP64 run of the same steps (computed on the device); "
                               "the bar is 1e-2"},
        "per_precision": results,
        "roofline": {"bound": "hbm", "achieved": results["f16"]["alg_gb_s"], "peak": pk,
                     "unit": "GB/s", "frac": round(results["f16"]["alg_gb_s"] / pk, 4),
                     "peak_source": pk_src, "note": "whole step (BC + pressure), 10 B/point"},
    }
    print(json.dumps(line))


def run_reference_fd(case: str, n: int, order: int, threads: int):
    """The reference's FD_D1 / FD_D2 test case (CacheBlk, its optimised CPU path) at n^3:
    its own 'Best Gpoint/s in FD' per operator, in the order the test case runs them."""
    from oracle import oracle
    exe = oracle.ref_binary("f32")
    args = [exe, "-testCase", case, "-testMode", "CacheBlk", "-fdOrder", str(order),
            "-n1", str(n), "-n2", str(n), "-n3", str(n), "-ntry", "3"]
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close")
    with tempfile.TemporaryDirectory() as d:
        out = subprocess.run(args, cwd=d, capture_output=True, text=True, env=env, timeout=900)
    if out.returncode != 0:
        raise RuntimeError(out.stdout[-2000:] + out.stderr[-2000:])
    return [float(x) for x in re.findall(r"Best Gpoint/s in FD\s+(\S+)", out.stdout)]


def fd_arm(a):
    """The single-operator test cases at n^3 (default 512), O8 (or --order), FP32:
    FD_D1_N1/N2/N3 (src/testCase_FD_D1.cpp) and FD_D2_N1/N2/N3 + FD_LAPLACIAN
    (src/testCase_FD_D2.cpp) on the test cases' own input sin(a1 x1) sin(a2 x2) sin(a3 x3).
    Each operator is launched --steps times back to back after --warmup launches and timed
    with CUDA events; one launch reads u and writes w over the inner points (8 B/point
    algorithmic; the 1 GB pair of grids is eight times L2, so nothing stays cached between
    launches). Beside it the reference's own CacheBlk numbers of the same test cases on the
    host cores."""
    import numpy as np
    import torch

    from hpcscan_b200 import layout as L
    from hpcscan_b200.grid import Grid, init_device

    n, order = a.size, a.order
    init_device(0)
    lay = L.b200_layout(3, n, n, n, order=order, prec="f32")
    U, W = Grid(lay), Grid(lay)
    U.initializeGrid()
    W.initializeGrid()
    U.defineUnitGrid()
    W.defineUnitGrid()
    U.fill(L.ALL_POINTS, L.FUNC_SINE, L.FUNC_SINE, L.FUNC_SINE, L.PI * 0.8, L.PI * 0.9, L.PI * 1.0,
           1.1)
    ops = ["FD_D1_N1", "FD_D1_N2", "FD_D1_N3", "FD_D2_N1", "FD_D2_N2", "FD_D2_N3", "FD_LAPLACIAN"]
    peak, peak_src = measured_peak()
    pts = lay.inner_points
    res = {}
    with ClockSampler(0) as clk:
        clk.begin()
        for op in ops:
            fn = getattr(U, op)
            for _ in range(max(a.warmup, 3)):
                fn(L.INNER_POINTS, W, order)
            sec = _timed(lambda: fn(L.INNER_POINTS, W, order), reps=a.steps)
            res[op] = {"gpoint_s": round(pts / sec / 1e9, 2), "us_per_launch": round(sec * 1e6, 2),
                       "alg_gb_s": round(8 * pts / sec / 1e9, 1),
                       "frac_of_peak": round(8 * pts / sec / 1e9 / peak, 4)}
        clk.end()
    cpu = {}
    if not a.no_cpu:
        threads = os.cpu_count() or 1
        try:
            d1 = run_reference_fd("FD_D1", n, order, threads)
            d2 = run_reference_fd("FD_D2", n, order, threads)
            for op, v in zip(ops, d1 + d2):
                cpu[op] = v
            cpu["cores"] = threads
        except Exception as e:
            cpu = {"unavailable": str(e)[:200]}
    d1_sec = sum(pts / (res[op]["gpoint_s"] * 1e9) for op in ops[:3])
    value = 3 * pts / d1_sec / 1e9
    line = {
        "metric": f"FD_D1 GPoint/s (staggered first derivative, O{order} FP32 {n}^3, mean of the "
                  "three axes)",
        "value": round(value, 2), "unit": "GPoint/s", "n_gpus": 1, "steps": a.steps,
        "warmup": max(a.warmup, 3), "ms_per_step": round(d1_sec / 3 * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (the test cases' own sine input)",
        "config": {"workload": f"FD_D1 / FD_D2 operator test cases, O{order} FP32 {n}^3",
                   "n": n, "order": order, "l2": "inputs 8x larger than L2, no flush"},
        "per_operator": res,
        "cpu_reference_gpoint_s": cpu,
        "roofline": {"bound": "hbm", "achieved": round(8 * value, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(8 * value / peak, 4), "peak_source": peak_src,
                     "alg_bytes": "8 B/point: read u, write w"},
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


def fdsweep_arm(a):
    """The FD_D2 test case's sweep at its stated sizes: FD_D2_N1/N2/N3 and FD_LAPLACIAN of
    u = sin(4 pi x1) sin(6 pi x2) sin(8 pi x3) on the unit cube (src/testCase_FD_D2.cpp:65-74 with
    -param1 4 -param2 6 -param3 8 -param4 1) for orders 2/4/8/12/16, cubes of 128/256/512/800
    inner points, FP32 and FP64. Per entry: device time per launch (--steps launches captured in a
    CUDA graph, the replay timed with CUDA events, after three warm-up launches; at 256^3 and
    above the pair of grids exceeds L2, at 128^3 it does not and the figure is marked so), the
    same launches called one by one from Python (us_per_call_eager: at 128^3 the host path of a
    call is longer than the kernel), GPoint/s, algorithmic GB/s (read u, write w: 8 B/point
    FP32, 16 FP64) and its fraction of the measured copy bandwidth, and the L1 error against the
    analytic derivative as the test case computes it (Grid::L1Err over the inner points, FP64
    sums on the device)."""
    import torch

    from hpcscan_b200 import layout as L
    from hpcscan_b200.grid import Grid, init_device

    init_device(0)
    peak, peak_src = measured_peak()
    sizes = [int(s) for s in (a.sizes.split(",") if a.sizes else ["128", "256", "512", "800"])]
    orders = [int(o) for o in (a.orders.split(",") if a.orders else ["2", "4", "8", "12", "16"])]
    a1, a2, a3 = L.PI * 4, L.PI * 6, L.PI * 8
    ops = [("FD_D2_N1", -a1 * a1), ("FD_D2_N2", -a2 * a2), ("FD_D2_N3", -a3 * a3),
           ("FD_LAPLACIAN", -(a1 * a1 + a2 * a2 + a3 * a3))]
    entries = []
    launches = 0
    with ClockSampler(0) as clk:
        clk.begin()
        for prec in ("f32", "f64"):
            bpp = 8 if prec == "f32" else 16
            for n in sizes:
                for order in orders:
                    lay = L.b200_layout(3, n, n, n, order=order, prec=prec)
                    U, W, R = Grid(lay), Grid(lay), Grid(lay)
                    for g in (U, W, R):
                        g.initializeGrid()
                        g.defineUnitGrid()
                    U.fill(L.ALL_POINTS, L.FUNC_SINE, L.FUNC_SINE, L.FUNC_SINE, a1, a2, a3, 1.0)
                    pts = lay.inner_points
                    for op, amp in ops:
                        fn = getattr(U, op)
                        W.fill(L.ALL_POINTS, 0.0)
                        for _ in range(3):
                            fn(L.INNER_POINTS, W, order)
                        eager = _timed(lambda: fn(L.INNER_POINTS, W, order), reps=a.steps)
                        # the same launches captured in a CUDA graph and replayed: the device
                        # time of the kernels without the host's per-call path (which, for the
                        # small cubes, is longer than the kernel)
                        sec = _graph_timed(lambda st: fn(L.INNER_POINTS, W, order, stream=st),
                                           a.steps)
                        launches += 3 + 3 * a.steps
                        R.fill(L.ALL_POINTS, L.FUNC_SINE, L.FUNC_SINE, L.FUNC_SINE, a1, a2, a3, amp)
                        err = W.L1Err(L.INNER_POINTS, R)
                        gbs = bpp * pts / sec / 1e9
                        entries.append({"prec": prec, "n": n, "order": order, "op": op,
                                        "us_per_launch": round(sec * 1e6, 2),
                                        "us_per_call_eager": round(eager * 1e6, 2),
                                        "gpoint_s": round(pts / sec / 1e9, 2),
                                        "alg_gb_s": round(gbs, 1),
                                        "frac_of_peak": round(gbs / peak, 4),
                                        "l1_err_vs_analytic": float(err),
                                        "pass_1e-3": bool(err < 1e-3),
                                        "in_l2": 2 * lay.nbytes < 126e6})
                    del U, W, R
                    torch.cuda.empty_cache()
        clk.end()
    st = ctypes_status()
    if st:
        raise RuntimeError(f"device-side error word {st}")
    head = [e for e in entries if (e["prec"], e["n"], e["order"], e["op"]) ==
            ("f32", 512, 8, "FD_LAPLACIAN")]
    value = head[0]["gpoint_s"] if head else entries[-1]["gpoint_s"]
    cols = ["prec", "n", "order", "op", "us_per_launch", "us_per_call_eager", "gpoint_s",
            "alg_gb_s", "frac_of_peak", "l1_err_vs_analytic", "pass_1e-3", "in_l2"]
    line = {
        "metric": "FD_D2 sweep GPoint/s (FD_LAPLACIAN O8 FP32 512^3 as the value; every entry in "
                  "`entries`)",
        "value": value, "unit": "GPoint/s", "n_gpus": 1, "steps": a.steps, "warmup": 3,
        "ms_per_step": round(head[0]["us_per_launch"] / 1e3, 5) if head else None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
        "data": "synthetic (the FD_D2 test case's own sine input, k = (2, 3, 4))",
        "config": {"workload": "FD_D2 test-case sweep: orders x cubes x precisions",
                   "orders": orders, "sizes": sizes, "precisions": ["f32", "f64"],
                   "l2": "inputs larger than L2 from 256^3 on; 128^3 entries flagged in_l2"},
        "gpu_launches": launches,
        "peak_gb_s": peak, "peak_source": peak_src,
        "entries_columns": cols,
        "entries": [[e[c] for c in cols] for e in entries],
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


def launches_arm(a):
    """One launch of each hot kernel at n^3 (default 512), for a profiler: the pressure update
    in FP32 at each of --orders (default 8,12), the Laplacian at each of them, and the pressure
    update on FP16 wavefields (FP32 coef) at the first order; inputs filled on the device (the
    eigen-mode fields, the test case's sine product). Run with HPCSCAN_B200_AUTOTUNE=0 the
    launches use the untuned defaults and nothing else of the library runs between them. Prints
    the device time of each launch (CUDA events) in one JSON line."""
    import torch

    from hpcscan_b200 import layout as L
    from hpcscan_b200.grid import Grid, init_device

    init_device(0)
    n = a.size
    orders = [int(o) for o in (a.orders.split(",") if a.orders else ["8", "12"])]
    samp = L.Sampling((1.0 / (n - 1),) * 3, (0.0,) * 3)

    def grid(lay, scale=1.0):
        g = Grid(lay, samp, scale=scale)
        g.initializeGrid()
        return g

    def timed_once(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return round(e0.elapsed_time(e1) * 1e3, 1)

    out = []

    def pressure(order, prec, coef, scale):
        lay = L.b200_layout(3, n, n, n, order=order, prec=prec)
        clay = lay if coef == prec else L.GridLayout(dim=3, order=order, prec=coef, a1=lay.a1,
                                                     a2=lay.a2, a3=lay.a3, n_inner=lay.n_inner)
        prn, prc, cf = grid(lay, scale), grid(lay, scale), grid(clay)
        prc.fill(L.ALL_POINTS, L.FUNC_SINE, L.FUNC_SINE, L.FUNC_SINE, L.PI, L.PI, L.PI, 0.5)
        prn.fill(L.ALL_POINTS, L.FUNC_SINE, L.FUNC_SINE, L.FUNC_SINE, L.PI, L.PI, L.PI, 0.49)
        cf.fill(L.INNER_POINTS, 2.0e-6)
        us = timed_once(lambda: prn.computePressureWithFD(prc, cf, order))
        out.append({"kernel": "computePressureWithFD", "order": order, "wave": prec, "coef": coef,
                    "us": us})

    def laplacian(order):
        lay = L.b200_layout(3, n, n, n, order=order, prec="f32")
        U, W = grid(lay), grid(lay)
        U.fill(L.ALL_POINTS, L.FUNC_SINE, L.FUNC_SINE, L.FUNC_SINE, L.PI * 4, L.PI * 6, L.PI * 8, 1.0)
        us = timed_once(lambda: U.FD_LAPLACIAN(L.INNER_POINTS, W, order))
        out.append({"kernel": "FD_LAPLACIAN", "order": order, "wave": "f32", "us": us})

    for o in orders:
        pressure(o, "f32", "f32", 1.0)
    for o in orders:
        laplacian(o)
    pressure(orders[0], "f16", "f32", 16.0)
    st = ctypes_status()
    if st:
        raise RuntimeError(f"device-side error word {st}")
    print(json.dumps({"workload": f"one launch per hot kernel, {n}^3", "launches": out,
                      "note": "single cold launches for a profiler; bench figures come from the "
                              "other workloads"}))


def dropin_arm(a):
    """hpcscan's own Propa test case, unchanged, on -testMode B200 (hpcscan_b200/host/bin): its
    'Best Gpoint/s in FD' (inner points x steps / the propagator's compute-pressure timer, a host
    wall clock around each computePressureWithFD call that Grid_B200 ends with a device
    synchronisation; src/propagator_Ac2.cpp:379-389, src/testCase_Propa.cpp:192), one try (the
    timer accumulates over tries), the analytic check every --snap steps. Beside it the same
    step timed on the device through the Python API, so the cost of the per-call
    synchronisation and host timer is visible."""
    exe = os.path.join(REPO, "hpcscan_b200", "host", "bin", "hpcscan_b200_fp32")
    n, order, nt = a.size, a.order, a.nt or 200
    snap = a.snap or 50
    args = [exe, "-testCase", "Propa", "-testMode", "B200", "-propagator", a.propagator,
            "-fdOrder", str(order), "-n1", str(n), "-n2", str(n), "-n3", str(n),
            "-ratioCFL", "0.8", "-nt", str(nt), "-snapInc", str(snap), "-ntry", "1"]
    with tempfile.TemporaryDirectory() as d:
        out = subprocess.run(args, cwd=d, capture_output=True, text=True, timeout=900)
    if out.returncode != 0 or "TERMINATED SUCCESSFULLY" not in out.stdout:
        raise RuntimeError(out.stdout[-2000:] + out.stderr[-2000:])

    def grab(pat):
        m = re.findall(pat, out.stdout)
        return float(m[-1]) if m else None
    fd = grab(r"Best Gpoint/s in FD\s+(\S+)")
    det = {"best_gpoint_s_in_fd": fd, "best_gpoint_s_eff": grab(r"Best Gpoint/s eff\.\s+(\S+)"),
           "compute_pressure_s": grab(r"Compute pres\. time \(s\)\s+(\S+)"),
           "boundary_condition_s": grab(r"Bound\. cond\. time \(s\)\s+(\S+)"),
           "err_test_case": grab(r"errTestCase2\s+(\S+)"),
           "passed": "Test PASSED" in out.stdout}
    # the same launches on the device clock, through the Python API
    import torch

    from hpcscan_b200 import layout as L
    from hpcscan_b200.grid import init_device
    from hpcscan_b200.propagator import Propagator_Ac2
    init_device(0)
    lay = L.b200_layout(3, n, n, n, order=order, prec="f32")
    propa = Propagator_Ac2(lay)
    propa.initialize(ratio_cfl=0.8, nt=1, snap_inc=1, modes=(1, 1, 1))
    prn, prc = propa.prnGrid, propa.prcGrid
    for _ in range(3):
        propa.computePressureWithFD(prn, prc)
    sec = _timed(lambda: propa.computePressureWithFD(prn, prc), reps=nt)
    dev = lay.inner_points / sec / 1e9
    host_us = det["compute_pressure_s"] / nt * 1e6 if det["compute_pressure_s"] else None
    line = {
        "metric": f"Propa 'Best Gpoint/s in FD' through hpcscan's own driver (O{order} FP32 {n}^3)",
        "value": fd, "unit": "GPoint/s", "n_gpus": 1, "steps": nt, "warmup": 0,
        "ms_per_step": round(host_us / 1e3, 5) if host_us else None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (eigen mode, the reference's Propa initialisation)",
        "config": {"workload": f"hpcscan -testCase Propa -testMode B200 O{order} {n}^3 {nt} steps",
                   "n": n, "order": order, "nt": nt, "snap_inc": snap,
                   "command": " ".join(["hpcscan_b200_fp32"] + args[1:])},
        "driver": det,
        "device_timed_gpoint_s": round(dev, 2),
        "device_us_per_call": round(sec * 1e6, 2),
        "driver_us_per_call": round(host_us, 2) if host_us else None,
        "gpu_launches": None,
    }
    print(json.dumps(line))


def sustained_arm(a):
    """The headline step (boundary condition + pressure update, 512^3 O8 FP32 eigen mode) run
    back to back for --nt steps (default 3000, about 1.3 s), timed in bins of 100 steps with
    CUDA events, with the SM clock, board power and clock-event reasons sampled through NVML in
    each bin. On a 1000 W B200 this shows the power cap: after about 100 ms of back-to-back
    steps the SM clock falls below its maximum (reason sw_power_cap) and the step time rises
    with it, since the kernel's time follows the SM clock at that point."""
    import torch

    from hpcscan_b200 import layout as L
    from hpcscan_b200.grid import init_device
    from hpcscan_b200.propagator import Propagator_Ac2

    init_device(0)
    lay = L.b200_layout(3, a.size, a.size, a.size, order=a.order, prec="f32")
    propa = Propagator_Ac2(lay)
    propa.initialize(ratio_cfl=0.8, nt=1, snap_inc=1, modes=(1, 1, 1))
    prn, prc = propa.prnGrid, propa.prcGrid
    stream = torch.cuda.current_stream()
    bin_steps = 100
    nbins = max(1, (a.nt or 3000) // bin_steps)
    nt = nbins * bin_steps

    def step():
        nonlocal prn, prc
        prc.applyBoundaryCondition()
        propa.computePressureWithFD(prn, prc)
        prn, prc = prc, prn

    bins = []
    with ClockSampler(torch.cuda.current_device()) as clk:
        for _ in range(a.warmup):
            step()
        torch.cuda.synchronize()
        time.sleep(1.0)                  # the board back at rest after the set-up
        for _ in range(nbins):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(stream)
            for _ in range(bin_steps):
                step()
            e1.record(stream)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            bins.append((e0.elapsed_time(e1) / bin_steps, clk.between(t0, t1)))
    st = ctypes_status()
    if st:
        raise RuntimeError(f"device-side error word {st}")
    pts = lay.inner_points
    total_ms = sum(ms for ms, _ in bins) * bin_steps
    tail = bins[len(bins) // 2:]
    seen = sorted({r for _, c in bins for r in c["reasons"]})
    line = {
        "metric": f"Propa GPoint/s sustained (O{a.order} FP32 {a.size}^3, {nt} back-to-back steps)",
        "value": round(pts * nt / (total_ms * 1e-3) / 1e9, 4), "unit": UNIT, "n_gpus": 1,
        "steps": nt, "warmup": a.warmup, "ms_per_step": round(total_ms / nt, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (eigen mode, the reference's Propa initialisation)",
        "config": {"workload": f"Propa Ac2Standard O{a.order} FP32 {a.size}^3 eigen mode, "
                               "steps back to back, timed in bins", "bin_steps": bin_steps,
                   "l2": "inputs larger than L2"},
        "gpu_launches": (2 if min(lay.n_inner) >= 2 * lay.halo + 2 else 3) * nt,
        "first_bin": {"ms_per_step": round(bins[0][0], 5), **bins[0][1]},
        "second_half": {"ms_per_step": round(statistics.mean(ms for ms, _ in tail), 5),
                        "sm_mhz": statistics.median([c["sm_mhz"] for _, c in tail
                                                     if c["sm_mhz"] is not None] or [0]),
                        "power_w_max": max([c["power_w"] for _, c in tail
                                            if c["power_w"] is not None] or [0])},
        "reasons_seen": seen,
        "bins": [[round(ms, 5), c["sm_mhz"], c["power_w"], c["reasons"]] for ms, c in bins],
        "bins_columns": ["ms_per_step", "sm_mhz (median)", "power_w (NVML running average)",
                         "reasons"],
    }
    print(json.dumps(line))


def ctypes_status():
    """The library's device-side error word (non-zero: a bounded wait ran out)."""
    import ctypes

    from hpcscan_b200 import _lib
    st = ctypes.c_int()
    _lib.call("b200_device_status", ctypes.byref(st), 1)
    return st.value


def main():
    a = parse_args()
    if a.workload != "propa":
        rank, world, _ = dist_env()
        if a.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no "
                                  "adjoint and no batched modelling path (fd: its CacheBlk "
                                  "numbers are in the b200 line; sustained: the reference CPU "
                                  "path of this step is the propa workload's reference line)"}))
            return
        if a.workload in ("adjoint", "modeling"):
            # shot-parallel: every rank runs its share of the survey
            {"adjoint": adjoint_arm, "modeling": modeling_arm}[a.workload](a)
            return
        if world > 1 and rank != 0:
            return
        {"mixed": mixed_arm, "fd": fd_arm, "fdsweep": fdsweep_arm, "dropin": dropin_arm,
         "launches": launches_arm, "sustained": sustained_arm}[a.workload](a)
        return
    if a.impl == "reference":
        reference_arm(a)
    elif a.impl == "reference-gpu":
        reference_gpu_arm(a)
    else:
        b200_arm(a)


if __name__ == "__main__":
    main()
