"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the hpcscan reference CPU binaries (oracle/_ref/hpcscan_fp32|fp64, built
unchanged from the reference sources by oracle/Makefile) with -writeGrid on
small cases of the hot-path test cases FD_D2, FD_D1 and Propa, reads back the
grids they write (<name>.proc0.grid.bin / .grid.info, src/grid.cpp:1245-1287;
successive writes of one name are appended), and stores:

  fd_*.npz     U (full grid, reference layout) and the inner points of the W
               grid of each case (Axis1..3, Laplacian), plus the L1 errors the
               reference printed;
  fdd1_*.npz   the same for the staggered first derivative (cases Axis1..3);
  propa_*.npz  the inner points of prn at every check step, plus nt, dt and
               the reference's errTestCase.

Re-run with:  python tests/golden/make_golden.py   (needs oracle/_ref built)
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from hpcscan_b200.layout import reference_layout  # noqa: E402

BIN = {"f32": os.path.join(REPO, "oracle", "_ref", "hpcscan_fp32"),
       "f64": os.path.join(REPO, "oracle", "_ref", "hpcscan_fp64")}

# name, prec, dim, (n1, n2, n3), order, extra flags
FD_CASES = [
    ("fd3_o8_k234", 3, (20, 22, 24), 8, ["-param1", "4", "-param2", "6", "-param3", "8",
                                         "-param4", "1"]),
    ("fd3_27x36x41_o8", 3, (27, 36, 41), 8, []),
    ("fd2_o4", 2, (20, 21, 1), 4, []),
    ("fd1_o16", 1, (30, 1, 1), 16, []),
    ("fd3_autopad_o6", 3, (21, 20, 20), 6, ["-autoPad"]),
    ("fd3_addpad_o10", 3, (20, 21, 20), 10, ["-n1AddPad", "3", "-n2AddPad", "2",
                                              "-n3AddPad", "1"]),
    ("fd3_mulpad_o14", 3, (20, 20, 21), 14, ["-n1MulPad", "8", "-n2MulPad", "5",
                                              "-n3MulPad", "3"]),
] + [(f"fd3_all_o{o}", 3, (20, 21, 22), o, []) for o in (2, 4, 6, 8, 10, 12, 14, 16)]

# cases kept for both precisions; the others are stored in FP32 only
FD_F64 = {"fd3_o8_k234", "fd2_o4", "fd1_o16", "fd3_all_o4", "fd3_all_o12",
          "fd3_all_o16"}
# the order sweep stores Axis1 and the Laplacian only (Axis2/3 are covered above)
FD_SWEEP_CASES = ("Axis1", "Laplacian3D")

# FD_D1 (src/testCase_FD_D1.cpp): name, dim, (n1, n2, n3), order, extra flags
FDD1_CASES = [
    ("fdd1_3d_o8", 3, (20, 22, 24), 8, ["-param1", "3", "-param2", "5", "-param3", "7"]),
    ("fdd1_2d_o6", 2, (20, 21, 1), 6, []),
    ("fdd1_1d_o16", 1, (30, 1, 1), 16, []),
    ("fdd1_3d_autopad_o12", 3, (21, 20, 23), 12, ["-autoPad"]),
] + [(f"fdd1_3d_o{o}", 3, (20, 20, 21), o, []) for o in (2, 4, 6, 10, 14, 16)]
FDD1_F64 = {"fdd1_3d_o8", "fdd1_1d_o16", "fdd1_3d_o4", "fdd1_3d_o16"}

PROPA_CASES = [
    ("propa3_o8", 3, (20, 20, 20), 8, "Ac2Standard",
     ["-ratioCFL", "0.8", "-param1", "1", "-param2", "1", "-param3", "1", "-nt", "21",
      "-snapInc", "10"]),
    ("propa3_o4_split", 3, (20, 21, 22), 4, "Ac2SplitComp", ["-nt", "11", "-snapInc", "5"]),
    ("propa3_o16", 3, (20, 21, 22), 16, "Ac2Standard", ["-nt", "9", "-snapInc", "4"]),
    ("propa2_o12", 2, (24, 25, 1), 12, "Ac2Standard", ["-nt", "31", "-snapInc", "15"]),
    ("propa1_o2", 1, (40, 1, 1), 2, "Ac2Standard", ["-nt", "31", "-snapInc", "10"]),
]


def parse_pad_flags(flags):
    kw = {"auto_pad": "-autoPad" in flags, "add_pad": [None] * 3, "mul_pad": [None] * 3}
    for i, f in enumerate(flags):
        m = re.match(r"-n([123])(Add|Mul)Pad", f)
        if m:
            a = int(m.group(1)) - 1
            kw["add_pad" if m.group(2) == "Add" else "mul_pad"][a] = int(flags[i + 1])
    kw["add_pad"] = tuple(kw["add_pad"])
    kw["mul_pad"] = tuple(kw["mul_pad"])
    return kw


def read_grids(d, name, prec):
    info = open(os.path.join(d, f"{name}.proc0.grid.info")).read().split()
    n1, n2, n3 = (int(x) for x in info[:3])
    raw = np.fromfile(os.path.join(d, f"{name}.proc0.grid.bin"),
                      dtype=np.float32 if prec == "f32" else np.float64)
    return raw.reshape(-1, n1 * n2 * n3), (n1, n2, n3)


def run(prec, args, d):
    out = subprocess.run([BIN[prec]] + args + ["-writeGrid", "-ntry", "1"], cwd=d,
                         capture_output=True, text=True, env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert out.returncode == 0, out.stderr
    return out.stdout


def gen_fd(manifest):
    for name, dim, n, order, extra in FD_CASES:
        for prec in (("f32", "f64") if name in FD_F64 else ("f32",)):
            with tempfile.TemporaryDirectory() as d:
                args = ["-testCase", "FD_D2", "-testMode", "Baseline", "-dim", str(dim),
                        "-fdOrder", str(order), "-n1", str(n[0]), "-n2", str(n[1]),
                        "-n3", str(n[2])] + extra
                txt = run(prec, args, d)
                errs = [float(x) for x in re.findall(r"Test PASSED / L1 err\.\s+(\S+)", txt)] + \
                       [float(x) for x in re.findall(r"Test FAILED! / L1 err\.\s+(\S+)", txt)]
                lay = reference_layout(dim, *n, order=order, prec=prec, **parse_pad_flags(extra))
                U, shp = read_grids(d, "FD_D2U", prec)
                assert shp == (lay.n1, lay.n2, lay.n3), (shp, lay)
                cases = ["Axis1", "Axis2", "Axis3"][:dim] + [f"Laplacian{dim}D"]
                if name.startswith("fd3_all_"):
                    cases = list(FD_SWEEP_CASES)
                # U (the separable fill) is pinned by the non-sweep cases only
                arrs = {} if name.startswith("fd3_all_") else {"U": U[0]}
                for c in cases:
                    W, _ = read_grids(d, f"FD_D2{c}W", prec)
                    arrs[c] = np.ascontiguousarray(lay.inner(W[0]))
                fn = f"{name}_{prec}.npz"
                np.savez_compressed(os.path.join(HERE, fn), **arrs)
                manifest[fn] = {"kind": "FD_D2", "prec": prec, "dim": dim, "n": n, "order": order,
                                "flags": extra, "cases": cases, "l1_err": errs}
                print(fn, errs)


def gen_fd_d1(manifest):
    for name, dim, n, order, extra in FDD1_CASES:
        for prec in (("f32", "f64") if name in FDD1_F64 else ("f32",)):
            with tempfile.TemporaryDirectory() as d:
                args = ["-testCase", "FD_D1", "-testMode", "Baseline", "-dim", str(dim),
                        "-fdOrder", str(order), "-n1", str(n[0]), "-n2", str(n[1]),
                        "-n3", str(n[2])] + extra
                txt = run(prec, args, d)
                errs = [float(x) for x in
                        re.findall(r"Test (?:PASSED|FAILED!) / L1 err\.\s+(\S+)", txt)]
                lay = reference_layout(dim, *n, order=order, prec=prec, **parse_pad_flags(extra))
                U, shp = read_grids(d, "FD_D1U", prec)
                assert shp == (lay.n1, lay.n2, lay.n3), (shp, lay)
                cases = ["Axis1", "Axis2", "Axis3"][:dim]
                arrs = {"U": U[0]}
                for c in cases:
                    W, _ = read_grids(d, f"FD_D1{c}W", prec)
                    arrs[c] = np.ascontiguousarray(lay.inner(W[0]))
                fn = f"{name}_{prec}.npz"
                np.savez_compressed(os.path.join(HERE, fn), **arrs)
                manifest[fn] = {"kind": "FD_D1", "prec": prec, "dim": dim, "n": n, "order": order,
                                "flags": extra, "cases": cases, "l1_err": errs}
                print(fn, errs)


def gen_propa(manifest):
    for name, dim, n, order, propa, extra in PROPA_CASES:
        for prec in ("f32", "f64"):
            with tempfile.TemporaryDirectory() as d:
                args = ["-testCase", "Propa", "-testMode", "Baseline", "-dim", str(dim),
                        "-fdOrder", str(order), "-n1", str(n[0]), "-n2", str(n[1]),
                        "-n3", str(n[2]), "-propagator", propa] + extra
                txt = run(prec, args, d)
                err = float(re.search(r"errTestCase2\s+(\S+)", txt).group(1))
                nt = int(re.search(r"No\. time steps\s+(\S+)", txt).group(1))
                dt = float(re.search(r"Time step \(s\)\s+(\S+)", txt).group(1))
                checks = [float(x) for x in re.findall(r"Check at time\s+(\S+)", txt)]
                lay = reference_layout(dim, *n, order=order, prec=prec)
                P, shp = read_grids(d, "PropaEigenModePrn", prec)
                assert shp == (lay.n1, lay.n2, lay.n3)
                arrs = {f"prn_{i}": np.ascontiguousarray(lay.inner(P[i])) for i in range(len(P))}
                fn = f"{name}_{prec}.npz"
                np.savez_compressed(os.path.join(HERE, fn), **arrs)
                manifest[fn] = {"kind": "Propa", "prec": prec, "dim": dim, "n": n, "order": order,
                                "propagator": propa, "flags": extra, "nt": nt, "dt": dt,
                                "check_times": checks, "err_test_case": err}
                print(fn, nt, dt, err, len(P))


def main():
    manifest = {}
    gen_fd(manifest)
    gen_fd_d1(manifest)
    gen_propa(manifest)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
