"""The C++ driver (cfd_b200_solver): the reference program on the library.

CPU: input errors are reported with exit status 1 before any device is touched.
GPU: on the same INP.DAT and parameters it writes the same output files, byte for byte,
as the Python Solver mirror (both sit on the same C ABI), and prints one "loop dmax"
line per step as the reference does (PSolver.cpp:1890).
"""
import subprocess
from pathlib import Path

import pytest

from cfd_solver_b200.grid import ogrid, cavity, write_inp

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "cfd_solver_b200" / "cfd_b200_solver"

needs_exe = pytest.mark.skipif(not EXE.exists(), reason="driver not built (make -C cfd_solver_b200/csrc)")


@needs_exe
def test_bad_input_exits_1(tmp_path):
    r = subprocess.run([str(EXE), str(tmp_path / "missing.dat")], capture_output=True, text=True)
    assert r.returncode == 1 and "cannot open" in r.stderr
    bad = tmp_path / "INP.DAT"
    bad.write_text("33 25 0.03125 0.04\n1 1 2\n")
    r = subprocess.run([str(EXE), str(bad)], capture_output=True, text=True)
    assert r.returncode == 1 and ("truncated" in r.stderr or "bad header" in r.stderr)
    r = subprocess.run([str(EXE), "--profile", "sphere"], capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr
    for bad_args in (["--steps", "-5"], ["--steps", "2.5"], ["--steps", "1e12"], ["--out-every", "-1"],
                     ["--Re"], ["--Re", "abc"], ["--precision", "fp16"], ["--unknown"]):
        r = subprocess.run([str(EXE), *bad_args], capture_output=True, text=True)
        assert r.returncode == 1 and "usage" in r.stderr, bad_args


@needs_exe
@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["ogrid", "cavity"])
def test_driver_outputs_match_python_solver(tmp_path, kind):
    from cfd_solver_b200.solver import Solver
    g = ogrid(33, 25, skew=0.1) if kind == "ogrid" else cavity(33, 33, skew=0.1)
    a, b = tmp_path / "cpp", tmp_path / "py"
    a.mkdir()
    b.mkdir()
    write_inp(g, a / "INP.DAT")
    write_inp(g, b / "INP.DAT")
    phys = dict(Re=200.0, Ri=1.0, Pr=0.71, dt=1e-3)
    r = subprocess.run([str(EXE), str(a / "INP.DAT"), "--steps", "101", "--Re", "200", "--Ri", "1",
                        "--Pr", "0.71", "--dt", "1e-3", "--profile", kind, "--dir", str(a)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 101 and lines[0].startswith("0 ") and lines[-1].startswith("100 ")
    s = Solver(b / "INP.DAT", profile=kind, **phys)
    s.timeLoop(101)
    s.close()
    for f in ("spt100.dat", "COEFF_HIS.dat", "COEFF_HIS_pr_vor.dat", "SURF_DIST.dat"):
        assert (a / f).read_bytes() == (b / f).read_bytes(), f
