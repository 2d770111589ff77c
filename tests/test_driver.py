"""The C++ driver (cfd_b200_solver): the reference program on the library.

CPU: input errors are reported with exit status 1 before any device is touched.
GPU: on the same INP.DAT and parameters it writes the same output files, byte for byte,
as the Python Solver mirror (both sit on the same C ABI), and prints one "loop dmax"
line per step as the reference does (PSolver.cpp:1890). Its files also agree with the
files the compiled reference itself (oracle/_ref/cfd_ref) writes for the same INP.DAT,
both run with tight inner tolerances, to the precision of each file's format.
"""
import subprocess
from pathlib import Path

import numpy as np
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
                     ["--Re"], ["--Re", "abc"], ["--precision", "fp16"], ["--unknown"],
                     ["--maxit-mom", "1"], ["--maxit-p", "0"], ["--atol-p", "x"]):
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


def _spt(path):
    """spt100.dat (PSolver.cpp:1991-2004): header lines, then x y u v T p si vort per point."""
    a = np.loadtxt(path, skiprows=3)
    return {k: a[:, m] for m, k in enumerate(("x", "y", "u", "v", "T", "p", "si", "vort"))}


@needs_exe
@pytest.mark.gpu
def test_driver_outputs_match_compiled_reference(tmp_path):
    """The driver's four files against the reference program's own, 101 steps of an O-grid.

    Both sides converge every inner solve tightly (the reference through its relative rule
    at 1e-13 / 1e-12, the library with an absolute floor as well), so each step depends on
    the discretisation only. spt100.dat carries 13 significant digits: u, v, T, p, si and
    vort agree within 1e-8 relative L2. COEFF_HIS*.dat carry 8 decimals (Cl, Cd, Cm, Nu and
    their pressure / viscous parts): within two units of the last decimal. SURF_DIST.dat
    carries 6 significant digits (%g): within one unit of the sixth digit.
    """
    from oracle import refrun
    try:
        refrun.binary()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    g = ogrid(33, 25, skew=0.1)
    steps = 101
    ref = refrun.run(g, steps, params=dict(Re=100.0, Ri=1.0, dt=1e-3, tol_gs=1e-13, maxit_gs=600,
                                           tol_sip=1e-12, maxit_sip=6000), timeout=600)
    write_inp(g, tmp_path / "INP.DAT")
    r = subprocess.run([str(EXE), str(tmp_path / "INP.DAT"), "--steps", str(steps), "--Re", "100", "--Ri", "1",
                        "--dt", "1e-3", "--tol-mom", "1e-13", "--atol-mom", "1e-13", "--maxit-mom", "600",
                        "--tol-p", "1e-12", "--atol-p", "1e-12", "--maxit-p", "600", "--quiet",
                        "--dir", str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    (tmp_path / "ref").mkdir()
    for name, text in ref["files"].items():
        (tmp_path / "ref" / name).write_text(text)
    a, b = _spt(tmp_path / "spt100.dat"), _spt(tmp_path / "ref" / "spt100.dat")
    np.testing.assert_allclose(a["x"], b["x"], rtol=0, atol=1e-9)
    for k in ("u", "v", "T", "p", "si", "vort"):
        err = np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b[k])
        assert err < 1e-8, f"spt100.dat {k}: rel L2 {err:.3e}"
    for name in ("COEFF_HIS.dat", "COEFF_HIS_pr_vor.dat"):
        ha = np.loadtxt(tmp_path / name, ndmin=2)
        hb = np.loadtxt(tmp_path / "ref" / name, ndmin=2)
        assert ha.shape == hb.shape == (2, 5), name
        np.testing.assert_allclose(ha, hb, rtol=0, atol=2e-8, err_msg=name)
    sa = np.loadtxt(tmp_path / "SURF_DIST.dat")
    sb = np.loadtxt(tmp_path / "ref" / "SURF_DIST.dat")
    assert sa.shape == sb.shape == (g.n0, 4)
    for m in range(4):
        scale = np.abs(sb[:, m]).max()
        np.testing.assert_allclose(sa[:, m], sb[:, m], rtol=1.1e-5, atol=1e-9 * scale,
                                   err_msg=f"SURF_DIST col {m}")
