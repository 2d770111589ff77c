"""Runner for the compiled reference solver (oracle/_ref/cfd_ref*) -- TEST INFRASTRUCTURE ONLY.

Only tests/, tests/golden/make_golden.py, bench.py's CPU-baseline leg and the
reference arm use this module. It runs the reference's own s.cpp, built by
oracle/build_ref.sh, on an INP.DAT written to a scratch directory, and reads
back the binary dumps described in oracle/ref_hooks.h.
"""
from __future__ import annotations

import os
import subprocess
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

# plane order of ref_dump() in ref_hooks.h
FIELD_NAMES = ("u", "v", "T", "p", "up", "vp", "us", "vs", "pcor", "q", "qu", "qv",
               "qt", "qup", "qvp", "si", "dil", "vort", "uxi", "uet")
COEF_NAMES = ("aup", "aue", "auw", "aun", "aus", "aune", "aunw", "ause", "ausw",
              "auee", "auww", "aunn", "auss", "aunnee", "aunnww", "aussee", "aussww",
              "aunne", "aunnw", "ausse", "aussw", "aunee", "aunww", "ausee", "ausww",
              "atp", "ate", "atw", "atn", "ats", "atne", "atnw", "atse", "atsw",
              "atee", "atww", "atnn", "atss", "atnnee", "atnnww", "atssee", "atssww",
              "atnne", "atnnw", "atsse", "atssw", "atnee", "atnww", "atsee", "atsww",
              "ap", "ae", "aw", "an", "as", "ane", "anw", "ase", "asw")
DIAG_NAMES = ("loop", "time", "dmax", "cl", "cd", "cm", "nu", "circ", "cl_pr", "cd_pr",
              "cl_vor", "cd_vor")

# physics / numerics parameter -> environment variable of the patched build
PARAM_ENV = {"Re": "CFD_RE", "Ri": "CFD_RI", "Pr": "CFD_PR", "F": "CFD_F",
             "alpha": "CFD_ALPHA", "dt": "CFD_DT", "tol_sip": "CFD_TOL_SIP",
             "maxit_sip": "CFD_MAXIT_SIP", "tol_gs": "CFD_TOL_GS", "maxit_gs": "CFD_MAXIT_GS"}


def binary(big: bool = False) -> Path:
    p = REF_DIR / ("cfd_ref_big" if big else "cfd_ref")
    if not p.exists():
        raise FileNotFoundError(f"{p} missing: run oracle/build_ref.sh")
    return p


def _read_dump(path: Path, names):
    raw = path.read_bytes()
    n0, n1, npl = np.frombuffer(raw[:12], dtype=np.int32)
    arr = np.frombuffer(raw[12:], dtype=np.float64).reshape(npl, n1, n0)
    assert npl == len(names), (npl, len(names))
    return {k: arr[i].copy() for i, k in enumerate(names)}


def run(grid, steps: int, params: dict | None = None, coef: bool = False,
        big: bool | None = None, timeout: float | None = None, keep_dir: str | None = None):
    """Run the reference for `steps` time steps; returns dict(fields, diag, coef, wall_s, files)."""
    from cfd_solver_b200.grid import write_inp

    params = dict(params or {})
    if big is None:
        big = grid.n0 > 350 or grid.n1 > 570
    exe = binary(big)
    with tempfile.TemporaryDirectory(prefix="cfdref_") as td:
        wd = Path(keep_dir) if keep_dir else Path(td)
        wd.mkdir(parents=True, exist_ok=True)
        write_inp(grid, wd / "INP.DAT")
        env = dict(os.environ)
        env["CFD_MAXSTEP"] = str(int(steps))
        env["CFD_DUMP"] = str(wd / "fields.bin")
        env["CFD_DIAG"] = str(wd / "diag.bin")
        if coef:
            env["CFD_DUMP_COEF"] = str(wd / "coef.bin")
        for k, v in params.items():
            env[PARAM_ENV[k]] = repr(float(v)) if not k.startswith("maxit") else str(int(v))
        t0 = time.perf_counter()
        subprocess.run([str(exe)], cwd=wd, env=env, check=True, stdout=subprocess.DEVNULL,
                       timeout=timeout)
        wall = time.perf_counter() - t0
        out = {"fields": _read_dump(wd / "fields.bin", FIELD_NAMES), "wall_s": wall}
        d = np.fromfile(wd / "diag.bin", dtype=np.float64).reshape(-1, len(DIAG_NAMES))
        out["diag"] = {k: d[:, i].copy() for i, k in enumerate(DIAG_NAMES)}
        if coef:
            out["coef"] = _read_dump(wd / "coef.bin", COEF_NAMES)
        out["files"] = {}
        for fn in ("spt100.dat", "COEFF_HIS.dat", "COEFF_HIS_pr_vor.dat", "SURF_DIST.dat"):
            if (wd / fn).exists():
                out["files"][fn] = (wd / fn).read_text()
        return out
