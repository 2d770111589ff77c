"""Writers of the reference's output files, in its formats (PSolver.cpp:1989-2040).

  spt100.dat            Tecplot zone: x y (fixed, 9 decimals) then u v T p si vort
                        (scientific, 13 digits), rows j outer / i inner, a blank
                        line after every j row (PSolver.cpp:1991-2004)
  COEFF_HIS.dat         appended: time cl cd cm Nu (fixed, 8 decimals; time is an
                        int in the C++ reference) (PSolver.cpp:2018-2021)
  COEFF_HIS_pr_vor.dat  appended: time CL_pr CD_pr CL_vor CD_vor (PSolver.cpp:2023-2026)
  SURF_DIST.dat         xi p vort dT/dn on the wall j = 0, default stream format
                        (6 significant digits) (PSolver.cpp:2032-2039)
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np


def _g6(x: float) -> str:
    """C++ ostream default formatting of a double (%g with precision 6)."""
    s = f"{x:g}"
    return s


def write_spt(path, grid, f: dict) -> None:
    n0, n1 = grid.n0, grid.n1
    lines = ["zone", f"I={n0}", f"J={n1}"]
    u, v, T, p, si, vo = f["u"], f["v"], f["T"], f["p"], f["si"], f["vort"]
    for j in range(n1):
        for i in range(n0):
            lines.append(f"{grid.x[j, i]:.9f} {grid.y[j, i]:.9f} {u[j, i]:.13e} {v[j, i]:.13e} "
                         f"{T[j, i]:.13e} {p[j, i]:.13e} {si[j, i]:.13e} {vo[j, i]:.13e}")
        lines.append("")
    Path(path).write_text("\n".join(lines) + "\n")


def write_coeff_his(path, time, a: float, b: float, c: float, d: float) -> None:
    """One line: the reference's int time (PSolver.cpp:2018-2026), or the time as a fixed
    8-decimal value when it is a float (time-accurate mode)."""
    t = f"{time:.8f}" if isinstance(time, float) else f"{int(time)}"
    with open(path, "a") as fh:
        fh.write(f"{t} {a:.8f} {b:.8f} {c:.8f} {d:.8f}\n")


def write_surf_dist(path, grid, f: dict) -> None:
    T, p, vo = f["T"], f["p"], f["vort"]
    out = []
    for i in range(grid.n0):
        dthdn = -(4 * T[1, i] - 3 * T[0, i] - T[2, i]) / (2 * grid.dxi1)
        dthdn = dthdn * math.sqrt(grid.etx[0, i] * grid.etx[0, i] + grid.ety[0, i] * grid.ety[0, i])
        out.append(f"{_g6(i * grid.dxi0)} {_g6(p[0, i])} {_g6(vo[0, i])} {_g6(dthdn)}")
    Path(path).write_text("\n".join(out) + "\n")


def parse_spt(path) -> dict:
    """Read an spt100.dat back into (n1, n0) arrays x y u v T p si vort."""
    lines = Path(path).read_text().split("\n")
    n0 = int(lines[1].split("=")[1])
    n1 = int(lines[2].split("=")[1])
    rows = [ln.split() for ln in lines[3:] if ln.strip()]
    a = np.array(rows, dtype=np.float64).reshape(n1, n0, 8)
    return {k: a[..., m] for m, k in enumerate(("x", "y", "u", "v", "T", "p", "si", "vort"))}
