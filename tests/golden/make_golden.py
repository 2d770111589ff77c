"""Generate the golden fixtures under tests/golden/ from the compiled reference.

Runs the reference's own solver (oracle/_ref/cfd_ref, built from s.cpp by
oracle/build_ref.sh) on generated INP.DAT grids and stores its final fields,
per-step diagnostics and (for one case) its assembled coefficient planes.
Entries the reference never assigns (us/vs on the boundary rows, q on the seam
column, 4th-order coefficients on the 9-point rows) are stored as NaN.

    python tests/golden/make_golden.py        # needs the compiled reference (oracle/build_ref.sh)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from cfd_solver_b200.grid import ogrid  # noqa: E402
from oracle import refrun  # noqa: E402

OUT = Path(__file__).resolve().parent

# (name, grid kwargs, params, steps, planes kept, coefficient dump)
CASES = [
    ("og33x25_re100_ri1", dict(n0=33, n1=25, skew=0.1),
     dict(Re=100.0, Ri=1.0, dt=1e-3), 5, None, True),
    ("og41x33_ar3_tight", dict(n0=41, n1=33, ar=3.0, skew=0.15),
     dict(Re=400.0, Ri=2.0, Pr=7.0, dt=5e-4, tol_gs=1e-10, maxit_gs=400, tol_sip=1e-10,
          maxit_sip=2000), 3, None, False),
    ("og24x20_circle_rot", dict(n0=24, n1=20, ar=1.0, skew=0.0),
     dict(Re=50.0, Ri=0.5, F=0.3, alpha=30.0, dt=2e-3), 6, None, False),
    ("og65x65_refdefaults", dict(n0=65, n1=65, skew=0.1), dict(), 3,
     ("u", "v", "T", "p", "pcor", "q", "vort", "up", "vp"), False),
]

COEF_4TH = {"auee", "auww", "aunn", "auss", "aunnee", "aunnww", "aussee", "aussww", "aunne",
            "aunnw", "ausse", "aussw", "aunee", "aunww", "ausee", "ausww"}


def mask_unassigned(name, a, n0, n1, coef=False):
    a = a.copy()
    if coef:
        a[0, :] = np.nan
        a[n1 - 1, :] = np.nan
        base = name if name.startswith("au") else "au" + name[2:]
        if name.startswith(("au", "at")) and base in COEF_4TH:
            a[1, :] = np.nan
            a[n1 - 2, :] = np.nan
        return a
    if name in ("us", "vs"):
        a[0, :] = np.nan
        a[n1 - 1, :] = np.nan
    if name == "q":
        a[0, :] = np.nan
        a[n1 - 1, :] = np.nan
        a[:, n0 - 1] = np.nan
    return a


def main():
    index = {}
    for name, gkw, prm, steps, keep, coef in CASES:
        g = ogrid(**gkw)
        r = refrun.run(g, steps, prm, coef=coef)
        arrays = {}
        for k, v in r["fields"].items():
            if keep is None or k in keep:
                arrays["f_" + k] = mask_unassigned(k, v, g.n0, g.n1)
        for k, v in r["diag"].items():
            arrays["d_" + k] = v
        if coef:
            for k, v in r["coef"].items():
                arrays["c_" + k] = mask_unassigned(k, v, g.n0, g.n1, coef=True)
        np.savez_compressed(OUT / f"{name}.npz", **arrays)
        index[name] = dict(grid=gkw, params=prm, steps=steps)
        print(name, "ok", f"{r['wall_s']:.2f}s")
    (OUT / "cases.json").write_text(json.dumps(index, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main()
