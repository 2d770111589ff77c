"""Golden steady state of the first benchmark configuration (cavity form), from the oracle.

The 65 x 65 skewed lid-driven cavity (skew 0.1, Re 100, Ri 1, Pr 0.71; dt from
workloads.cavity_dt) is advanced by the FP64 CPU restatement (oracle/cfd_oracle.c) with
tight inner tolerances (1e-10; at the reference's 0.75e-2, with its up/vp solves started
from zero every step, the step is never an exact fixed point and the steady residual
stalls near 1e-5) until the steady residual mean(|du| + |dv| + |dT|) / dt over the unknown
cells falls to 1e-12 of its first-step value. The steady state is the fixed point at which
every inner residual vanishes, so it does not depend on the inner solvers: the GPU path,
whose inner solvers differ, must reach the same fields.

    python tests/golden/make_c1.py      # writes tests/golden/c1_cavity65_steady.npz
"""
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from cfd_solver_b200.grid import cavity  # noqa: E402
from cfd_solver_b200.workloads import CONFIGS, cavity_dt  # noqa: E402
from oracle import oracle  # noqa: E402

TOL = 1e-12


def steady_res(o, prev, dt):
    cur = {k: o.field(k) for k in ("u", "v", "T")}
    d = sum(np.abs(cur[k][1:-1, 1:-1] - prev[k][1:-1, 1:-1]) for k in cur)
    return d.mean() / dt, cur


def main():
    c = CONFIGS["c1"]
    g = cavity(c["N"], c["N"], skew=c["skew"])
    dt = cavity_dt(c["N"], c["Ri"], c["Re"], c["Pr"])
    o = oracle.OracleCase(g, Re=c["Re"], Ri=c["Ri"], Pr=c["Pr"], dt=dt, tol_gs=1e-10, tol_sip=1e-10,
                          maxit_gs=5000, maxit_sip=20000)
    prev = {k: o.field(k) for k in ("u", "v", "T")}
    o.step(1)
    r0, prev = steady_res(o, prev, dt)
    steps, t0 = 1, time.time()
    rel = 1.0
    while rel > TOL and steps < 60000:
        o.step(99)
        prev = {k: o.field(k) for k in ("u", "v", "T")}
        d = o.step(1)
        steps += 100
        r, prev = steady_res(o, prev, dt)
        rel = r / r0
    p = o.field("p")
    out = dict(u=o.field("u"), v=o.field("v"), T=o.field("T"), p=p - p[1:-1, 1:-1].mean(),
               nu=d["nu"][-1], steps=steps, steady_res_rel=rel, dt=dt)
    np.savez_compressed(Path(__file__).with_name("c1_cavity65_steady.npz"), **out)
    print(f"{steps} steps, steady_res_rel {rel:.3e}, Nu {out['nu']:.12f}, {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
