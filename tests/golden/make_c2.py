"""Golden fixed-step state of the 513 x 513 benchmark configuration (O-grid twin), from the oracle.

The reference's own geometry (elliptic O-grid, aspect ratio 2, outer radius 20) at the
configuration's size and skew (513 x 513, skew 0.15, Re 400, Ri 1, Pr 0.71, the
reference's dt 1e-4 and flow angle) is advanced 2 steps by the FP64 CPU restatement
(oracle/cfd_oracle.c, bit-identical to the compiled reference on this profile) with tight
inner tolerances (1e-10), so the step depends on the discretisation only. The fixture
keeps every 8th point of u, v, T, p (65 x 65), the full-field L2 norms and Nu, dmax, Cl.

    python tests/golden/make_c2.py      # writes tests/golden/c2_twin513_2steps.npz (~5 minutes)
"""
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from cfd_solver_b200.workloads import CONFIGS, make_case  # noqa: E402
from oracle import oracle  # noqa: E402

STEPS = 2
TIGHT = dict(tol_gs=1e-10, maxit_gs=20000, tol_sip=1e-10, maxit_sip=20000)


def main():
    c = CONFIGS["c2"]
    g, prm = make_case(dict(N=c["N"], skew=c["skew"], Re=c["Re"], Ri=c["Ri"], Pr=c["Pr"]), "twin")
    t0 = time.time()
    o = oracle.OracleCase(g, **prm, **TIGHT)
    d = o.step(STEPS)
    out = {}
    for k in ("u", "v", "T", "p"):
        f = o.field(k)
        out[k + "_sub"] = f[::8, ::8].copy()
        out[k + "_l2"] = float(np.linalg.norm(f))
    out.update(nu=d["nu"][-1], dmax=d["dmax"][-1], cl=d["cl"][-1], steps=STEPS)
    np.savez_compressed(Path(__file__).with_name("c2_twin513_2steps.npz"), **out)
    print(f"{STEPS} steps in {time.time() - t0:.0f} s, Nu {out['nu']:.12f}")


if __name__ == "__main__":
    main()
