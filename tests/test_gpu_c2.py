"""Full-size parity: the 513 x 513 configuration (O-grid twin) against the oracle.

Two steps of the reference's geometry at 513 x 513 (skew 0.15, Re 400, Ri 1, Pr 0.71, dt
1e-4) with tight inner tolerances on both sides, against the fixture of
tests/golden/make_c2.py (FP64 CPU restatement, bit-identical to the compiled reference
on this profile). Bar 1e-8 relative: L2 of every 8th point and full-field L2 norms of
u, v, T, p; Nu, dmax and Cl.
"""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
FIX = Path(__file__).with_name("golden") / "c2_twin513_2steps.npz"
# absolute floors are L1 sums over the 262,656 unknown cells: 1e-9 is ~4e-15 per cell
TIGHT_GPU = dict(tol_mom=1e-13, atol_mom=1e-9, maxit_mom=2000, tol_p=1e-12, atol_p=1e-9, maxit_p=600)


@pytest.mark.skipif(not FIX.exists(), reason="golden 513 x 513 state not generated")
def test_twin513_two_steps_match_oracle():
    from cfd_solver_b200.solver import Batch, case_params
    from cfd_solver_b200.workloads import CONFIGS, make_case
    fx = np.load(FIX)
    c = CONFIGS["c2"]
    g, prm = make_case(dict(N=c["N"], skew=c["skew"], Re=c["Re"], Ri=c["Ri"], Pr=c["Pr"]), "twin")
    with Batch([g], [case_params(g, **prm, **TIGHT_GPU)]) as b:
        b.step(int(fx["steps"]))
        st = b.stats(0)
        f = {k: b.plane(0, k) for k in ("u", "v", "T", "p")}
    assert st["status"] == 0
    for k in ("u", "v", "T", "p"):
        sub = f[k][::8, ::8]
        rel = np.linalg.norm(sub - fx[k + "_sub"]) / np.linalg.norm(fx[k + "_sub"])
        assert rel < 1e-8, (k, rel)
        assert abs(np.linalg.norm(f[k]) - float(fx[k + "_l2"])) <= 1e-8 * float(fx[k + "_l2"]), k
    for k in ("nu", "dmax", "cl"):
        assert abs(st[k] - float(fx[k])) <= 1e-8 * max(abs(float(fx[k])), 1e-30), (k, st[k], float(fx[k]))
