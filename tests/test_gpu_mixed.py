"""The precision form (CFD_PRECISION_MIXED) against the plain FP64 path.

In the precision form the u/v/T/up/vp sweeps run on an FP32 correction d for
A d = r, where r = rhs - A x0 is formed in FP64 and x = x0 + d afterwards (one
defect-correction pass per solve). The steady state is a fixed point of the step in
which every inner residual vanishes, so FP32 rounding of the corrections does not move
it: converged fields and Nu must agree with the FP64 path within 1e-6 relative L2 (the
precision form's accuracy bar). A few steps from rest agree to the FP32 rounding of the
update, which for a field that starts at zero is the field itself (bound 1e-5).
"""
import numpy as np
import pytest

from cfd_solver_b200.grid import cavity, ogrid

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _params(g, precision, **kw):
    from cfd_solver_b200 import _lib
    from cfd_solver_b200.solver import case_params
    return case_params(g, precision=precision, **kw)


def test_one_step_matches_fp64():
    from cfd_solver_b200 import _lib
    from cfd_solver_b200.solver import Batch
    cases = [(ogrid(65, 49, skew=0.1), dict(Re=300.0, Ri=1.0, dt=1e-3)),
             (cavity(65, 65, skew=0.12), dict(Re=200.0, Ri=0.5, Pr=7.0, dt=2e-3))]
    out = {}
    for prec in (_lib.PRECISION_FP64, _lib.PRECISION_MIXED):
        gs = [g for g, _ in cases]
        ps = [_params(g, prec, **kw) for g, kw in cases]
        with Batch(gs, ps) as b:
            b.step(3)
            out[prec] = [({k: b.plane(c, k) for k in ("u", "v", "T", "up", "vp", "p")}, b.stats(c))
                         for c in range(len(cases))]
    for (f64, s64), (fmx, smx) in zip(out[_lib.PRECISION_FP64], out[_lib.PRECISION_MIXED]):
        assert smx["status"] == 0
        assert smx["it_mom"] == s64["it_mom"]
        for k in f64:
            assert rel_l2(fmx[k], f64[k]) < 1e-5, k


def test_steady_state_matches_fp64():
    from cfd_solver_b200 import _lib
    from cfd_solver_b200.solver import Batch
    g = cavity(33, 33, skew=0.1)
    kw = dict(Re=100.0, Ri=1.0, Pr=0.71, dt=0.4 / 32)
    res = {}
    for prec in (_lib.PRECISION_FP64, _lib.PRECISION_MIXED):
        with Batch([g], [_params(g, prec, **kw)]) as b:
            st = None
            for _ in range(200):
                b.step(50)
                st = b.stats(0)
                if st["steady_res_rel"] <= 1e-9 or st["status"]:
                    break
            assert st["status"] == 0 and st["steady_res_rel"] <= 1e-9, st
            p = b.plane(0, "p")
            res[prec] = ({"u": b.plane(0, "u"), "v": b.plane(0, "v"), "T": b.plane(0, "T"),
                          "p": p - p[1:-1, 1:-1].mean()}, st)
    f64, s64 = res[_lib.PRECISION_FP64]
    fmx, smx = res[_lib.PRECISION_MIXED]
    for k in f64:
        assert rel_l2(fmx[k], f64[k]) < 1e-6, (k, rel_l2(fmx[k], f64[k]))
    assert abs(smx["nu"] - s64["nu"]) <= 1e-6 * abs(s64["nu"])


def test_precision_is_one_per_batch():
    from cfd_solver_b200 import _lib
    from cfd_solver_b200.solver import Batch
    g = cavity(17, 17)
    with pytest.raises(_lib.CfdError):
        Batch([g, g], [_params(g, _lib.PRECISION_FP64), _params(g, _lib.PRECISION_MIXED)])
