"""Converged-state parity: the GPU path run to its own steady state against the oracle's.

tests/golden/make_steady.py advanced the FP64 CPU restatement (bit-identical to the
compiled reference on the O-grid) until one step changes u, v and T by at most 1e-12 of
the first step's change, with every inner solve converged tightly. That state is the
discretisation's fixed point. Here the CUDA path starts from the same initial state and
steps until its own steady residual (the same ratio, `steady_res_rel`) meets the same
bar, with its own inner solvers (Chebyshev-Jacobi sweeps, multigrid-preconditioned
BiCGStab) converged as tightly. The two fixed points must agree:

  FP64 (the plain path):  u, v, T, p, stream function, vorticity and dilatation within
                          1e-8 relative L2; Nu within 1e-8 relative; Cl, Cd, Cm, their
                          pressure and viscous parts, the circulation and dmax within 1e-8
                          of their magnitude (magnitudes below 1e-2 count as 1e-2).
  precision form (FP32 sweeps and multigrid inside FP64 defect correction), run to a
                          steady residual of 1e-10: the same quantities within 1e-6 of the
                          FP64 oracle's. Its u/v/T solves stop at 1e-5 of their first
                          residual (an FP32 correction cannot go much below that); the
                          outer iteration still converges to the FP64 fixed point, because
                          each solve's right-hand side is the FP64 defect, which vanishes
                          there.

In the closed cavity the pressure is fixed only up to a constant (every boundary
condition of the pressure correction is a copy of its neighbour), so p is compared with
its mean over the grid removed on both sides, and the wall forces that integrate p over
the open bottom wall (Cl, Cd, Cm and their pressure parts) are not compared; their
viscous parts, Nu, the circulation and dmax are. The cavity has no reference
implementation; its fixtures are pinned to the restatement only.
"""
import importlib.util
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
_spec = importlib.util.spec_from_file_location("make_steady", GOLDEN / "make_steady.py")
make_steady = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(make_steady)

INNER_GPU = dict(tol_mom=1e-13, atol_mom=1e-11, maxit_mom=600, tol_p=1e-13, atol_p=1e-11, maxit_p=600)
INNER_MX = dict(INNER_GPU, tol_mom=1e-5, atol_mom=0.0)
FIELDS = ("u", "v", "T", "p", "si", "vort", "dil")
SCALARS = ("cl", "cd", "cm", "circ", "cl_pr", "cd_pr", "cl_vor", "cd_vor", "dmax")
PRESSURE_FORCES = ("cl", "cd", "cm", "cl_pr", "cd_pr")


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def run_to_steady(name, precision, stop):
    from cfd_solver_b200 import _lib
    from cfd_solver_b200.solver import Batch, case_params
    spec = make_steady.CASES[name]
    fix = np.load(GOLDEN / f"steady_{name}.npz")
    g = make_steady.grid_of(spec)
    inner = INNER_GPU if precision == _lib.PRECISION_FP64 else INNER_MX
    prm = case_params(g, precision=precision, **spec["phys"], **inner)
    cap = 2 * int(fix["steps"]) + 2000
    with Batch([g], [prm]) as b:
        steps = 0
        st = None
        while steps < cap:
            b.step(100)
            steps += 100
            st = b.stats(0)
            assert st["status"] == 0, (steps, st)
            if st["steady_res_rel"] <= stop:
                break
        assert st["steady_res_rel"] <= stop, (steps, st["steady_res_rel"])
        got = {k: b.plane(0, k) for k in FIELDS}
    ref = {k: fix[k] for k in FIELDS}
    if spec["kind"] == "cavity":
        got["p"] = got["p"] - got["p"].mean()
        ref["p"] = ref["p"] - ref["p"].mean()
    return got, ref, st, fix, steps


def check(got, ref, st, fix, bar, cavity):
    for k in FIELDS:
        err = rel_l2(got[k], ref[k])
        assert err < bar, f"{k}: rel L2 {err:.3e}"
    assert abs(st["nu"] - fix["nu"]) <= bar * abs(fix["nu"]), (st["nu"], float(fix["nu"]))
    for k in SCALARS:
        if cavity and k in PRESSURE_FORCES:
            continue
        r = float(fix[k])
        assert abs(st[k] - r) <= bar * max(abs(r), 1e-2), (k, st[k], r)


@pytest.mark.parametrize("name", list(make_steady.CASES))
def test_fp64_steady_state_matches_oracle(name):
    from cfd_solver_b200 import _lib
    got, ref, st, fix, steps = run_to_steady(name, _lib.PRECISION_FP64, make_steady.STOP)
    check(got, ref, st, fix, 1e-8, make_steady.CASES[name]["kind"] == "cavity")


@pytest.mark.parametrize("name", list(make_steady.CASES))
def test_precision_form_steady_state_matches_oracle(name):
    from cfd_solver_b200 import _lib
    got, ref, st, fix, steps = run_to_steady(name, _lib.PRECISION_MIXED, 1e-10)
    check(got, ref, st, fix, 1e-6, make_steady.CASES[name]["kind"] == "cavity")
