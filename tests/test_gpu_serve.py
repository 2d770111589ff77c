"""Slots and continuous batching: a case admitted into a busy batch, or served in a
Poisson mix, gives the same bits as the same case run alone for the same steps."""
import numpy as np
import pytest

from cfd_solver_b200.grid import cavity, ogrid

pytestmark = pytest.mark.gpu


def test_admitted_case_equals_solo_run_bitwise():
    from cfd_solver_b200.solver import Batch, case_params
    gA, gB = ogrid(33, 25, skew=0.1), cavity(33, 33, skew=0.1)
    pA, pB = case_params(gA, Re=100.0, Ri=1.0, dt=1e-3), case_params(gB, Re=150.0, Ri=0.5, dt=2e-3)
    gX = cavity(33, 33, skew=0.05)
    pX = case_params(gX, Re=300.0, Ri=2.0, Pr=7.0, dt=1.5e-3)
    with Batch([gX], [pX]) as solo:
        solo.step(4)
        ref = {k: solo.plane(0, k) for k in ("u", "v", "T", "p")}
        ref_st = solo.stats(0)
    with Batch([gA, gB, gB], [pA, pB, pB]) as b:
        b.set_active(2, False)
        b.step(5)  # slots 0 and 1 run; slot 2 empty
        b.admit(2, gX, pX)
        b.step(4)
        got = {k: b.plane(2, k) for k in ("u", "v", "T", "p")}
        st = b.stats(2)
        others = b.all_stats()
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    assert st["steps"] == 4 and st["nu"] == ref_st["nu"]
    assert others[0]["steps"] == 9 and others[1]["steps"] == 9


def test_serve_results_equal_solo_runs():
    from cfd_solver_b200.solver import Batch, case_params, serve
    rng = np.random.default_rng(7)
    classes = [(cavity(33, 33, skew=0.1), 1)]
    reqs, cases = [], []
    t = 0.0
    for _ in range(6):
        t += rng.exponential(0.05)
        g = cavity(33, 33, skew=float(rng.uniform(0, 0.2)))
        prm = case_params(g, Re=float(rng.uniform(50, 200)), Ri=float(rng.uniform(0.1, 1.0)), dt=0.4 / 32)
        reqs.append((t, g, prm, 1e-3, 3000))
        cases.append((g, prm))
    results, stats = serve(reqs, classes, steps_per_tick=25, slots=[3])
    assert stats["converged"] == 6 and stats["slots"] == 3
    assert stats["p99_latency_s"] >= stats["p50_latency_s"] > 0
    for (g, prm), r in zip(cases, results):
        assert r["status"] == 0 and r["steady_res_rel"] <= 1e-3
        with Batch([g], [prm]) as solo:
            solo.step(r["steps"])
            assert solo.stats(0)["nu"] == r["nu"]
