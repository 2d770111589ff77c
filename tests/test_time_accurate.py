"""Time-accurate mode (`time_accurate = 1`): the oscillating cylinder of PSolver.cpp:1617-1630.

The reference keeps its time as an int (PSolver.cpp:186), so with dt < 1 the wall motion
cos(2 pi F t) always sees t = 0: the cylinder turns at a constant rate instead of
oscillating. In time-accurate mode the time is a double, t = n dt, and the wall velocity and
the wall acceleration of the boundary pressure follow it. The oracle carries the same switch;
with it off, both keep the reference's behaviour (the golden fixtures cover that).
"""
import math

import numpy as np
import pytest

from cfd_solver_b200.grid import ogrid

F, DT, STEPS = 5.0, 1e-2, 8


def _wall_u(speed_amp_scale, y0, t):
    return -speed_amp_scale * math.cos(2.0 * math.pi * F * t) * y0


def test_oracle_wall_follows_the_double_time():
    from oracle import oracle
    g = ogrid(24, 20, ar=1.0)
    amp = (math.pi / 12.0) * 2.0 * math.pi * F  # thetamax * 2 pi F (PSolver.cpp:176-179)
    for acc in (0, 1):
        ref = oracle.OracleCase(g, Re=50.0, F=F, dt=DT, time_accurate=acc)
        d = ref.step(STEPS)
        u = ref.field("u")
        t = STEPS * DT if acc else 0.0
        want = np.array([_wall_u(amp, g.y[0, i], t) for i in range(g.n0)])
        np.testing.assert_allclose(u[0], want, rtol=1e-12, atol=1e-14)
        assert d["time"][-1] == pytest.approx(t if acc else int(STEPS * DT), abs=1e-12)


@pytest.mark.gpu
def test_gpu_time_accurate_matches_oracle():
    from test_gpu_parity import REL, rel_l2, run_pair
    g = ogrid(33, 25, skew=0.1)
    phys = dict(Re=100.0, Ri=0.5, F=F, dt=DT, time_accurate=1)
    gpu, ref, st, d = run_pair(g, phys, STEPS, fields=("u", "v", "T", "p"))
    assert st["status"] == 0
    for k in gpu:
        assert rel_l2(gpu[k], ref[k]) < REL, k
    # the stats carry the double time; the wall moved with cos(2 pi F t)
    assert st["time"] == pytest.approx(STEPS * DT, abs=1e-12)
    amp = (math.pi / 12.0) * 2.0 * math.pi * F
    want = np.array([_wall_u(amp, g.y[0, i], STEPS * DT) for i in range(g.n0)])
    np.testing.assert_allclose(gpu["u"][0], want, rtol=1e-12, atol=1e-13)


@pytest.mark.gpu
def test_gpu_int_time_keeps_the_reference_behaviour():
    from cfd_solver_b200.solver import Batch, case_params
    g = ogrid(33, 25, skew=0.1)
    with Batch([g], [case_params(g, Re=100.0, F=F, dt=DT)]) as b:
        b.step(STEPS)
        st = b.stats(0)
        u = b.plane(0, "u")
    assert st["time"] == 0.0  # int(n * 0.01) truncated every step, as the reference
    amp = (math.pi / 12.0) * 2.0 * math.pi * F
    want = np.array([_wall_u(amp, g.y[0, i], 0.0) for i in range(g.n0)])
    np.testing.assert_allclose(u[0], want, rtol=1e-12, atol=1e-13)
