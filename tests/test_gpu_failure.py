"""Failure statuses, made on the host or with iteration caps -- no GPU fault is ever caused.

The reference has none of this: its solves loop to maxiter = 100000 without a word
(PSolver.cpp:2087, 2291), it never checks for NaN, and a bad INP.DAT leaves the object
uninitialised (PSolver.cpp:511-514). Here every case carries a status word written by the
device, and every device wait is bounded:
  * a NaN planted on the host (through the state image) in one case of a batch makes
    only that case report CFD_STATUS_NAN; the other cases keep the bits of a clean run,
    also after the bad case's slot is emptied (retired) and the batch steps on;
  * a pressure or momentum solve stopped by its iteration cap sets CFD_STATUS_MAXITER
    for that step, and cfd_case_step returns CFD_E_MAXITER;
  * a bulk-copy wait whose poll limit runs out sets the batch's error flag, the step
    fails with CFD_E_CUDA, and the device stays usable for a new batch.
"""
import ctypes

import numpy as np
import pytest

from cfd_solver_b200.grid import cavity, ogrid

pytestmark = pytest.mark.gpu

ST_MAXITER, ST_BREAKDOWN, ST_NAN = 1, 2, 4
E_CUDA, E_DIVERGED, E_MAXITER = -2, -4, -5


def _cases():
    from cfd_solver_b200.solver import case_params
    gs = [ogrid(33, 25, skew=0.1), cavity(33, 33, skew=0.1), ogrid(41, 29, ar=3.0, skew=0.05)]
    ps = [case_params(gs[0], Re=100.0, Ri=1.0, dt=1e-3), case_params(gs[1], Re=200.0, Ri=1.0, dt=2e-3),
          case_params(gs[2], Re=300.0, dt=5e-4)]
    return gs, ps


def _state_offset(grids, case):
    """Offset (in doubles) of `case`'s first plane (u) in the batch's state image."""
    off = 0
    for g in grids[:case]:
        w = g.n0 - 1 if g.kind == "ogrid" else g.n0
        off += 6 * g.n1 * w + 16
    return off


def _fields(b, n):
    return [{k: b.plane(c, k) for k in ("u", "v", "T", "p")} for c in range(n)]


def test_nan_in_one_case_retires_only_that_case():
    from cfd_solver_b200.solver import Batch
    gs, ps = _cases()
    with Batch(gs, ps) as b:
        b.step(5)
        clean = _fields(b, 3)
    with Batch(gs, ps) as b:
        img = np.zeros(b.state_bytes() // 8, dtype=np.float64)
        b.get_state(img)
        w = gs[1].n0  # the cavity stores every column
        img[_state_offset(gs, 1) + 9 * w + 7] = np.nan  # u at (i, j) = (7, 9) of case 1
        b.set_state(img)
        b.step(3)
        st = b.all_stats()
        assert st[1]["status"] & ST_NAN, st[1]
        assert st[0]["status"] == 0 and st[2]["status"] == 0
        b.set_active(1, False)  # retire the bad case; the others step on
        b.step(2)
        dirty = _fields(b, 3)
    for c in (0, 2):
        for k in clean[c]:
            np.testing.assert_array_equal(dirty[c][k], clean[c][k], err_msg=f"case {c} {k}")


def test_case_step_reports_divergence():
    from cfd_solver_b200 import _lib
    from cfd_solver_b200.solver import Batch, case_params
    g = ogrid(33, 25, skew=0.1)
    with Batch([g], [case_params(g, Re=100.0, dt=1e-3)]) as b:
        img = np.zeros(b.state_bytes() // 8, dtype=np.float64)
        b.get_state(img)
        img[5 * (g.n0 - 1) + 3] = np.inf  # u at (3, 5)
        b.set_state(img)
        st = _lib.CfdStepStats()
        rc = _lib.lib().cfd_case_step(b.h, 1, ctypes.byref(st))
        assert rc == E_DIVERGED
        assert st.status & ST_NAN


@pytest.mark.parametrize("which", ["pressure", "momentum"])
def test_iteration_cap_is_reported(which):
    from cfd_solver_b200 import _lib
    from cfd_solver_b200.solver import Batch, case_params
    g = ogrid(33, 25, skew=0.1)
    if which == "pressure":
        capped = dict(tol_p=1e-15, atol_p=0.0, maxit_p=1)
    else:
        capped = dict(tol_mom=1e-15, atol_mom=0.0, maxit_mom=2)
    for kw, expect in ((dict(), 0), (capped, ST_MAXITER)):
        with Batch([g], [case_params(g, Re=100.0, dt=1e-3, **kw)]) as b:
            st = _lib.CfdStepStats()
            rc = _lib.lib().cfd_case_step(b.h, 2, ctypes.byref(st))
            assert (st.status & ST_MAXITER) == expect, (which, kw, st.status)
            assert rc == (E_MAXITER if expect else 0), (rc, _lib.lib().cfd_last_error())
            if which == "pressure" and expect:
                assert st.it_p == 1
            if which == "momentum" and expect:
                assert list(st.it_mom) == [2] * 5


def test_bounded_wait_that_runs_out_is_reported():
    from cfd_solver_b200 import _lib
    from cfd_solver_b200.solver import Batch, case_params
    g = ogrid(33, 25, skew=0.1)
    p = case_params(g, Re=100.0, dt=1e-3, maxit_mom=8, maxit_p=8)
    with Batch([g], [p]) as b:
        b.set_wait_limit(0)  # every kernel's first copy wait gives up at once
        with pytest.raises(_lib.CfdError, match="bounded wait"):
            b.step(1)
    # the device is still usable: a new batch steps like one that never saw the error
    with Batch([g], [p]) as b:
        b.step(2)
        again = _fields(b, 1)[0]
        assert b.stats(0)["status"] == 0
    with Batch([g], [p]) as b:
        b.set_wait_limit(-1)  # the default limit
        b.step(2)
        ref = _fields(b, 1)[0]
    for k in ref:
        np.testing.assert_array_equal(again[k], ref[k], err_msg=k)
