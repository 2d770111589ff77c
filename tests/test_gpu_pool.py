"""The slot pool (cfd_pool_*) and serving by free device memory.

The reference runs one case per process; here a request loop admits cases of any size
into one device arena by its free bytes (cfd_pool_create / cfd_pool_admit /
cfd_pool_release), and cfd_serve does so when no fixed slots are given:
  * admission follows the free bytes: a case is placed while a free region fits it, and
    memory a retired case gives back is re-cut for cases of another size;
  * a pooled case steps bit for bit as it does alone, whatever is admitted or released
    around it (its tiles keep their order in every launch);
  * a burst of one size uses all of the budget (more cases at once than an equal split
    between sizes would give), and every served result equals its solo run.
"""
import numpy as np
import pytest

from cfd_solver_b200.grid import cavity, ogrid

pytestmark = pytest.mark.gpu


def _fields(b, c):
    return {k: b.plane(c, k) for k in ("u", "v", "T", "p")}


def test_pool_admission_follows_free_memory():
    from cfd_solver_b200.solver import Pool, case_params
    big, small = cavity(65, 65, skew=0.1), cavity(33, 33, skew=0.1)
    pb, ps = case_params(big, Re=100.0, dt=5e-3), case_params(small, Re=100.0, dt=1e-2)
    Bb, Bs = Pool.case_bytes(big), Pool.case_bytes(small)
    assert Bb > 3 * Bs
    budget = 2 * Bb + Bb // 2
    with Pool(budget, max_cases=64) as pool:
        total0, _ = pool.free()
        s0, s1 = pool.place(big, pb), pool.place(big, pb)
        assert s0 is not None and s1 is not None
        assert pool.place(big, pb) is None  # half a big case is left: it does not fit
        free, largest = pool.free()
        assert free == total0 - 2 * Bb and largest == free
        n = 0
        while pool.place(small, ps) is not None:
            n += 1
        assert n == free // Bs  # the rest is cut into small cases
        pool.release(s0)  # a big case's memory goes back ...
        m = 0
        while pool.place(small, ps) is not None:
            m += 1
        assert m >= Bb // Bs  # ... and is re-cut for small ones
        pool.step(2)
        st = pool.all_stats()
        assert all(x["status"] == 0 for x in st)


def test_pooled_cases_step_like_solo_runs_bitwise():
    from cfd_solver_b200.solver import Batch, Pool, case_params
    gA, gB, gC = ogrid(33, 25, skew=0.1), cavity(41, 33, skew=0.15), ogrid(65, 33, ar=3.0, skew=0.05)
    pA = case_params(gA, Re=100.0, Ri=1.0, dt=1e-3)
    pB = case_params(gB, Re=400.0, Ri=2.0, Pr=7.0, dt=1e-3)
    pC = case_params(gC, Re=300.0, dt=5e-4)
    solo = {}
    for name, g, p, n in (("A", gA, pA, 7), ("B", gB, pB, 6), ("C", gC, pC, 2)):
        with Batch([g], [p]) as b:
            b.step(n)
            solo[name] = _fields(b, 0)
    budget = 3 * max(Pool.case_bytes(g) for g in (gA, gB, gC))
    with Pool(budget, max_cases=8) as pool:
        a = pool.place(gA, pA)
        pool.step(3)
        bb = pool.place(gB, pB)
        pool.step(4)
        got_a = _fields(pool, a)  # A: 7 steps, B: 4
        pool.release(a)
        c = pool.place(gC, pC)  # C may take A's memory
        pool.step(2)
        got_b, got_c = _fields(pool, bb), _fields(pool, c)
    for name, got in (("A", got_a), ("B", got_b), ("C", got_c)):
        for k in got:
            np.testing.assert_array_equal(got[k], solo[name][k], err_msg=f"{name} {k}")


def _concurrency(results):
    ev = sorted([(r["admit_s"], 1) for r in results] + [(r["done_s"], -1) for r in results])
    cur = peak = 0
    for _, d in ev:
        cur += d
        peak = max(peak, cur)
    return peak


def test_serve_by_free_memory_uses_the_whole_budget():
    from cfd_solver_b200.solver import Batch, Pool, case_params, serve
    rng = np.random.default_rng(11)
    small, mid = cavity(33, 33, skew=0.1), cavity(49, 49, skew=0.1)
    Bs, Bm = Pool.case_bytes(small), Pool.case_bytes(mid)
    budget = 6 * Bs + Bs // 2  # an equal split with the 49 x 49 class would leave 3 small slots
    reqs, cases = [], []
    t = 0.0
    for k in range(10):  # a burst of small requests, then two mid-size ones
        t += rng.exponential(0.001)
        g = cavity(49, 49, skew=float(rng.uniform(0, 0.2))) if k >= 8 else \
            cavity(33, 33, skew=float(rng.uniform(0, 0.2)))
        N = g.n0
        prm = case_params(g, Re=float(rng.uniform(50, 200)), Ri=float(rng.uniform(0.1, 1.0)), dt=0.4 / (N - 1))
        reqs.append((t, g, prm, 1e-3, 3000))
        cases.append((g, prm))
    assert Bm <= budget
    results, stats = serve(reqs, [], steps_per_tick=25, slots=None, hbm_budget=budget)
    assert stats["converged"] == len(reqs)
    assert _concurrency(results[:8]) >= 5
    for (g, prm), r in zip(cases, results):
        assert r["status"] == 0 and r["steady_res_rel"] <= 1e-3
        with Batch([g], [prm]) as solo:
            solo.step(r["steps"])
            assert solo.stats(0)["nu"] == r["nu"]


def test_serve_rejects_a_request_larger_than_the_budget():
    from cfd_solver_b200 import _lib
    from cfd_solver_b200.solver import Pool, case_params, serve
    g = cavity(65, 65, skew=0.1)
    reqs = [(0.0, g, case_params(g, Re=100.0, dt=5e-3), 1e-3, 100)]
    with pytest.raises(_lib.CfdError, match="whole budget"):
        serve(reqs, [], slots=None, hbm_budget=Pool.case_bytes(g) // 2)
