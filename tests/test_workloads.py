"""The seeded benchmark workloads match their configuration table: the 256-case sweep's
draws (N in {65, 129, 193, 257}, skew U[0, 0.2], Re logU[50, 1000], Ri logU[0.1, 10],
Pr in {0.71, 7}), the single-case configurations, the two case forms and the cavity's
time-step limits. Host logic only."""
import math

import numpy as np

from cfd_solver_b200 import workloads as W


def test_sweep_draws_are_seeded_and_within_the_table():
    a = W.sweep_draws(256)
    assert a == W.sweep_draws(256, W.SWEEP_SEED)
    assert a != W.sweep_draws(256, W.SWEEP_SEED + 1)  # per-rank seeds give other cases
    assert len(a) == 256
    assert {d["N"] for d in a} == {65, 129, 193, 257}
    assert {d["Pr"] for d in a} == {0.71, 7.0}
    for d in a:
        assert 0.0 <= d["skew"] < 0.2
        assert 50.0 <= d["Re"] <= 1000.0
        assert 0.1 <= d["Ri"] <= 10.0
    # log-uniform: the median of log Re sits near the middle of [log 50, log 1000]
    mid = 0.5 * (math.log(50.0) + math.log(1000.0))
    assert abs(np.median([math.log(d["Re"]) for d in a]) - mid) < 0.3
    assert W.sweep_draws(8) == a[:8]  # a shorter sweep is a prefix of the full one


def test_single_case_configurations():
    assert W.CONFIGS["c1"] == dict(N=65, skew=0.1, Re=100.0, Ri=1.0, Pr=0.71)
    assert W.CONFIGS["c2"] == dict(N=513, skew=0.15, Re=400.0, Ri=1.0, Pr=0.71)
    assert W.CONFIGS["c3"] == dict(N=1025, skew=0.15, Re=1000.0, Ri=2.0, Pr=0.71)


def test_case_forms():
    d = W.CONFIGS["c1"]
    g, prm = W.make_case(d, "twin")
    assert (g.n0, g.n1, g.kind) == (65, 65, "ogrid") and g.ar == 2.0 and g.a_grid == 20.0
    assert prm["dt"] == 1e-4 and prm["alpha"] == 82.0  # the reference's own dt and flow angle
    g, prm = W.make_case(d, "cavity")
    assert (g.n0, g.n1, g.kind) == (65, 65, "cavity")
    assert prm["dt"] == W.cavity_dt(65, 1.0, 100.0, 0.71)
    try:
        W.make_case(d, "other")
    except ValueError:
        pass
    else:
        raise AssertionError("unknown form accepted")


def test_cavity_dt_limits():
    for N, Ri, Re, Pr in [(65, 1.0, 100.0, 0.71), (257, 10.0, 1000.0, 7.0), (129, 0.1, 50.0, 0.71)]:
        dt = W.cavity_dt(N, Ri, Re, Pr)
        U = max(1.0, math.sqrt(Ri))
        assert dt <= 0.4 / (N - 1) / U * (1 + 1e-15)  # CFL 0.4 on the velocity scale
        assert dt <= 1.0 / (Re * max(1.0, Pr) * U * U) * (1 + 1e-15)  # half the convective bound
        assert dt in (0.4 / (N - 1) / U, 1.0 / (Re * max(1.0, Pr) * U * U))
    assert W.cavity_dt(65, 1.0) == 0.4 / 64  # no Re: CFL only


def test_serve_stream_is_a_seeded_poisson_stream_with_the_size_mix():
    n, rate = 4096, 8.0  # the served configuration's request count
    s = W.serve_stream(n, rate)
    assert s == W.serve_stream(n, rate)
    t = np.array([a for a, _ in s])
    assert np.all(np.diff(t) > 0) and t[0] > 0
    gaps = np.diff(np.concatenate([[0.0], t]))
    # exponential gaps: mean 1/rate (4-sigma band of the sample mean), coefficient of variation ~1
    assert abs(gaps.mean() * rate - 1.0) < 4.0 / math.sqrt(n)
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.1
    Ns = np.array([d["N"] for _, d in s])
    for N, p in zip(W.SERVE_SIZES, W.SERVE_PROBS):
        f = np.mean(Ns == N)
        assert abs(f - p) < 4.0 * math.sqrt(p * (1 - p) / n), (N, f, p)
    draws = W.sweep_draws(n, seed=W.SWEEP_SEED + 7)
    for (_, d), b in zip(s, draws):  # everything but N is the sweep draw of the same seed
        assert {k: v for k, v in d.items() if k != "N"} == {k: v for k, v in b.items() if k != "N"}
