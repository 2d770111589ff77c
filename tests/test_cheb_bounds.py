"""The Chebyshev interval of the u/v/T sweeps contains the spectrum of D^-1 A.

The sweeps (csrc/cfd_sweep.cu) run Chebyshev-accelerated Jacobi on the 25-point / 9-point
operator of each momentum or energy system (the reference's gauss() systems,
PSolver.cpp:752-940, 2280-2446). The library bounds the eigenvalues of D^-1 A by
[a0, b0] = [1/(1 + 2.5 Emax), 1 + rmax] (cheb_bounds / cheb_finish in csrc/cfd_api.cu) and
widens that interval on each side by 2 % of its width, capped at 0.1 a0 below and 0.05 b0
above. These tests assemble the operators with the
oracle (its coefficient planes, the reference's boundary-row folding), form D^-1 A densely on
small grids, and check that every eigenvalue's real part lies inside the margin-free
interval, for the u-type and the T systems (with the reference's atnw-for-annw slip on the
O-grid), at time steps from the reference's to the large steps of steady runs. The
imaginary parts stay small. The formula is restated here from the library's.
"""
import numpy as np
import pytest

from cfd_solver_b200.grid import cavity, ogrid

ORDER = ("p", "e", "w", "n", "s", "ne", "nw", "se", "sw", "ee", "ww", "nn", "ss", "nnee", "nnww",
         "ssee", "ssww", "nne", "nnw", "sse", "ssw", "nee", "nww", "see", "sww")
OFF = {"p": (0, 0), "e": (1, 0), "w": (-1, 0), "n": (0, 1), "s": (0, -1), "ne": (1, 1), "nw": (-1, 1),
       "se": (1, -1), "sw": (-1, -1), "ee": (2, 0), "ww": (-2, 0), "nn": (0, 2), "ss": (0, -2),
       "nnee": (2, 2), "nnww": (-2, 2), "ssee": (2, -2), "ssww": (-2, -2), "nne": (1, 2), "nnw": (-1, 2),
       "sse": (1, -2), "ssw": (-1, -2), "nee": (2, 1), "nww": (-2, 1), "see": (2, -1), "sww": (-2, -1)}


def dinv_a(case, g, prefix, slip):
    """D^-1 A of one system on the unknown cells (boundary rows and, in the cavity, boundary
    columns held), from the oracle's assembled planes."""
    A = {k: case.field(prefix + k) for k in ORDER}
    if slip:
        A["nnw"] = A["nw"]  # the reference's T call passes atnw in the annw slot (PSolver.cpp:1290)
    per = g.kind == "ogrid"
    W = g.n0 - 1 if per else g.n0
    cols = range(W) if per else range(1, g.n0 - 1)
    idx = {(j, i): k for k, (j, i) in enumerate((j, i) for j in range(1, g.n1 - 1) for i in cols)}
    M = np.zeros((len(idx), len(idx)))
    for (j, i), r in idx.items():
        nearw = j == 1 or j == g.n1 - 2 or (not per and i in (1, g.n0 - 2))
        for k in ORDER:
            di, dj = OFF[k]
            if nearw and max(abs(di), abs(dj)) > 1:
                continue
            a = A[k][j, i]
            if not np.isfinite(a) or a == 0.0:
                continue
            ii = (i + di) % W if per else i + di
            c = idx.get((j + dj, ii))
            if c is not None:
                M[r, c] += a
    return M / np.diag(M)[:, None]


def library_interval(g, prm, energy, slip):
    """[1/(1 + 2.5 Emax), 1 + rmax] as cheb_bounds() forms it (before the margins)."""
    scale = prm["Re"] * (prm.get("Pr", 0.71) if energy else 1.0)
    cross = 4.5 + 7.0 / 9.0 if slip else 4.5
    rows = slice(1, -1)
    E = prm["dt"] / scale * (g.alph[rows] / g.dxi0 ** 2 + g.gam[rows] / g.dxi1 ** 2)
    cc = prm["dt"] / (scale * g.dxi0 * g.dxi1)
    rmax = (((17.0 / 6.0) * E + cross * np.abs(g.beta[rows]) * cc) / (1.0 + 2.5 * E)).max()
    return 1.0 / (1.0 + 2.5 * E.max()), 1.0 + rmax


CASES = [
    ("O-grid, reference dt", ogrid(24, 20, ar=2.0, skew=0.1), dict(Re=100.0, Ri=1.0, dt=1e-3)),
    ("O-grid, steady-run dt", ogrid(24, 20, ar=2.0, skew=0.1), dict(Re=10.0, dt=0.03)),
    ("O-grid circle", ogrid(24, 20, ar=1.0), dict(Re=50.0, Ri=0.5, dt=2e-3)),
    ("cavity, large dt", cavity(19, 19, skew=0.1), dict(Re=100.0, Ri=1.0, Pr=0.71, dt=0.02)),
    ("cavity, Pr 7", cavity(19, 19, skew=0.15), dict(Re=400.0, Ri=2.0, Pr=7.0, dt=1e-3)),
]


@pytest.mark.parametrize("label,g,prm", CASES, ids=[c[0] for c in CASES])
def test_spectrum_inside_the_chebyshev_interval(oracle_lib, label, g, prm):
    case = oracle_lib.OracleCase(g, **prm)
    slip = g.kind == "ogrid"  # the O-grid keeps the reference's T coefficient
    for energy, prefix in ((False, "au"), (True, "at")):
        ev = np.linalg.eigvals(dinv_a(case, g, prefix, slip and energy))
        lo, hi = library_interval(g, prm, energy, slip and energy)
        assert ev.real.min() >= lo, (label, prefix, ev.real.min(), lo)
        assert ev.real.max() <= hi, (label, prefix, ev.real.max(), hi)
        assert np.abs(ev.imag).max() <= 0.02 * (hi - lo) + 1e-12, (label, prefix, np.abs(ev.imag).max())


def library_margins(a0, b0):
    """The widened interval of cheb_finish(): 2 % of the width on each side, at most 0.1 a0
    below and 0.05 b0 above."""
    w = b0 - a0
    return a0 - min(0.1 * a0, 0.02 * w), b0 + min(0.05 * b0, 0.02 * w)


def chebyshev_sweeps(DA, e0, a, b, tol=0.75e-2, kmax=150):
    """Sweeps a Chebyshev-Jacobi solve on [a, b] needs to bring the L1 residual of the error
    e0 below tol of its start (the reference's momentum tolerance, PSolver.cpp:2291), tested
    on each sweep's input iterate as k_sweep_fin does; the recurrence of cfd_sweep.cu."""
    s2 = ((b + a) / (b - a)) ** 2
    g = 2.0 / (a + b)
    e, ep, w, r0 = e0.copy(), e0.copy(), 1.0, None
    for k in range(kmax):
        r = DA @ e
        rn = np.abs(r).sum()
        r0 = rn if r0 is None else r0
        if rn / r0 < tol:
            return k + 1
        w = 1.0 if k == 0 else (1.0 / (1.0 - 1.0 / (2.0 * s2)) if k == 1 else 1.0 / (1.0 - w / (4.0 * s2)))
        en = e - g * r
        if k > 0:
            en = w * (en - ep) + ep
        ep, e = e, en
    return kmax


MARGIN_CASES = [
    # a wide interval: E of 6.5 (u) and 9.2 (T), as the 257 x 257 cavities of the sweep draws
    ("cavity, E 7-9", cavity(25, 25, skew=0.1), dict(Re=50.0, Ri=0.0, Pr=0.71, dt=0.25), 2),
    # a narrow one: the benchmark twin at the reference's time step
    ("twin, reference dt", ogrid(33, 33, ar=2.0, r_outer=20.0, skew=0.1),
     dict(Re=100.0, Ri=1.0, dt=1e-4, alpha=82.0), 8),
]


@pytest.mark.parametrize("label,g,prm,nstep", MARGIN_CASES, ids=[c[0] for c in MARGIN_CASES])
def test_margins_fit_narrow_and_wide_intervals(oracle_lib, label, g, prm, nstep):
    """A solve started from the previous step's field, on the error of one real step: the
    library's margins need no more sweeps than either plain rule, fixed fractions of the
    bounds (0.9 a0, 1.05 b0) or 2 % of the width (which leaves a0 - 0.02 w near zero on a wide
    interval)."""
    slip = g.kind == "ogrid"
    case = oracle_lib.OracleCase(g, tol_gs=1e-13, atol_gs=1e-15, maxit_gs=20000, **prm)
    case.step(nstep)
    per = g.kind == "ogrid"
    cols = slice(0, g.n0 - 1) if per else slice(1, g.n0 - 1)
    for energy, name, prefix in ((False, "u", "au"), (True, "T", "at")):
        x0 = case.field(name).copy()
        case.step(1)
        e0 = (x0 - case.field(name))[1:-1, cols].ravel()
        DA = dinv_a(case, g, prefix, slip and energy)
        a0, b0 = library_interval(g, prm, energy, slip and energy)
        w = b0 - a0
        lib = chebyshev_sweeps(DA, e0, *library_margins(a0, b0))
        frac = chebyshev_sweeps(DA, e0, 0.9 * a0, 1.05 * b0)
        width = chebyshev_sweeps(DA, e0, a0 - 0.02 * w, b0 + 0.02 * w)
        assert lib <= min(frac, width), (label, name, lib, frac, width)
        if g.kind == "cavity":
            assert width > 2 * lib, (label, name, lib, width)  # the case the caps are for
        else:
            assert lib == 2 and frac == 3, (label, name, lib, frac)
