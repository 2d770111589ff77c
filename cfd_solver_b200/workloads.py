"""Seeded synthetic workloads of the benchmark configurations.

The reference publishes no benchmark data; every case here is generated from a
seed. Each configuration exists in two forms:
  * cavity -- the lid-driven skewed unit square the configurations describe;
  * twin   -- the O-grid around an elliptic cylinder (the reference's own
              geometry and boundary conditions) with the same N, Re, Ri, Pr and
              skew, the form the compiled reference can run.
"""
from __future__ import annotations

import math

import numpy as np

from .grid import cavity, ogrid

SWEEP_SEED = 1234


def sweep_draws(ncases: int = 256, seed: int = SWEEP_SEED):
    """The batched sweep: N in {65,129,193,257}, skew U[0,0.2], Re logU[50,1000],
    Ri logU[0.1,10], Pr in {0.71, 7.0}."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(ncases):
        N = int(rng.choice([65, 129, 193, 257]))
        skew = float(rng.uniform(0.0, 0.2))
        Re = float(math.exp(rng.uniform(math.log(50.0), math.log(1000.0))))
        Ri = float(math.exp(rng.uniform(math.log(0.1), math.log(10.0))))
        Pr = float(rng.choice([0.71, 7.0]))
        out.append(dict(N=N, skew=skew, Re=Re, Ri=Ri, Pr=Pr))
    return out


SERVE_SIZES = (129, 257, 513, 1025)
SERVE_PROBS = (0.4, 0.3, 0.2, 0.1)


def serve_stream(nrequests: int, rate: float, seed: int = SWEEP_SEED + 7, sizes=SERVE_SIZES,
                 probs=SERVE_PROBS):
    """The served request stream: Poisson arrivals at `rate` requests/s, N in
    {129, 257, 513, 1025} with probability {.4, .3, .2, .1}, the other physics of the
    sweep draws of the same seed. `sizes` restricts N to a subset of the classes (their
    probabilities renormalised). Returns [(arrival_s, draw)] in arrival order."""
    rng = np.random.default_rng(seed)
    p = np.array([probs[list(SERVE_SIZES).index(n)] for n in sizes], dtype=float)
    p /= p.sum()
    out = []
    t = 0.0
    for d in sweep_draws(nrequests, seed=seed):
        d = dict(d, N=int(rng.choice(list(sizes), p=list(p))))
        t += float(rng.exponential(1.0 / rate))
        out.append((t, d))
    return out


def cavity_dt(N: int, Ri: float, Re: float = 0.0, Pr: float = 1.0, cfl: float = 0.4) -> float:
    """Time step of the cavity form, velocity scale U = max(1, sqrt(Ri)) (lid speed or
    buoyant velocity). Two limits: CFL `cfl` on U, and the stability of explicit
    (forward-Euler) convection with implicit diffusion, whose low-wavenumber modes grow
    unless dt <= 2 / (Re Pr_eff U^2) with Pr_eff = max(1, Pr) (u, v: 1/Re; T: 1/(Re Pr));
    half of that bound is used."""
    U = max(1.0, math.sqrt(Ri))
    dt = cfl / (N - 1) / U
    if Re > 0.0:
        dt = min(dt, 1.0 / (Re * max(1.0, Pr) * U * U))
    return dt


def make_case(d: dict, form: str):
    """(grid, params-dict) of one draw in the given form."""
    if form == "cavity":
        g = cavity(d["N"], d["N"], skew=d["skew"])
        prm = dict(Re=d["Re"], Ri=d["Ri"], Pr=d["Pr"], dt=cavity_dt(d["N"], d["Ri"], d["Re"], d["Pr"]))
    elif form == "twin":
        g = ogrid(d["N"], d["N"], ar=2.0, r_outer=20.0, skew=d["skew"])
        # the reference's own time step and flow angle (PSolver.cpp:169-174)
        prm = dict(Re=d["Re"], Ri=d["Ri"], Pr=d["Pr"], dt=1e-4, alpha=82.0)
    else:
        raise ValueError(form)
    return g, prm


# the single-case configurations
CONFIGS = {
    "c1": dict(N=65, skew=0.1, Re=100.0, Ri=1.0, Pr=0.71),
    "c2": dict(N=513, skew=0.15, Re=400.0, Ri=1.0, Pr=0.71),
    "c3": dict(N=1025, skew=0.15, Re=1000.0, Ri=2.0, Pr=0.71),
}
