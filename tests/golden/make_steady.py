"""Golden steady states from the oracle, for converged-state parity of the GPU path.

Each case is advanced by the FP64 CPU restatement (oracle/cfd_oracle.c; on the O-grid
profile bit-identical to the compiled reference, tests/test_oracle_golden.py) from the
reference's initial state until its steady residual -- the L1 change of u, v and T over
one step, relative to the first step's -- is at most STOP. The inner solves run to a
relative L1 residual of 1e-13 with an absolute floor of 1e-11 (the floor is what lets a
solve started from the previous step's solution stop near the steady state). At that
point every step reproduces the state to rounding, so the state is the discretisation's
fixed point: it no longer depends on the inner solvers (lexicographic Gauss-Seidel and
SIP here, Chebyshev-Jacobi and multigrid BiCGStab on the GPU) or on the path taken.

Cases (time step chosen as large as the explicit convection stays stable):
  og33_re10_ri0     O-grid twin 33 x 25 (aspect ratio 2, outer radius 20, skew 0.1),
                    Re 10, Ri 0, dt 0.03, the reference's C++ coefficients;
  og33_re10_ri025   the same with buoyancy, Ri 0.25 (at Ri 1 this twin does not settle:
                    it diverges at Re 10 and drifts at Re 5);
  cav33_c1          skewed lid-driven cavity 33 x 33 (skew 0.1), Re 100, Ri 1, Pr 0.71,
                    dt 0.0125 -- the first benchmark configuration's physics at 33 x 33;
  cav65_c1          the first benchmark configuration itself: cavity 65 x 65, skew 0.1,
                    Re 100, Ri 1, Pr 0.71, dt 0.00625 (about 20 minutes of CPU).
The cavity profile has no reference implementation: its fixtures are pinned to the
restatement only, whose interior discretisation is the pinned O-grid code.

    python tests/golden/make_steady.py [case ...]   # writes tests/golden/steady_<case>.npz
"""
import multiprocessing as mp
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

STOP = 1e-12
INNER = dict(tol_gs=1e-13, atol_gs=1e-11, maxit_gs=4000, tol_sip=1e-13, atol_sip=1e-11,
             maxit_sip=20000)

CASES = {
    "og33_re10_ri0": dict(kind="ogrid", n0=33, n1=25, skew=0.1,
                          phys=dict(Re=10.0, Ri=0.0, Pr=0.71, dt=0.03), max_steps=40000),
    "og33_re10_ri025": dict(kind="ogrid", n0=33, n1=25, skew=0.1,
                            phys=dict(Re=10.0, Ri=0.25, Pr=0.71, dt=0.03), max_steps=60000),
    "cav33_c1": dict(kind="cavity", n0=33, n1=33, skew=0.1,
                     phys=dict(Re=100.0, Ri=1.0, Pr=0.71, dt=0.0125), max_steps=40000),
    "cav65_c1": dict(kind="cavity", n0=65, n1=65, skew=0.1,
                     phys=dict(Re=100.0, Ri=1.0, Pr=0.71, dt=0.00625), max_steps=60000),
}
FIELDS = ("u", "v", "T", "p", "si", "vort", "dil")
DIAGS = ("nu", "cl", "cd", "cm", "circ", "cl_pr", "cd_pr", "cl_vor", "cd_vor", "dmax")


def grid_of(spec):
    from cfd_solver_b200.grid import cavity, ogrid
    if spec["kind"] == "ogrid":
        return ogrid(spec["n0"], spec["n1"], ar=2.0, r_outer=20.0, skew=spec["skew"])
    return cavity(spec["n0"], spec["n1"], skew=spec["skew"])


def run(name):
    try:
        return run_case(name)
    except RuntimeError as e:
        return name, -1, str(e), 0.0, 0.0


def run_case(name):
    from oracle import oracle
    spec = CASES[name]
    g = grid_of(spec)
    t0 = time.time()
    o = oracle.OracleCase(g, **spec["phys"], **INNER)
    ref = None
    steps = 0
    res = np.inf
    while steps < spec["max_steps"]:
        d = o.step(100)
        ch = d["du_l1"] + d["dT_l1"]
        if ref is None:
            ref = ch[0]
        steps += 100
        res = float(ch[-1] / ref)
        if not np.isfinite(res):
            raise RuntimeError(f"{name}: diverged at step {steps}")
        if res <= STOP:
            break
    if res > STOP:
        raise RuntimeError(f"{name}: steady residual {res:.2e} after {steps} steps")
    out = {k: o.field(k) for k in FIELDS}
    out.update({k: float(d[k][-1]) for k in DIAGS})
    out.update(steps=steps, steady_res_rel=res, it_sip=float(d["it_sip"][-1]))
    np.savez_compressed(Path(__file__).with_name(f"steady_{name}.npz"), **out)
    return name, steps, res, time.time() - t0, out["nu"]


def main(names):
    names = names or list(CASES)
    with mp.get_context("spawn").Pool(len(names)) as pool:
        for name, steps, res, wall, nu in pool.imap_unordered(run, names):
            if steps < 0:
                print(f"{name}: FAILED: {res}", flush=True)
                continue
            print(f"{name}: {steps} steps, steady residual {res:.2e}, Nu {nu:.12f}, {wall:.0f} s",
                  flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
