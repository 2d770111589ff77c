"""The gauss() seam (cfd_gauss_solve) against the oracle's own gauss() solves.

Inputs are the oracle's assembled coefficient planes, its initial field and the
right-hand side it built in one step; the oracle's result is its tightly converged
lexicographic Gauss-Seidel solution (PSolver.cpp:2280-2446 restated)."""
import ctypes

import numpy as np
import pytest

from cfd_solver_b200.grid import cavity, ogrid

pytestmark = pytest.mark.gpu

GAUSS_ORDER = ("p", "e", "s", "n", "w", "se", "sw", "ne", "nw", "ss", "ssee", "ssww", "sse",
               "ssw", "see", "sww", "nn", "nnee", "nnww", "nne", "nnw", "nee", "nww", "ee", "ww")


def system(g, which, fix_T=0):
    """(coefficient planes in gauss() order, phi0, q, oracle result) of one system."""
    from oracle import oracle
    c = oracle.OracleCase(g, Re=100.0, Ri=1.0, dt=2e-3, tol_gs=1e-13, maxit_gs=600,
                          fix_T_annw=fix_T)
    field, rhs, out, pre = {"u": ("u", "qu", "us", "au"), "T": ("T", "qt", "T", "at")}[which]
    phi0 = c.field(field).copy()
    c.step(1)
    coefs = []
    for s in GAUSS_ORDER:
        name = pre + s
        if pre == "at" and s == "nnw" and not fix_T:
            name = "atnw"  # the reference's T call passes atnw in the annw slot (PSolver.cpp:1290)
        coefs.append(c.field(name))
    return coefs, phi0, c.field(rhs), c.field(out)


def gpu_solve(fn, g, coefs, phi0, q, periodic, tol=1e-13, maxit=600, **kw):
    import torch
    from cfd_solver_b200 import _lib
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in coefs]
    ptrs = (ctypes.c_void_p * 25)(*[t.data_ptr() for t in dev])
    phi = torch.from_numpy(phi0.copy()).cuda()
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    sweeps = ctypes.c_int(0)
    torch.cuda.synchronize()
    rc = fn(g.n0, g.n1, periodic, ptrs, ctypes.c_void_p(phi.data_ptr()), ctypes.c_void_p(qd.data_ptr()),
            tol, maxit, ctypes.byref(sweeps), None)
    torch.cuda.synchronize()
    assert rc == 0, _lib.lib().cfd_last_error()
    return phi.cpu().numpy(), sweeps.value


@pytest.mark.parametrize("which", ["u", "T"])
def test_gauss_seam_ogrid(which):
    from cfd_solver_b200 import _lib
    g = ogrid(33, 25, skew=0.1)
    coefs, phi0, q, ref = system(g, which)
    # the u system starts within ~1e-3 of its solution, so 1e-13 relative is below the
    # round-off floor; 1e-11 still leaves the result far inside the 1e-10 bar
    phi, sweeps = gpu_solve(_lib.lib().cfd_gauss_solve, g, coefs, phi0, q, 1, tol=1e-11)
    err = np.linalg.norm(phi[1:-1] - ref[1:-1]) / np.linalg.norm(ref[1:-1])
    assert err < 1e-10, err
    assert np.array_equal(phi[:, -1], phi[:, 0])  # seam column kept
    assert sweeps >= 2


def test_gauss_seam_cavity():
    from cfd_solver_b200 import _lib
    g = cavity(33, 29, skew=0.15)
    coefs, phi0, q, ref = system(g, "u", fix_T=1)
    phi, _ = gpu_solve(_lib.lib().cfd_gauss_solve, g, coefs, phi0, q, 0)
    err = np.linalg.norm(phi[1:-1, 1:-1] - ref[1:-1, 1:-1]) / np.linalg.norm(ref[1:-1, 1:-1])
    assert err < 1e-10, err


# ---- the sip9p() seam (cfd_sip_solve) ----
SIP_ORDER = ("ap", "ae", "as", "an", "aw", "ase", "asw", "ane", "anw")  # PSolver.cpp:2067-2069


def sip_gpu(g, coefs, phi0, q, periodic, tol=1e-13, maxit=400):
    import torch
    from cfd_solver_b200 import _lib
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in coefs]
    ptrs = (ctypes.c_void_p * 9)(*[t.data_ptr() for t in dev])
    phi = torch.from_numpy(np.ascontiguousarray(phi0, dtype=np.float64).copy()).cuda()
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    iters = ctypes.c_int(0)
    torch.cuda.synchronize()
    rc = _lib.lib().cfd_sip_solve(g.n0, g.n1, periodic, ptrs, ctypes.c_void_p(phi.data_ptr()),
                                  ctypes.c_void_p(qd.data_ptr()), tol, maxit, ctypes.byref(iters), None)
    torch.cuda.synchronize()
    return rc, phi.cpu().numpy(), iters.value


def direct_solve(coefs, phi0, q, periodic):
    """The 9-point system on the unknown cells, boundary values of phi0 moved to the right-hand
    side, solved by sparse LU (scipy) -- the exact answer sip9p converges to."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    a = dict(zip(SIP_ORDER, coefs))
    n1, n0 = q.shape
    cols = list(range(n0 - 1)) if periodic else list(range(1, n0 - 1))
    idx = {}
    for j in range(1, n1 - 1):
        for i in cols:
            idx[(j, i)] = len(idx)
    nb = (("ae", 1, 0), ("aw", -1, 0), ("an", 0, 1), ("as", 0, -1), ("ane", 1, 1), ("anw", -1, 1),
          ("ase", 1, -1), ("asw", -1, -1))
    rows, cs, vals = [], [], []
    rhs = np.zeros(len(idx))
    for (j, i), r in idx.items():
        rows.append(r); cs.append(r); vals.append(a["ap"][j, i])
        rhs[r] = q[j, i]
        for name, di, dj in nb:
            ii, jj = i + di, j + dj
            if periodic:
                ii %= n0 - 1
            if (jj, ii) in idx:
                rows.append(r); cs.append(idx[(jj, ii)]); vals.append(a[name][j, i])
            else:
                rhs[r] -= a[name][j, i] * phi0[jj, ii]
    A = sp.csr_matrix((vals, (rows, cs)), shape=(len(idx), len(idx)))
    x = spla.spsolve(A.tocsc(), rhs)
    phi = phi0.copy()
    for (j, i), r in idx.items():
        phi[j, i] = x[r]
    if periodic:
        phi[:, -1] = phi[:, 0]
    return phi


def test_sip_seam_matches_oracle_pressure_correction():
    """The oracle's tightly converged SIP solve of one step (pcor from zero, q the continuity
    source of PSolver.cpp:1390-1449) against the seam on the oracle's own nine planes."""
    from oracle import oracle
    g = ogrid(33, 25, skew=0.1)
    c = oracle.OracleCase(g, Re=100.0, Ri=1.0, dt=2e-3, tol_gs=1e-13, maxit_gs=600, tol_sip=1e-13,
                          atol_sip=1e-14, maxit_sip=20000)
    c.step(1)
    coefs = [c.field(k) for k in SIP_ORDER]
    q, ref = c.field("q"), c.field("pcor")
    rc, phi, iters = sip_gpu(g, coefs, np.zeros_like(q), q, 1)
    assert rc == 0
    err = np.linalg.norm(phi[1:-1] - ref[1:-1]) / np.linalg.norm(ref[1:-1])
    assert err < 1e-9, err
    assert np.array_equal(phi[:, -1], phi[:, 0])
    assert np.all(phi[0] == 0.0) and np.all(phi[-1] == 0.0)  # boundary rows held
    assert 1 <= iters < 400


@pytest.mark.parametrize("kind", ["ogrid", "cavity"])
def test_sip_seam_matches_direct_solve(kind):
    """A nonzero initial guess with nonzero boundary values: the seam must hold the boundary
    values and solve for the rest exactly as the stored system says."""
    from oracle import oracle
    g = ogrid(24, 17, ar=1.5, skew=0.1) if kind == "ogrid" else cavity(21, 17, skew=0.15)
    periodic = 1 if kind == "ogrid" else 0
    c = oracle.OracleCase(g, Re=100.0, dt=2e-3)
    coefs = [c.field(k) for k in SIP_ORDER]
    rng = np.random.default_rng(7)
    phi0 = rng.standard_normal((g.n1, g.n0))
    if periodic:
        phi0[:, -1] = phi0[:, 0]
    q = rng.standard_normal((g.n1, g.n0))
    ref = direct_solve(coefs, phi0, q, periodic)
    rc, phi, iters = sip_gpu(g, coefs, phi0, q, periodic)
    assert rc == 0
    err = np.linalg.norm(phi - ref) / np.linalg.norm(ref)
    assert err < 1e-10, err
    np.testing.assert_array_equal(phi[0], phi0[0])
    np.testing.assert_array_equal(phi[-1], phi0[-1])
    if not periodic:
        np.testing.assert_array_equal(phi[:, 0], phi0[:, 0])
        np.testing.assert_array_equal(phi[:, -1], phi0[:, -1])


def test_sip_seam_reports_its_cap_and_bad_arguments():
    from oracle import oracle
    from cfd_solver_b200 import _lib
    g = ogrid(33, 25, skew=0.1)
    c = oracle.OracleCase(g, Re=100.0, dt=2e-3)
    coefs = [c.field(k) for k in SIP_ORDER]
    q = np.random.default_rng(1).standard_normal((g.n1, g.n0))
    rc, phi, iters = sip_gpu(g, coefs, np.zeros_like(q), q, 1, tol=1e-15, maxit=2)
    assert rc == -5 and iters == 2  # CFD_E_MAXITER
    null = (ctypes.c_void_p * 9)()
    assert _lib.lib().cfd_sip_solve(g.n0, g.n1, 1, null, None, None, 1e-8, 10, None, None) == -1
