"""cfd_gauss_solve_noalloc against cfd_gauss_solve.

The no-alloc entry point serves callers that cannot call cudaMalloc (a host whose
device memory belongs to another allocator or budget, a loop that must not take the
allocator's locks or meet an out-of-memory failure mid-step): its scratch is a static
device array, and it must give the same answer as the allocating entry point -- on two
calls in a row, since every call reuses (and leaves behind) the same scratch -- and
leave the device's free memory unchanged. This file is named to be collected last; it
also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from cfd_solver_b200.grid import cavity, ogrid

pytestmark = pytest.mark.gpu

REL = 1e-10  # the tolerance of the seam tests (tests/test_gpu_seam.py)


def _system(g, seed):
    """A gauss() system from the oracle's assembly: 25 planes in gauss() order, phi0, q."""
    from oracle import oracle
    order = ("p", "e", "s", "n", "w", "se", "sw", "ne", "nw", "ss", "ssee", "ssww", "sse", "ssw",
             "see", "sww", "nn", "nnee", "nnww", "nne", "nnw", "nee", "nww", "ee", "ww")
    c = oracle.OracleCase(g, Re=150.0, Ri=1.0, dt=2e-3, fix_T_annw=1)
    phi0 = c.field("u").copy()
    c.step(1)
    rng = np.random.default_rng(seed)
    q = c.field("qu") + 1e-3 * rng.standard_normal((g.n1, g.n0))
    return [c.field("au" + s) for s in order], phi0, q


def _solve(fn, g, coefs, phi0, q, periodic):
    import torch
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in coefs]
    ptrs = (ctypes.c_void_p * 25)(*[t.data_ptr() for t in dev])
    phi = torch.from_numpy(phi0.copy()).cuda()
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    sweeps = ctypes.c_int(0)
    torch.cuda.synchronize()
    rc = fn(g.n0, g.n1, periodic, ptrs, ctypes.c_void_p(phi.data_ptr()),
            ctypes.c_void_p(qd.data_ptr()), 1e-12, 600, ctypes.byref(sweeps), None)
    torch.cuda.synchronize()
    return rc, phi.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    from cfd_solver_b200 import _lib
    L = _lib.lib()
    cases = [(ogrid(33, 25, skew=0.1), 1, 0), (cavity(41, 33, skew=0.15), 0, 1)]
    for g, periodic, seed in cases:  # two calls in a row on the shared static scratch
        coefs, phi0, q = _system(g, seed)
        rc_a, ref = _solve(L.cfd_gauss_solve, g, coefs, phi0, q, periodic)
        rc_b, got = _solve(L.cfd_gauss_solve_noalloc, g, coefs, phi0, q, periodic)
        assert rc_a == 0 and rc_b == 0, L.cfd_last_error()
        sl = (slice(1, -1), slice(None)) if periodic else (slice(1, -1), slice(1, -1))
        err = np.linalg.norm(got[sl] - ref[sl]) / np.linalg.norm(ref[sl])
        assert err < REL, err


def test_noalloc_leaves_free_device_memory_unchanged():
    import torch
    from cfd_solver_b200 import _lib
    L = _lib.lib()
    g = ogrid(33, 25, skew=0.1)
    coefs, phi0, q = _system(g, 2)
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in coefs]
    ptrs = (ctypes.c_void_p * 25)(*[t.data_ptr() for t in dev])
    phi = torch.from_numpy(phi0.copy()).cuda()
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    sweeps = ctypes.c_int(0)

    def call():
        phi.copy_(torch.from_numpy(phi0))
        torch.cuda.synchronize()
        rc = L.cfd_gauss_solve_noalloc(g.n0, g.n1, 1, ptrs, ctypes.c_void_p(phi.data_ptr()),
                                       ctypes.c_void_p(qd.data_ptr()), 1e-12, 600, ctypes.byref(sweeps), None)
        torch.cuda.synchronize()
        assert rc == 0, L.cfd_last_error()

    call()  # warm: the first call on a device looks up the array's address
    free0, _ = torch.cuda.mem_get_info()
    call()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_sweeps_never_exceed_an_odd_cap():
    from cfd_solver_b200 import _lib
    L = _lib.lib()
    g = ogrid(33, 25, skew=0.1)
    coefs, phi0, q = _system(g, 3)
    import torch
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in coefs]
    ptrs = (ctypes.c_void_p * 25)(*[t.data_ptr() for t in dev])
    phi = torch.from_numpy(phi0.copy()).cuda()
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    sweeps = ctypes.c_int(0)
    rc = L.cfd_gauss_solve_noalloc(g.n0, g.n1, 1, ptrs, ctypes.c_void_p(phi.data_ptr()),
                                   ctypes.c_void_p(qd.data_ptr()), 1e-300, 5, ctypes.byref(sweeps), None)
    torch.cuda.synchronize()
    assert rc == -5  # CFD_E_MAXITER
    assert sweeps.value == 4


def test_noalloc_rejects_grids_beyond_its_limit():
    from cfd_solver_b200 import _lib
    L = _lib.lib()
    n0 = 2049
    n1 = (1 << 20) // n0 + 2  # n0 * n1 just above CFD_NOALLOC_MAX_POINTS
    dummy = (ctypes.c_void_p * 25)(*([1] * 25))
    rc = L.cfd_gauss_solve_noalloc(n0, n1, 1, dummy, ctypes.c_void_p(1), ctypes.c_void_p(1), 1e-8, 10,
                                   None, None)
    assert rc == -1
    assert b"limit" in L.cfd_last_error()
