"""Host-side contract of the library on a machine without a GPU: the batch constructor
fails loudly (there is no CPU path to fall back to), an invalid case is rejected before
any device is looked for, and the admission budget (cfd_case_bytes) covers at least the
case's FP64 planes and grows with the grid."""
import pytest

from cfd_solver_b200 import _lib
from cfd_solver_b200 import grid as G

NPLANES_FP64 = 54  # FP64 planes per case: grid 10, pressure stencil 9, state 9, u*/v* 2,
#                    right-hand sides 5, sweep scratch 5, q/pcor/diagnostics 5, normals 1,
#                    BiCGStab vectors 8


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


pytestmark = pytest.mark.skipif(not _lib.LIB_PATH.exists(), reason="library not built")


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_batch_without_a_gpu_fails_loudly():
    from cfd_solver_b200.solver import Batch, case_params
    g = G.ogrid(33, 25)
    with pytest.raises(_lib.CfdError, match="no CUDA device"):
        Batch([g], [case_params(g)])


def test_invalid_case_is_rejected_before_the_device_lookup():
    from cfd_solver_b200.solver import Batch, case_params
    g = G.ogrid(33, 25)
    with pytest.raises(_lib.CfdError, match="dt, Re, Pr"):
        Batch([g], [case_params(g, dt=0.0)])
    with pytest.raises(_lib.CfdError, match="unknown precision"):
        Batch([g], [case_params(g, precision=7)])


def test_case_bytes_budget():
    L = _lib.lib()
    for prof in (_lib.PROFILE_OGRID, _lib.PROFILE_CAVITY):
        prev = 0
        for n in (65, 129, 257, 513, 1025):
            b = L.cfd_case_bytes(n, n, prof)
            assert b >= NPLANES_FP64 * n * n * 8, (prof, n, b)
            assert b <= 2 * NPLANES_FP64 * n * n * 8 + (1 << 20), (prof, n, b)
            assert b > prev
            prev = b
        assert L.cfd_case_bytes(7, 65, prof) == 0 and L.cfd_case_bytes(65, 5, prof) == 0


def test_serve_rejects_bad_requests_before_any_device_work():
    """cfd_serve checks every request (a grid of one of the slot classes, the slots'
    precision) and the slot counts before it creates its batch."""
    from cfd_solver_b200.solver import case_params, serve
    g = G.cavity(33, 33)
    cls = [(g, _lib.PROFILE_CAVITY)]
    ok = (0.0, g, case_params(g), 1e-8, 10)
    other = G.cavity(65, 65)
    with pytest.raises(_lib.CfdError, match="request 1 matches no slot class"):
        serve([ok, (0.1, other, case_params(other), 1e-8, 10)], cls, slots=[2])
    with pytest.raises(_lib.CfdError, match="request 0 has another precision"):
        serve([(0.0, g, case_params(g, precision=_lib.PRECISION_MIXED), 1e-8, 10)], cls, slots=[2])
    with pytest.raises(_lib.CfdError, match="class_slots must be > 0"):
        serve([ok], cls, slots=[0])


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_serve_without_a_gpu_fails_loudly():
    from cfd_solver_b200.solver import case_params, serve
    g = G.cavity(33, 33)
    with pytest.raises(_lib.CfdError, match="no CUDA device"):
        serve([(0.0, g, case_params(g), 1e-8, 10)], [(g, _lib.PROFILE_CAVITY)], slots=[2])


def test_pool_case_bytes_cover_both_arenas():
    """cfd_pool_case_bytes: a case's FP64 planes and its FP32 levels and planes, each part
    256-byte aligned -- at least the FP64 planes, and growing with the grid."""
    L = _lib.lib()
    for prof in (_lib.PROFILE_OGRID, _lib.PROFILE_CAVITY):
        prev = 0
        for n in (33, 65, 129, 257, 513, 1025):
            b = L.cfd_pool_case_bytes(n, n, prof)
            assert b % 256 == 0 and b >= NPLANES_FP64 * n * n * 8 and b > prev, (prof, n, b)
            prev = b
        assert L.cfd_pool_case_bytes(7, 65, prof) == 0


def test_serve_by_free_memory_rejects_bad_requests_before_any_device_work():
    """With no fixed slots cfd_serve admits by free device memory: any grid size is taken,
    but a request larger than the whole budget, of another precision or without a grid is
    rejected before the session's pool exists (so also on a host without a GPU)."""
    from cfd_solver_b200.solver import Pool, case_params, serve
    g = G.cavity(65, 65)
    ok = (0.0, g, case_params(g), 1e-8, 10)
    with pytest.raises(_lib.CfdError, match="CFD_E_OOM: cfd_serve: request 0 needs more device memory"):
        serve([ok], [], slots=None, hbm_budget=Pool.case_bytes(g) - 256)
    with pytest.raises(_lib.CfdError, match="request 1 has another precision"):
        serve([ok, (0.1, g, case_params(g, precision=_lib.PRECISION_MIXED), 1e-8, 10)], [], slots=None,
              hbm_budget=1 << 30)


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_pool_without_a_gpu_fails_loudly():
    from cfd_solver_b200.solver import Pool
    with pytest.raises(_lib.CfdError, match="no CUDA device"):
        Pool(1 << 30, max_cases=4)


def test_seams_reject_bad_arguments_before_any_device_work():
    import ctypes
    L = _lib.lib()
    nulls9 = (ctypes.c_void_p * 9)()
    nulls25 = (ctypes.c_void_p * 25)()
    one = ctypes.c_void_p(8)
    # sip9p seam: grid too small, null planes, a cap below one iteration
    assert L.cfd_sip_solve(7, 25, 1, nulls9, one, one, 1e-8, 10, None, None) == -1
    assert L.cfd_sip_solve(33, 25, 1, nulls9, one, one, 1e-8, 10, None, None) == -1
    assert b"null coefficient plane" in L.cfd_last_error()
    assert L.cfd_sip_solve(33, 25, 1, None, one, one, 1e-8, 0, None, None) == -1
    # gauss seams
    for fn in (L.cfd_gauss_solve, L.cfd_gauss_solve_noalloc):
        assert fn(33, 25, 1, nulls25, one, one, 1e-8, 10, None, None) == -1
        assert fn(33, 25, 1, None, one, one, 1e-8, 1, None, None) == -1
    assert L.cfd_batch_set_wait_limit(None, 0) == -1
