"""ctypes binding of libcfd_b200.so (the C ABI declared in include/cfd_b200.h).

There is no CPU fallback: if the shared library is missing or no CUDA device
is present, the calls below raise.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libcfd_b200.so"

OK = 0
ERRORS = {-1: "CFD_E_ARG", -2: "CFD_E_CUDA", -3: "CFD_E_OOM", -4: "CFD_E_DIVERGED",
          -5: "CFD_E_MAXITER", -6: "CFD_E_BREAKDOWN", -7: "CFD_E_NOTCONV"}
PROFILE_OGRID, PROFILE_CAVITY = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1

# exported symbols (kept in sync with include/cfd_b200.h; tests check both)
SYMBOLS = ("cfd_params_default", "cfd_last_error", "cfd_device_count", "cfd_set_device",
           "cfd_case_create",
           "cfd_case_step", "cfd_case_solve_to", "cfd_case_get_fields", "cfd_case_destroy",
           "cfd_batch_create", "cfd_batch_step", "cfd_batch_stats", "cfd_batch_get_plane",
           "cfd_batch_destroy", "cfd_case_bytes", "cfd_batch_profile", "cfd_batch_kernel_times",
           "cfd_batch_sync", "cfd_batch_stream", "cfd_batch_launches", "cfd_batch_work",
           "cfd_batch_state_bytes", "cfd_batch_get_state", "cfd_batch_set_state",
           "cfd_gauss_solve", "cfd_gauss_solve_noalloc", "cfd_batch_fetch_stats", "cfd_batch_admit",
           "cfd_batch_set_active", "cfd_serve", "cfd_batch_set_mg", "cfd_batch_get_mg",
           "cfd_batch_autotune", "cfd_batch_save", "cfd_batch_load", "cfd_grid_generate",
           "cfd_batch_admit_spec", "cfd_batch_set_wait_limit", "cfd_sip_solve", "cfd_pool_create",
           "cfd_pool_admit", "cfd_pool_release", "cfd_pool_free", "cfd_pool_case_bytes")

_D = ctypes.c_double
_PD = ctypes.POINTER(ctypes.c_double)


class CfdGrid(ctypes.Structure):
    _fields_ = [("n0", ctypes.c_int), ("n1", ctypes.c_int), ("dxi0", _D), ("dxi1", _D),
                ("p_grid", _D), ("a_grid", _D), ("ar", _D),
                ("x", _PD), ("y", _PD), ("xix", _PD), ("xiy", _PD), ("etx", _PD), ("ety", _PD),
                ("alph", _PD), ("beta", _PD), ("gam", _PD), ("jac", _PD),
                ("xnix", _PD), ("xniy", _PD), ("xnox", _PD), ("xnoy", _PD)]


class CfdGridSpec(ctypes.Structure):
    _fields_ = [("profile", ctypes.c_int), ("n0", ctypes.c_int), ("n1", ctypes.c_int),
                ("ar", _D), ("r_outer", _D), ("skew", _D)]


class CfdParams(ctypes.Structure):
    _fields_ = [("Re", _D), ("Ri", _D), ("Pr", _D), ("F", _D), ("alpha_deg", _D), ("dt", _D),
                ("tol_mom", _D), ("atol_mom", _D), ("tol_p", _D), ("atol_p", _D),
                ("maxit_mom", ctypes.c_int), ("maxit_p", ctypes.c_int), ("profile", ctypes.c_int),
                ("fix_T_annw", ctypes.c_int), ("fix_circ_de", ctypes.c_int),
                ("warm_start", ctypes.c_int), ("omega_p", _D), ("lid_u", _D), ("precision", ctypes.c_int),
                ("time_accurate", ctypes.c_int)]


class CfdStepStats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int), ("status", ctypes.c_int), ("it_mom", ctypes.c_int * 5),
                ("it_p", ctypes.c_int), ("dmax", _D), ("cl", _D), ("cd", _D), ("cm", _D),
                ("nu", _D), ("circ", _D), ("cl_pr", _D), ("cd_pr", _D), ("cl_vor", _D),
                ("cd_vor", _D), ("q_l1", _D), ("q_l2", _D), ("q_max", _D), ("dT_l1", _D),
                ("dT_max", _D), ("p_res_rel", _D), ("mass_res_rel", _D), ("steady_res", _D),
                ("steady_res_rel", _D), ("time", _D)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "it_mom"}
        d["it_mom"] = list(self.it_mom)
        return d


class CfdRequest(ctypes.Structure):
    _fields_ = [("arrival_s", _D), ("grid", ctypes.POINTER(CfdGrid)), ("params", CfdParams),
                ("tol", _D), ("max_steps", ctypes.c_int)]


class CfdResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("slot", ctypes.c_int), ("steps", ctypes.c_int),
                ("arrival_s", _D), ("admit_s", _D), ("done_s", _D), ("latency_s", _D),
                ("nu", _D), ("steady_res_rel", _D), ("mass_res_rel", _D)]


class CfdServeConfig(ctypes.Structure):
    _fields_ = [("nclasses", ctypes.c_int), ("class_grids", ctypes.POINTER(CfdGrid)),
                ("class_profile", ctypes.POINTER(ctypes.c_int)),
                ("class_slots", ctypes.POINTER(ctypes.c_int)), ("hbm_budget", ctypes.c_size_t),
                ("steps_per_tick", ctypes.c_int), ("precision", ctypes.c_int)]


class CfdServeStats(ctypes.Structure):
    _fields_ = [("makespan_s", _D), ("cases_per_s", _D), ("p50_latency_s", _D),
                ("p99_latency_s", _D), ("mean_latency_s", _D), ("steps", ctypes.c_longlong),
                ("cell_updates", ctypes.c_longlong), ("converged", ctypes.c_int),
                ("failed", ctypes.c_int), ("slots", ctypes.c_int)]


class CfdError(RuntimeError):
    pass


_lib = None


def lib():
    """Load the solver library (raises if it is missing: the product has no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("CFD_B200_LIB", LIB_PATH))
    if not path.exists():
        raise CfdError(f"{path} not built: run `make -C cfd_solver_b200/csrc` "
                       "(or __graft_entry__.build()); there is no CPU fallback")
    L = ctypes.CDLL(str(path))
    vp = ctypes.c_void_p
    L.cfd_params_default.argtypes = [ctypes.POINTER(CfdParams)]
    L.cfd_params_default.restype = None
    L.cfd_last_error.restype = ctypes.c_char_p
    L.cfd_device_count.argtypes = [ctypes.POINTER(ctypes.c_int)]
    L.cfd_set_device.argtypes = [ctypes.c_int]
    L.cfd_case_create.argtypes = [ctypes.POINTER(CfdGrid), ctypes.POINTER(CfdParams), ctypes.POINTER(vp)]
    L.cfd_case_step.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CfdStepStats)]
    L.cfd_case_solve_to.argtypes = [vp, _D, ctypes.c_int, ctypes.POINTER(CfdStepStats)]
    L.cfd_case_get_fields.argtypes = [vp] + [_PD] * 6
    L.cfd_case_destroy.argtypes = [vp]
    L.cfd_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(CfdGrid), ctypes.POINTER(CfdParams),
                                   ctypes.POINTER(vp)]
    L.cfd_batch_step.argtypes = [vp, ctypes.c_int]
    L.cfd_batch_stats.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CfdStepStats)]
    L.cfd_batch_get_plane.argtypes = [vp, ctypes.c_int, ctypes.c_char_p, _PD]
    L.cfd_batch_destroy.argtypes = [vp]
    L.cfd_case_bytes.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.cfd_case_bytes.restype = ctypes.c_size_t
    L.cfd_batch_profile.argtypes = [vp, ctypes.c_int]
    L.cfd_batch_kernel_times.argtypes = [vp, ctypes.POINTER(ctypes.c_char_p), _PD,
                                         ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
    L.cfd_batch_sync.argtypes = [vp]
    L.cfd_batch_stream.argtypes = [vp]
    L.cfd_batch_stream.restype = vp
    L.cfd_batch_launches.argtypes = [vp]
    L.cfd_batch_launches.restype = ctypes.c_longlong
    L.cfd_batch_work.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong)]
    L.cfd_batch_state_bytes.argtypes = [vp]
    L.cfd_batch_state_bytes.restype = ctypes.c_size_t
    L.cfd_batch_get_state.argtypes = [vp, vp, ctypes.c_size_t]
    L.cfd_batch_set_state.argtypes = [vp, vp, ctypes.c_size_t]
    L.cfd_gauss_solve.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_void_p,
                                  _D, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]
    L.cfd_gauss_solve_noalloc.argtypes = L.cfd_gauss_solve.argtypes
    L.cfd_sip_solve.argtypes = L.cfd_gauss_solve.argtypes
    L.cfd_batch_fetch_stats.argtypes = [vp, ctypes.POINTER(CfdStepStats), ctypes.c_int]
    L.cfd_batch_admit.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CfdGrid), ctypes.POINTER(CfdParams)]
    L.cfd_batch_set_active.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.cfd_batch_set_mg.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    ip = ctypes.POINTER(ctypes.c_int)
    L.cfd_batch_get_mg.argtypes = [vp, ip, ip, ip, ip]
    L.cfd_batch_set_wait_limit.argtypes = [vp, ctypes.c_longlong]
    L.cfd_pool_create.argtypes = [ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.cfd_pool_admit.argtypes = [vp, ctypes.POINTER(CfdGrid), ctypes.POINTER(CfdParams), ip]
    L.cfd_pool_release.argtypes = [vp, ctypes.c_int]
    L.cfd_pool_free.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
    L.cfd_pool_case_bytes.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.cfd_pool_case_bytes.restype = ctypes.c_size_t
    L.cfd_batch_autotune.argtypes = [vp, ctypes.c_int, ip, ctypes.POINTER(ctypes.c_double)]
    L.cfd_batch_save.argtypes = [vp, ctypes.c_char_p]
    L.cfd_batch_load.argtypes = [vp, ctypes.c_char_p]
    L.cfd_grid_generate.argtypes = [ctypes.POINTER(CfdGridSpec), _PD, _PD]
    L.cfd_batch_admit_spec.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CfdGridSpec), ctypes.POINTER(CfdParams)]
    L.cfd_serve.argtypes = [ctypes.POINTER(CfdServeConfig), ctypes.POINTER(CfdRequest), ctypes.c_int,
                            ctypes.POINTER(CfdResult), ctypes.POINTER(CfdServeStats)]
    special = {"cfd_params_default", "cfd_last_error", "cfd_case_bytes", "cfd_batch_stream",
               "cfd_batch_launches", "cfd_batch_state_bytes", "cfd_pool_case_bytes"}
    for name in SYMBOLS:
        if name not in special:
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def check(rc: int, what: str = ""):
    if rc != OK:
        msg = lib().cfd_last_error().decode(errors="replace")
        raise CfdError(f"{what}: {ERRORS.get(rc, rc)}: {msg}")


def default_params(**overrides) -> CfdParams:
    p = CfdParams()
    lib().cfd_params_default(ctypes.byref(p))
    alias = {"alpha": "alpha_deg"}
    for k, v in overrides.items():
        k = alias.get(k, k)
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def make_grid(g) -> tuple[CfdGrid, list]:
    """CfdGrid view of a cfd_solver_b200.grid.Grid; returns (struct, keep-alive arrays)."""
    keep = []

    def ptr(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return a.ctypes.data_as(_PD)

    s = CfdGrid(n0=g.n0, n1=g.n1, dxi0=g.dxi0, dxi1=g.dxi1, p_grid=g.p_grid, a_grid=g.a_grid, ar=g.ar,
                x=ptr(g.x), y=ptr(g.y), xix=ptr(g.xix), xiy=ptr(g.xiy), etx=ptr(g.etx),
                ety=ptr(g.ety), alph=ptr(g.alph), beta=ptr(g.beta), gam=ptr(g.gam),
                jac=ptr(g.jac), xnix=ptr(g.xnix), xniy=ptr(g.xniy), xnox=ptr(g.xnox),
                xnoy=ptr(g.xnoy))
    return s, keep
