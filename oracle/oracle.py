"""ctypes wrapper of the oracle's C restatement (oracle/cfd_oracle.c) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this module; the product path never imports it.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "liborc.so"

OGRID, CAVITY = 0, 1

DIAG_NAMES = ("loop", "time", "dmax", "cl", "cd", "cm", "nu", "circ", "cl_pr", "cd_pr",
              "cl_vor", "cd_vor", "q_l1", "q_l2", "q_max", "dT_l1", "dT_max", "du_l1",
              "it_u", "it_v", "it_T", "it_up", "it_vp", "it_sip")


class OrcParams(ctypes.Structure):
    _fields_ = [("Re", ctypes.c_double), ("Ri", ctypes.c_double), ("Pr", ctypes.c_double),
                ("F", ctypes.c_double), ("alpha_deg", ctypes.c_double), ("dt", ctypes.c_double),
                ("tol_gs", ctypes.c_double), ("tol_sip", ctypes.c_double),
                ("maxit_gs", ctypes.c_int), ("maxit_sip", ctypes.c_int),
                ("profile", ctypes.c_int), ("fix_T_annw", ctypes.c_int),
                ("fix_circ_de", ctypes.c_int), ("omega_p", ctypes.c_double),
                ("lid_u", ctypes.c_double), ("time_accurate", ctypes.c_int),
                ("atol_gs", ctypes.c_double), ("atol_sip", ctypes.c_double)]


# the reference's own values (PSolver.cpp:160-174, 2086-2088, 2290-2291)
REFERENCE_DEFAULTS = dict(Re=1000.0, Ri=0.0, Pr=0.71, F=0.0, alpha=82.0, dt=1e-4,
                          tol_gs=0.75e-2, tol_sip=0.75e-2, maxit_gs=100000, maxit_sip=100000,
                          profile=OGRID, fix_T_annw=0, fix_circ_de=0, omega_p=1.0, lid_u=1.0,
                          time_accurate=0, atol_gs=0.0, atol_sip=0.0)

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE), "_ref/liborc.so"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.POINTER(OrcParams)]
        L.orc_step.restype = ctypes.c_int
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.orc_field.restype = ctypes.POINTER(ctypes.c_double)
        L.orc_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_diag_count.restype = ctypes.c_int
        assert L.orc_diag_count() == len(DIAG_NAMES)
        _lib = L
    return _lib


def make_params(**kw) -> OrcParams:
    d = dict(REFERENCE_DEFAULTS)
    d.update(kw)
    return OrcParams(Re=d["Re"], Ri=d["Ri"], Pr=d["Pr"], F=d["F"], alpha_deg=d["alpha"],
                     dt=d["dt"], tol_gs=d["tol_gs"], tol_sip=d["tol_sip"],
                     maxit_gs=int(d["maxit_gs"]), maxit_sip=int(d["maxit_sip"]),
                     profile=int(d["profile"]), fix_T_annw=int(d["fix_T_annw"]),
                     fix_circ_de=int(d["fix_circ_de"]), omega_p=d["omega_p"], lid_u=d["lid_u"],
                     time_accurate=int(d["time_accurate"]), atol_gs=d["atol_gs"],
                     atol_sip=d["atol_sip"])


class OracleCase:
    """One case of the FP64 CPU restatement."""

    def __init__(self, grid, **params):
        L = lib()
        self.grid = grid
        if "profile" not in params:
            params["profile"] = CAVITY if grid.kind == "cavity" else OGRID
        if params["profile"] == CAVITY:
            # the C++ T-solve slot bug destabilises T on skewed grids; the cavity takes the
            # Fortran-intent coefficient by default, as the library's case_params does
            params.setdefault("fix_T_annw", 1)
        self.params = make_params(**params)
        self._planes = np.ascontiguousarray(grid.planes())
        self._normals = np.ascontiguousarray(grid.normals())
        self.h = L.orc_create(grid.n0, grid.n1, grid.dxi0, grid.dxi1, grid.ar,
                              self._planes.ctypes.data, self._normals.ctypes.data,
                              ctypes.byref(self.params))
        if not self.h:
            raise ValueError("orc_create rejected the grid")
        self.history = []

    def step(self, n: int = 1):
        hist = np.zeros((n, len(DIAG_NAMES)), dtype=np.float64)
        lib().orc_step(self.h, n, hist.ctypes.data)
        self.history.extend(hist)
        return {k: hist[:, i].copy() for i, k in enumerate(DIAG_NAMES)}

    def field(self, name: str) -> np.ndarray:
        ptr = lib().orc_field(self.h, name.encode())
        if not ptr:
            raise KeyError(name)
        n = self.grid.n0 if name.startswith("b") else self.grid.n0 * self.grid.n1
        a = np.ctypeslib.as_array(ptr, shape=(n,)).copy()
        return a if name.startswith("b") else a.reshape(self.grid.n1, self.grid.n0)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
