"""The C-ABI library loads on a CPU-only host and exports every entry point that
include/*.h declares (no compute call is made here)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(cfd_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_header_declares_the_abi():
    names = declared_symbols()
    assert {"cfd_case_create", "cfd_case_step", "cfd_batch_create", "cfd_batch_step"} <= names


def test_library_exports_every_declared_symbol():
    from cfd_solver_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.skip("library not built")
    L = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in sorted(declared_symbols()) if not hasattr(L, n)]
    assert not missing, missing
    assert set(_lib.SYMBOLS) <= declared_symbols()


def test_params_default_are_the_reference_values():
    from cfd_solver_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.skip("library not built")
    p = _lib.default_params()
    # PSolver.cpp:160-174 and the solver locals at PSolver.cpp:2086-2088, 2290-2291
    assert (p.Re, p.Ri, p.Pr, p.F, p.alpha_deg, p.dt) == (1000.0, 0.0, 0.71, 0.0, 82.0, 1e-4)
    assert p.tol_mom == 0.75e-2 and p.tol_p == 0.75e-2 and p.omega_p == 1.0
