"""Host side of the drop-in: batches of cases on the GPU and an INP.DAT-driven
`Solver` that mirrors the reference's `class Solver` (PSolver.cpp:11-2453).

The reference's constructor reads INP.DAT, applies the initial and boundary
conditions, assembles the coefficient matrices and runs the whole time loop;
`timeLoop()` is the per-step body. `Solver` here keeps that shape: the
constructor loads the grid and sets up the device case, `timeLoop(nsteps)`
advances it and writes the reference's output files every 100 steps
(PSolver.cpp:1989-2040).
"""
from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np

from . import _lib
from .grid import Grid, read_inp
from .outputs import write_coeff_his, write_spt, write_surf_dist


class Batch:
    """Many cases advanced together by one set of launches (cfd_batch_* of the C ABI)."""

    def __init__(self, grids, params):
        L = _lib.lib()
        if len(grids) != len(params) or not grids:
            raise ValueError("grids and params must be non-empty and of equal length")
        self.grids = list(grids)
        structs, self._keep = [], []
        for g in self.grids:
            s, keep = _lib.make_grid(g)
            structs.append(s)
            self._keep.extend(keep)
        self._garr = (_lib.CfdGrid * len(structs))(*structs)
        self._parr = (_lib.CfdParams * len(params))(*params)
        self.h = ctypes.c_void_p()
        _lib.check(L.cfd_batch_create(len(structs), self._garr, self._parr, ctypes.byref(self.h)),
                   "cfd_batch_create")
        self.steps = 0

    def step(self, n: int = 1):
        _lib.check(_lib.lib().cfd_batch_step(self.h, int(n)), "cfd_batch_step")
        self.steps += n

    def stats(self, i: int = 0) -> dict:
        s = _lib.CfdStepStats()
        _lib.check(_lib.lib().cfd_batch_stats(self.h, i, ctypes.byref(s)), "cfd_batch_stats")
        return s.as_dict()

    def plane(self, i: int, name: str) -> np.ndarray:
        g = self.grids[i]
        out = np.empty((g.n1, g.n0), dtype=np.float64)
        _lib.check(_lib.lib().cfd_batch_get_plane(self.h, i, name.encode(),
                                                   out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                   f"cfd_batch_get_plane({name})")
        return out

    def profile(self, enable: bool = True):
        _lib.check(_lib.lib().cfd_batch_profile(self.h, int(enable)), "cfd_batch_profile")

    def kernel_times(self) -> dict:
        cap = 64
        names = (ctypes.c_char_p * cap)()
        ms = (ctypes.c_double * cap)()
        cnt = (ctypes.c_longlong * cap)()
        n = _lib.lib().cfd_batch_kernel_times(self.h, names, ms, cnt, cap)
        if n < 0:
            _lib.check(n, "cfd_batch_kernel_times")
        return {names[k].decode(): (ms[k], cnt[k]) for k in range(min(n, cap))}

    def sync(self):
        _lib.check(_lib.lib().cfd_batch_sync(self.h), "cfd_batch_sync")

    def admit(self, slot: int, grid, params):
        """Write a new case into `slot` (same n0, n1, profile); the other slots keep running."""
        s, keep = _lib.make_grid(grid)
        self._keep.extend(keep)
        self.grids[slot] = grid
        _lib.check(_lib.lib().cfd_batch_admit(self.h, slot, ctypes.byref(s), ctypes.byref(params)),
                   "cfd_batch_admit")

    def admit_spec(self, slot: int, kind: str, params, ar: float = 2.0, r_outer: float = 20.0,
                   skew: float = 0.0):
        """admit() of the grid generate_on_device(kind, n0, n1, ...) would return, generated
        straight into the slot's device planes (cfd_batch_admit_spec); n0, n1 are the slot's."""
        g = self.grids[slot]
        prof = _lib.PROFILE_OGRID if kind == "ogrid" else _lib.PROFILE_CAVITY
        spec = _lib.CfdGridSpec(profile=prof, n0=g.n0, n1=g.n1, ar=ar, r_outer=r_outer, skew=skew)
        _lib.check(_lib.lib().cfd_batch_admit_spec(self.h, slot, ctypes.byref(spec), ctypes.byref(params)),
                   "cfd_batch_admit_spec")

    def set_active(self, slot: int, active: bool):
        _lib.check(_lib.lib().cfd_batch_set_active(self.h, slot, int(active)), "cfd_batch_set_active")

    def set_mg(self, nu_pre: int, nu_post: int, coarse_sweeps: int, fused: int = 0):
        _lib.check(_lib.lib().cfd_batch_set_mg(self.h, nu_pre, nu_post, coarse_sweeps, fused), "cfd_batch_set_mg")

    def set_wait_limit(self, polls: int):
        """Polls of a kernel's bounded copy wait before it gives up (negative: the default)."""
        _lib.check(_lib.lib().cfd_batch_set_wait_limit(self.h, int(polls)), "cfd_batch_set_wait_limit")

    def get_mg(self) -> tuple:
        v = [ctypes.c_int() for _ in range(4)]
        _lib.check(_lib.lib().cfd_batch_get_mg(self.h, *[ctypes.byref(x) for x in v]), "cfd_batch_get_mg")
        return tuple(x.value for x in v)

    def autotune(self, steps: int = 5) -> tuple:
        """Pick the fastest multigrid schedule by timing candidates from the current state
        (which is restored). Returns ((pre, post, coarse, fused), ms per step)."""
        out = (ctypes.c_int * 4)()
        ms = ctypes.c_double()
        _lib.check(_lib.lib().cfd_batch_autotune(self.h, steps, out, ctypes.byref(ms)), "cfd_batch_autotune")
        return tuple(out), ms.value

    def all_stats(self) -> list:
        n = len(self.grids)
        arr = (_lib.CfdStepStats * n)()
        _lib.check(_lib.lib().cfd_batch_fetch_stats(self.h, arr, n), "cfd_batch_fetch_stats")
        return [a.as_dict() for a in arr]

    def stream(self) -> int:
        return int(_lib.lib().cfd_batch_stream(self.h) or 0)

    def launches(self) -> int:
        return int(_lib.lib().cfd_batch_launches(self.h))

    def work(self) -> tuple:
        w = (ctypes.c_ulonglong * 4)()
        _lib.check(_lib.lib().cfd_batch_work(self.h, w), "cfd_batch_work")
        return tuple(int(x) for x in w)

    def state_bytes(self) -> int:
        return int(_lib.lib().cfd_batch_state_bytes(self.h))

    def get_state(self, buf):
        """Copy the resident state into `buf` (a writable buffer of state_bytes())."""
        _lib.check(_lib.lib().cfd_batch_get_state(self.h, ctypes.c_void_p(_addr(buf)), self.state_bytes()),
                   "cfd_batch_get_state")

    def set_state(self, buf):
        _lib.check(_lib.lib().cfd_batch_set_state(self.h, ctypes.c_void_p(_addr(buf)), self.state_bytes()),
                   "cfd_batch_set_state")

    def save(self, path):
        """Write a checkpoint file of every case's state (cfd_batch_save)."""
        _lib.check(_lib.lib().cfd_batch_save(self.h, str(path).encode()), "cfd_batch_save")

    def load(self, path):
        """Restore a checkpoint written by save() for the same cases (cfd_batch_load)."""
        _lib.check(_lib.lib().cfd_batch_load(self.h, str(path).encode()), "cfd_batch_load")

    def close(self):
        if self.h:
            _lib.lib().cfd_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Pool(Batch):
    """A slot pool (cfd_pool_*): cases of any size placed in one device arena of
    `hbm_budget` bytes as they are admitted and given back when released. Every Batch
    method works on it; its case indices are slots."""

    def __init__(self, hbm_budget: int, max_cases: int = 256, precision: int = _lib.PRECISION_FP64):
        L = _lib.lib()
        self.grids = [None] * int(max_cases)
        self._keep = []
        self.h = ctypes.c_void_p()
        _lib.check(L.cfd_pool_create(int(hbm_budget), int(max_cases), int(precision), ctypes.byref(self.h)),
                   "cfd_pool_create")
        self.steps = 0

    def place(self, grid, params):
        """Admit a case; returns its slot, or None when no free region of the budget (or no
        slot) is left for it (CFD_E_OOM: nothing changed)."""
        s, keep = _lib.make_grid(grid)
        slot = ctypes.c_int(-1)
        rc = _lib.lib().cfd_pool_admit(self.h, ctypes.byref(s), ctypes.byref(params), ctypes.byref(slot))
        if rc == -3:
            return None
        _lib.check(rc, "cfd_pool_admit")
        self._keep.extend(keep)
        self.grids[slot.value] = grid
        return slot.value

    def release(self, slot: int):
        _lib.check(_lib.lib().cfd_pool_release(self.h, int(slot)), "cfd_pool_release")
        self.grids[slot] = None

    def free(self) -> tuple:
        """(free bytes, largest free region) of the budget."""
        a, b = ctypes.c_size_t(), ctypes.c_size_t()
        _lib.check(_lib.lib().cfd_pool_free(self.h, ctypes.byref(a), ctypes.byref(b)), "cfd_pool_free")
        return a.value, b.value

    @staticmethod
    def case_bytes(grid) -> int:
        prof = _lib.PROFILE_CAVITY if grid.kind == "cavity" else _lib.PROFILE_OGRID
        return int(_lib.lib().cfd_pool_case_bytes(grid.n0, grid.n1, prof))


def serve(requests, classes, steps_per_tick: int = 50, slots=None, hbm_budget: int = 0,
          precision: int = _lib.PRECISION_FP64):
    """Run a real-time serving session (cfd_serve).

    requests: list of (arrival_s, grid, params, tol, max_steps); classes: list of
    (template grid, profile) with slots: fixed slots per class; or slots=None: admission by
    free device memory into a slot pool of hbm_budget bytes (requests of any size; classes
    may be empty); precision: CFD_PRECISION_* of the session (every request's params must
    match). Returns (list of result dicts, stats dict).
    """
    keep = []
    grids = []
    for g, prof in classes:
        s, k = _lib.make_grid(g)
        keep.extend(k)
        grids.append(s)
    garr = (_lib.CfdGrid * max(1, len(grids)))(*grids)
    profs = (ctypes.c_int * max(1, len(classes)))(*[p for _, p in classes])
    sl = (ctypes.c_int * len(classes))(*slots) if slots is not None else None
    cfg = _lib.CfdServeConfig(nclasses=len(classes), class_grids=garr, class_profile=profs,
                              class_slots=sl, hbm_budget=int(hbm_budget), steps_per_tick=steps_per_tick,
                              precision=precision)
    rgrids = []
    reqs = (_lib.CfdRequest * len(requests))()
    for i, (t, g, prm, tol, mx) in enumerate(requests):
        s, k = _lib.make_grid(g)
        keep.extend(k)
        rgrids.append(s)
        reqs[i].arrival_s = t
        reqs[i].grid = ctypes.pointer(rgrids[-1])
        reqs[i].params = prm
        reqs[i].tol = tol
        reqs[i].max_steps = mx
    res = (_lib.CfdResult * len(requests))()
    st = _lib.CfdServeStats()
    _lib.check(_lib.lib().cfd_serve(ctypes.byref(cfg), reqs, len(requests), res, ctypes.byref(st)),
               "cfd_serve")
    results = [{k: getattr(r, k) for k, _ in r._fields_} for r in res]
    stats = {k: getattr(st, k) for k, _ in st._fields_}
    return results, stats


def _addr(buf) -> int:
    if isinstance(buf, np.ndarray):
        return buf.ctypes.data
    if hasattr(buf, "data_ptr"):  # torch tensor (pinned host memory)
        return buf.data_ptr()
    return ctypes.addressof(ctypes.c_char.from_buffer(buf))


def case_params(grid: Grid | None = None, **kw) -> _lib.CfdParams:
    """cfd_params with the reference's defaults, the profile taken from the grid."""
    if grid is not None and "profile" not in kw:
        kw["profile"] = _lib.PROFILE_CAVITY if grid.kind == "cavity" else _lib.PROFILE_OGRID
    if kw.get("profile") == _lib.PROFILE_CAVITY:
        # the reference's T-solve coefficient slip (atnw in the annw slot, PSolver.cpp:1290)
        # makes the energy equation unstable on skewed grids; the cavity uses the
        # Fortran-intent coefficient (solver.for:907) unless told otherwise
        kw.setdefault("fix_T_annw", 1)
    return _lib.default_params(**kw)


class Solver:
    """INP.DAT-driven solver with the reference's outputs (PSolver.cpp:502-1043, 1051-2065)."""

    def __init__(self, inp: str | Path = "INP.DAT", workdir: str | Path | None = None,
                 grid: Grid | None = None, profile: str = "ogrid", **params):
        self.workdir = Path(workdir) if workdir is not None else Path(inp).resolve().parent
        self.grid = grid if grid is not None else read_inp(inp, kind=profile)
        self.params = case_params(self.grid, **params)
        self.batch = Batch([self.grid], [self.params])
        self.loop = 0
        # the reference keeps time as an int (PSolver.cpp:186); time-accurate mode, a float
        self.time = 0.0 if self.params.time_accurate else 0
        self.history = []

    def fields(self) -> dict:
        return {k: self.batch.plane(0, k) for k in ("u", "v", "T", "p", "si", "vort")}

    def timeLoop(self, nsteps: int, output_every: int = 100, write: bool = True):
        """Advance nsteps; write spt100.dat / COEFF_HIS*.dat / SURF_DIST.dat when loop % 100 == 0."""
        for _ in range(nsteps):
            self.batch.step(1)
            st = self.batch.stats(0)
            self.time = st["time"] if self.params.time_accurate else int(self.time + self.params.dt)
            self.history.append(st)
            if write and output_every and self.loop % output_every == 0:
                self.write_outputs(st)
            self.loop += 1
        return self.history[-1] if self.history else None

    def run_steps(self, nsteps: int):
        """Advance nsteps without per-step host work (throughput path)."""
        self.batch.step(nsteps)
        self.loop += nsteps
        st = self.batch.stats(0)
        if self.params.time_accurate:
            self.time = st["time"]
        else:
            for _ in range(nsteps):
                self.time = int(self.time + self.params.dt)
        return st

    def write_outputs(self, st: dict):
        f = self.fields()
        g = self.grid
        write_spt(self.workdir / "spt100.dat", g, f)
        write_coeff_his(self.workdir / "COEFF_HIS.dat", self.time, st["cl"], st["cd"], st["cm"], st["nu"])
        write_coeff_his(self.workdir / "COEFF_HIS_pr_vor.dat", self.time, st["cl_pr"], st["cd_pr"],
                        st["cl_vor"], st["cd_vor"])
        write_surf_dist(self.workdir / "SURF_DIST.dat", g, f)

    def close(self):
        self.batch.close()
