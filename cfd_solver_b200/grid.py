"""Grids in the reference's INP.DAT format: generators, writer and reader.

The reference reads one whitespace-separated text file, INP.DAT
(PSolver.cpp:510-547):

  line 1      n0 n1 dxi0 dxi1
  line 2      p_grid a_grid ar           (only ar is used, for the Nusselt number)
  line 3      ic1 ic2 ic3 ic4            (unused)
  n0*n1 rows  xi eta x y                 (j outer, i inner)
  n0*n1 rows  xi_x xi_y eta_x eta_y
  n0*n1 rows  alpha beta gamma           alpha = xi_x^2+xi_y^2, gamma = eta_x^2+eta_y^2,
                                         beta = -(xi_x eta_x + xi_y eta_y)
  n0*n1 rows  J                          J = x_xi y_eta - x_eta y_xi
  n0 rows     xnix xniy xnox xnoy        inner / outer boundary normals; the outer
                                         one points into the domain (inflow <=>
                                         U_inf . n_o >= 0, PSolver.cpp:1360-1362)

The reference has no grid generator. Two families are generated here:

* ``ogrid``  -- the reference's own geometry: an O-grid around an elliptic
  cylinder (semi-axes 1 and 1/ar) in elliptic coordinates, xi periodic with the
  seam column i = n0-1 duplicating i = 0, j = 0 on the body, j = n1-1 on the far
  field.  An optional skew perturbs the radial coordinate,
  mu = mu0 + (mu1 - mu0) [eta + s eta (1 - eta) sin(2 pi xi)].
  J < 0 (xi runs counter-clockwise, eta outward), the orientation the
  reference's signed line integrals assume (Nusselt number, PSolver.cpp:1965).
* ``cavity`` -- the unit square mapped to the skewed curvilinear grid
  x = xi + s xi (1 - xi) sin(2 pi eta),  y = eta + s eta (1 - eta) sin(2 pi xi).

Metrics are the exact derivatives of the mappings.  Arrays are float64,
shape (n1, n0), [j][i] order.
"""
from __future__ import annotations

import dataclasses
import math
from pathlib import Path

import numpy as np

FIELD_ORDER = ("x", "y", "xix", "xiy", "etx", "ety", "alph", "beta", "gam", "jac")


@dataclasses.dataclass
class Grid:
    """One INP.DAT grid. 2-D arrays are (n1, n0) float64; normals are (n0,)."""

    n0: int
    n1: int
    dxi0: float
    dxi1: float
    p_grid: float
    a_grid: float
    ar: float
    x: np.ndarray
    y: np.ndarray
    xix: np.ndarray
    xiy: np.ndarray
    etx: np.ndarray
    ety: np.ndarray
    alph: np.ndarray
    beta: np.ndarray
    gam: np.ndarray
    jac: np.ndarray
    xnix: np.ndarray
    xniy: np.ndarray
    xnox: np.ndarray
    xnoy: np.ndarray
    kind: str = "ogrid"
    ic: tuple = (0, 0, 0, 0)

    def planes(self) -> np.ndarray:
        """The ten 2-D planes stacked as (10, n1, n0) in FIELD_ORDER."""
        return np.stack([getattr(self, k) for k in FIELD_ORDER]).astype(np.float64)

    def normals(self) -> np.ndarray:
        """(4, n0): xnix, xniy, xnox, xnoy."""
        return np.stack([self.xnix, self.xniy, self.xnox, self.xnoy]).astype(np.float64)


def _metrics(x_xi, x_eta, y_xi, y_eta):
    jac = x_xi * y_eta - x_eta * y_xi
    xix = y_eta / jac
    xiy = -x_eta / jac
    etx = -y_xi / jac
    ety = x_xi / jac
    alph = xix * xix + xiy * xiy
    gam = etx * etx + ety * ety
    beta = -(xix * etx + xiy * ety)
    return xix, xiy, etx, ety, alph, beta, gam, jac


def ogrid(n0: int, n1: int, ar: float = 2.0, r_outer: float = 20.0,
          skew: float = 0.0) -> Grid:
    """Elliptic-cylinder O-grid (the reference's geometry).

    Semi-axes a = 1 (x) and b = 1/ar (y); far field where c*cosh(mu1) = r_outer.
    For ar == 1 the circle uses log-polar coordinates r = exp(mu).
    """
    if n0 < 8 or n1 < 6:
        raise ValueError("ogrid needs n0 >= 8 and n1 >= 6")
    if ar < 1.0:
        raise ValueError("ar must be >= 1 (semi-major axis along x)")
    xi = np.arange(n0, dtype=np.float64) / (n0 - 1)
    eta = np.arange(n1, dtype=np.float64) / (n1 - 1)
    XI, ETA = np.meshgrid(xi, eta)  # (n1, n0)
    two_pi = 2.0 * math.pi
    th = two_pi * XI
    if ar > 1.0:
        a, b = 1.0, 1.0 / ar
        c = math.sqrt(a * a - b * b)
        mu0 = math.atanh(b / a)
        mu1 = math.acosh(r_outer / c)
    else:
        c = None
        mu0, mu1 = 0.0, math.log(r_outer)
    L = mu1 - mu0
    f = ETA + skew * ETA * (1.0 - ETA) * np.sin(two_pi * XI)
    f_xi = skew * ETA * (1.0 - ETA) * two_pi * np.cos(two_pi * XI)
    f_eta = 1.0 + skew * (1.0 - 2.0 * ETA) * np.sin(two_pi * XI)
    mu = mu0 + L * f
    mu_xi, mu_eta = L * f_xi, L * f_eta
    if c is not None:
        ch, sh = np.cosh(mu), np.sinh(mu)
        ct, st = np.cos(th), np.sin(th)
        x = c * ch * ct
        y = c * sh * st
        x_mu, x_th = c * sh * ct, -c * ch * st
        y_mu, y_th = c * ch * st, c * sh * ct
    else:
        r = np.exp(mu)
        ct, st = np.cos(th), np.sin(th)
        x, y = r * ct, r * st
        x_mu, x_th = r * ct, -r * st
        y_mu, y_th = r * st, r * ct
    x_xi = x_mu * mu_xi + x_th * two_pi
    y_xi = y_mu * mu_xi + y_th * two_pi
    x_eta = x_mu * mu_eta
    y_eta = y_mu * mu_eta
    xix, xiy, etx, ety, alph, beta, gam, jac = _metrics(x_xi, x_eta, y_xi, y_eta)
    planes = dict(x=x, y=y, xix=xix, xiy=xiy, etx=etx, ety=ety, alph=alph,
                  beta=beta, gam=gam, jac=jac)
    # the seam column duplicates column 0 exactly
    for k, v in planes.items():
        v[:, n0 - 1] = v[:, 0]
    ge = np.sqrt(planes["gam"])
    xnix = planes["etx"][0] / ge[0]
    xniy = planes["ety"][0] / ge[0]
    xnox = -planes["etx"][n1 - 1] / ge[n1 - 1]
    xnoy = -planes["ety"][n1 - 1] / ge[n1 - 1]
    return Grid(n0=n0, n1=n1, dxi0=1.0 / (n0 - 1), dxi1=1.0 / (n1 - 1), p_grid=0.0,
                a_grid=float(r_outer), ar=float(ar), xnix=xnix, xniy=xniy, xnox=xnox,
                xnoy=xnoy, kind="ogrid", **planes)


def cavity(n0: int, n1: int | None = None, skew: float = 0.1) -> Grid:
    """Unit-square cavity on x = xi + s xi(1-xi) sin(2 pi eta), y = eta + s eta(1-eta) sin(2 pi xi)."""
    n1 = n0 if n1 is None else n1
    if n0 < 7 or n1 < 7:
        raise ValueError("cavity needs n0, n1 >= 7")
    xi = np.arange(n0, dtype=np.float64) / (n0 - 1)
    eta = np.arange(n1, dtype=np.float64) / (n1 - 1)
    XI, ETA = np.meshgrid(xi, eta)
    two_pi = 2.0 * math.pi
    s = skew
    x = XI + s * XI * (1.0 - XI) * np.sin(two_pi * ETA)
    y = ETA + s * ETA * (1.0 - ETA) * np.sin(two_pi * XI)
    x_xi = 1.0 + s * (1.0 - 2.0 * XI) * np.sin(two_pi * ETA)
    x_eta = s * XI * (1.0 - XI) * two_pi * np.cos(two_pi * ETA)
    y_xi = s * ETA * (1.0 - ETA) * two_pi * np.cos(two_pi * XI)
    y_eta = 1.0 + s * (1.0 - 2.0 * ETA) * np.sin(two_pi * XI)
    xix, xiy, etx, ety, alph, beta, gam, jac = _metrics(x_xi, x_eta, y_xi, y_eta)
    ge = np.sqrt(gam)
    # inner (bottom wall) normal into the fluid, outer (lid) normal into the fluid
    xnix, xniy = etx[0] / ge[0], ety[0] / ge[0]
    xnox, xnoy = -etx[n1 - 1] / ge[n1 - 1], -ety[n1 - 1] / ge[n1 - 1]
    return Grid(n0=n0, n1=n1, dxi0=1.0 / (n0 - 1), dxi1=1.0 / (n1 - 1), p_grid=0.0,
                a_grid=0.0, ar=1.0, x=x, y=y, xix=xix, xiy=xiy, etx=etx, ety=ety,
                alph=alph, beta=beta, gam=gam, jac=jac, xnix=xnix, xniy=xniy,
                xnox=xnox, xnoy=xnoy, kind="cavity")


def generate_on_device(kind: str, n0: int, n1: int | None = None, ar: float = 2.0,
                       r_outer: float = 20.0, skew: float = 0.0) -> Grid:
    """The grid of ogrid() / cavity(), generated on the GPU (cfd_grid_generate): the same
    analytic map and metric formulas, evaluated by one thread per point."""
    import ctypes
    from . import _lib
    n1 = n0 if n1 is None else n1
    prof = _lib.PROFILE_OGRID if kind == "ogrid" else _lib.PROFILE_CAVITY
    spec = _lib.CfdGridSpec(profile=prof, n0=n0, n1=n1, ar=ar, r_outer=r_outer, skew=skew)
    planes = np.empty((10, n1, n0), dtype=np.float64)
    normals = np.empty((4, n0), dtype=np.float64)
    pd = ctypes.POINTER(ctypes.c_double)
    _lib.check(_lib.lib().cfd_grid_generate(ctypes.byref(spec), planes.ctypes.data_as(pd),
                                            normals.ctypes.data_as(pd)), "cfd_grid_generate")
    f = {k: planes[q] for q, k in enumerate(FIELD_ORDER)}
    if kind == "ogrid":
        return Grid(n0=n0, n1=n1, dxi0=1.0 / (n0 - 1), dxi1=1.0 / (n1 - 1), p_grid=0.0,
                    a_grid=float(r_outer), ar=float(ar), xnix=normals[0], xniy=normals[1],
                    xnox=normals[2], xnoy=normals[3], kind="ogrid", **f)
    return Grid(n0=n0, n1=n1, dxi0=1.0 / (n0 - 1), dxi1=1.0 / (n1 - 1), p_grid=0.0, a_grid=0.0,
                ar=1.0, xnix=normals[0], xniy=normals[1], xnox=normals[2], xnoy=normals[3],
                kind="cavity", **f)


def write_inp(g: Grid, path: str | Path) -> None:
    """Write INP.DAT with round-trip (%.17g) precision."""
    n0, n1 = g.n0, g.n1
    XI, ETA = np.meshgrid(np.arange(n0) * g.dxi0, np.arange(n1) * g.dxi1)
    out = [f"{n0} {n1} {g.dxi0:.17g} {g.dxi1:.17g}",
           f"{g.p_grid:.17g} {g.a_grid:.17g} {g.ar:.17g}",
           " ".join(str(int(v)) for v in g.ic)]

    def rows(*arrs):
        stacked = np.stack([np.asarray(a, dtype=np.float64).reshape(-1) for a in arrs], axis=1)
        return "\n".join(" ".join(f"{v:.17g}" for v in r) for r in stacked)

    out.append(rows(XI, ETA, g.x, g.y))
    out.append(rows(g.xix, g.xiy, g.etx, g.ety))
    out.append(rows(g.alph, g.beta, g.gam))
    out.append(rows(g.jac))
    out.append(rows(g.xnix, g.xniy, g.xnox, g.xnoy))
    Path(path).write_text("\n".join(out) + "\n")


def read_inp(path: str | Path, kind: str = "ogrid") -> Grid:
    """Read INP.DAT in the reference's token order (PSolver.cpp:517-547).

    Raises ValueError on a malformed or truncated file (the reference itself
    prints to stderr and carries on with uninitialised state, PSolver.cpp:511-514).
    """
    toks = Path(path).read_text().split()
    try:
        n0, n1 = int(toks[0]), int(toks[1])
    except (IndexError, ValueError) as e:
        raise ValueError(f"{path}: bad header") from e
    if n0 < 6 or n1 < 5:
        raise ValueError(f"{path}: grid {n0}x{n1} too small")
    need = 4 + 3 + 4 + n0 * n1 * (4 + 4 + 3 + 1) + 4 * n0
    if len(toks) < need:
        raise ValueError(f"{path}: truncated ({len(toks)} tokens, need {need})")
    try:
        vals = np.array([float(t) for t in toks[:need]], dtype=np.float64)
    except ValueError as e:
        raise ValueError(f"{path}: non-numeric token") from e
    dxi0, dxi1 = vals[2], vals[3]
    p_grid, a_grid, ar = vals[4], vals[5], vals[6]
    ic = tuple(int(v) for v in vals[7:11])
    pos = 11
    npts = n0 * n1
    b1 = vals[pos:pos + 4 * npts].reshape(n1, n0, 4); pos += 4 * npts
    b2 = vals[pos:pos + 4 * npts].reshape(n1, n0, 4); pos += 4 * npts
    b3 = vals[pos:pos + 3 * npts].reshape(n1, n0, 3); pos += 3 * npts
    b4 = vals[pos:pos + npts].reshape(n1, n0); pos += npts
    b5 = vals[pos:pos + 4 * n0].reshape(n0, 4)
    return Grid(n0=n0, n1=n1, dxi0=float(dxi0), dxi1=float(dxi1), p_grid=float(p_grid),
                a_grid=float(a_grid), ar=float(ar), x=b1[..., 2].copy(), y=b1[..., 3].copy(),
                xix=b2[..., 0].copy(), xiy=b2[..., 1].copy(), etx=b2[..., 2].copy(),
                ety=b2[..., 3].copy(), alph=b3[..., 0].copy(), beta=b3[..., 1].copy(),
                gam=b3[..., 2].copy(), jac=b4.copy(), xnix=b5[:, 0].copy(),
                xniy=b5[:, 1].copy(), xnox=b5[:, 2].copy(), xnoy=b5[:, 3].copy(),
                kind=kind, ic=ic)
