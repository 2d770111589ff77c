"""Grid generation on the GPU (cfd_grid_generate) against the Python generator.

Both evaluate the same analytic map and metric formulas; they differ only in the last bits
of the transcendental functions, so the planes agree to 1e-13 of each plane's magnitude and
a case stepped on either grid gives the same fields to 1e-10.
"""
import numpy as np
import pytest

from cfd_solver_b200 import grid as G

SHAPES = [("ogrid", dict(n0=65, n1=49, ar=2.0, skew=0.1)),
          ("ogrid", dict(n0=33, n1=25, ar=1.0, skew=0.0)),
          ("ogrid", dict(n0=129, n1=97, ar=3.0, skew=0.2, r_outer=30.0)),
          ("cavity", dict(n0=65, n1=65, skew=0.15)),
          ("cavity", dict(n0=33, n1=49, skew=0.0))]


def _host(kind, kw):
    if kind == "ogrid":
        return G.ogrid(kw["n0"], kw["n1"], ar=kw.get("ar", 2.0), r_outer=kw.get("r_outer", 20.0),
                       skew=kw.get("skew", 0.0))
    return G.cavity(kw["n0"], kw["n1"], skew=kw.get("skew", 0.1))


def test_invalid_spec_is_rejected_before_any_device_work():
    from cfd_solver_b200 import _lib
    for kind, kw in [("ogrid", dict(n0=7, n1=20)), ("ogrid", dict(n0=33, n1=25, ar=0.5)),
                     ("cavity", dict(n0=6, n1=33))]:
        with pytest.raises(_lib.CfdError):
            G.generate_on_device(kind, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,kw", SHAPES)
def test_device_grid_matches_host_grid(kind, kw):
    dev = G.generate_on_device(kind, **kw)
    host = _host(kind, kw)
    for k in G.FIELD_ORDER:
        a, b = getattr(dev, k), getattr(host, k)
        # beta vanishes on an orthogonal grid (both sides are rounding noise there): it is
        # measured against alpha, the scale of the metric tensor it belongs to
        scale = max(np.abs(b).max(), np.abs(host.alph).max() if k == "beta" else 0.0)
        assert np.abs(a - b).max() <= 1e-13 * scale, k
    for k in ("xnix", "xniy", "xnox", "xnoy"):
        np.testing.assert_allclose(getattr(dev, k), getattr(host, k), rtol=0, atol=1e-13)
    if kind == "ogrid":  # the seam column repeats column 0 exactly
        for k in G.FIELD_ORDER:
            np.testing.assert_array_equal(getattr(dev, k)[:, -1], getattr(dev, k)[:, 0])


@pytest.mark.gpu
def test_case_on_device_grid_steps_like_host_grid():
    from cfd_solver_b200.solver import Batch, case_params
    kw = dict(n0=65, n1=49, ar=2.0, skew=0.1)
    out = []
    for g in (G.generate_on_device("ogrid", **kw), _host("ogrid", kw)):
        with Batch([g], [case_params(g, Re=200.0, Ri=1.0, dt=1e-3)]) as b:
            b.step(5)
            out.append({k: b.plane(0, k) for k in ("u", "v", "T", "p")})
    for k in out[0]:
        d = np.linalg.norm(out[0][k] - out[1][k]) / np.linalg.norm(out[1][k])
        assert d < 1e-10, (k, d)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,kw", [SHAPES[0], SHAPES[2], SHAPES[3]])
def test_admit_spec_steps_like_admit_of_the_generated_grid(kind, kw):
    """A case generated straight into a slot (cfd_batch_admit_spec) steps bit for bit like
    cfd_batch_admit() of the grid cfd_grid_generate() returns: the same padded grid planes,
    the same Chebyshev bounds (the device scan rounds every operation as the host loop
    does) and the same initial state, which admit_spec writes on the device (the O-grid
    case has a rotating wall, F != 0, so its wall row carries the wall velocity; the batch
    has taken an odd number of steps, so the state goes to the second T/up/vp buffers)."""
    from cfd_solver_b200.solver import Batch, case_params
    spec_kw = {k: v for k, v in kw.items() if k not in ("n0", "n1")}
    gdev = G.generate_on_device(kind, **kw)
    first = G.generate_on_device(kind, **dict(kw, skew=0.05))  # the slots' first occupant
    prm = case_params(gdev, Re=200.0, Ri=1.0, dt=1e-3, F=0.3 if kind == "ogrid" else 0.0)
    with Batch([first, first], [prm, prm]) as b:
        b.step(3)
        b.admit_spec(0, kind, prm, **spec_kw)
        b.admit(1, gdev, prm)
        for name in ("x", "y", "xix", "ety", "alph", "beta", "gam", "jac", "u", "v", "T", "p", "up", "vp"):
            assert np.array_equal(b.plane(0, name), b.plane(1, name)), name
        b.step(4)
        for name in ("u", "v", "T", "p", "up", "vp"):
            assert np.array_equal(b.plane(0, name), b.plane(1, name)), name
        s0, s1 = b.stats(0), b.stats(1)
        assert s0["it_mom"] == s1["it_mom"] and s0["it_p"] == s1["it_p"] and s0["nu"] == s1["nu"]


@pytest.mark.gpu
def test_admit_spec_rejects_a_mismatch_and_leaves_the_slot():
    from cfd_solver_b200 import _lib
    from cfd_solver_b200.solver import Batch, case_params
    g = G.generate_on_device("ogrid", n0=65, n1=49)
    prm = case_params(g, Re=200.0, dt=1e-3)
    with Batch([g], [prm]) as b:
        b.step(2)
        before = {k: b.plane(0, k) for k in ("x", "alph", "u", "p")}
        with pytest.raises(_lib.CfdError):  # another profile than the slot's
            b.admit_spec(0, "cavity", case_params(g, Re=200.0, dt=1e-3, profile=_lib.PROFILE_CAVITY))
        with pytest.raises(_lib.CfdError):  # an invalid spec (semi-axis ratio below 1)
            b.admit_spec(0, "ogrid", prm, ar=0.5)
        for k, v in before.items():
            assert np.array_equal(b.plane(0, k), v), k
        b.step(1)
        assert b.stats(0)["status"] == 0
