"""Grid generator and INP.DAT reader/writer."""
import numpy as np
import pytest

from cfd_solver_b200.grid import cavity, ogrid, read_inp, write_inp


@pytest.mark.parametrize("make", [lambda: ogrid(33, 29, skew=0.1), lambda: ogrid(24, 17, ar=1.0),
                                  lambda: cavity(33, 25, skew=0.15)])
def test_metric_identities(make):
    g = make()
    # xi_x x_xi + xi_y y_xi = 1 with centred differences of x, y (interior)
    x_xi = (g.x[1:-1, 2:] - g.x[1:-1, :-2]) / (2 * g.dxi0)
    y_xi = (g.y[1:-1, 2:] - g.y[1:-1, :-2]) / (2 * g.dxi0)
    x_et = (g.x[2:, 1:-1] - g.x[:-2, 1:-1]) / (2 * g.dxi1)
    y_et = (g.y[2:, 1:-1] - g.y[:-2, 1:-1]) / (2 * g.dxi1)
    xix, xiy = g.xix[1:-1, 1:-1], g.xiy[1:-1, 1:-1]
    etx, ety = g.etx[1:-1, 1:-1], g.ety[1:-1, 1:-1]
    assert np.allclose(xix * x_xi + xiy * y_xi, 1.0, atol=0.05)
    assert np.allclose(etx * x_et + ety * y_et, 1.0, atol=0.05)
    assert np.allclose(g.alph, g.xix ** 2 + g.xiy ** 2)
    assert np.allclose(g.gam, g.etx ** 2 + g.ety ** 2)
    assert np.allclose(g.beta, -(g.xix * g.etx + g.xiy * g.ety))


def test_ogrid_orientation_and_seam():
    g = ogrid(33, 25, skew=0.1)
    assert (g.jac < 0).all()  # orientation the reference's signed integrals assume
    for k in ("x", "y", "xix", "xiy", "etx", "ety", "alph", "beta", "gam", "jac"):
        a = getattr(g, k)
        assert np.array_equal(a[:, -1], a[:, 0])
    # body = ellipse with semi-axes 1 and 1/ar
    assert np.allclose(g.x[0] ** 2 + (g.y[0] * 2.0) ** 2, 1.0)
    # outer normal points into the domain
    r = np.stack([g.x[-1], g.y[-1]])
    assert (g.xnox * r[0] + g.xnoy * r[1] < 0).all()


def test_cavity_is_unit_square():
    g = cavity(17, skew=0.1)
    assert (g.jac > 0).all()
    assert np.allclose(g.x[:, 0], 0) and np.allclose(g.x[:, -1], 1)
    assert np.allclose(g.y[0], 0) and np.allclose(g.y[-1], 1)


def test_inp_roundtrip(tmp_path):
    g = ogrid(20, 14, skew=0.05)
    p = tmp_path / "INP.DAT"
    write_inp(g, p)
    h = read_inp(p)
    assert (h.n0, h.n1) == (g.n0, g.n1)
    for k in ("x", "y", "xix", "xiy", "etx", "ety", "alph", "beta", "gam", "jac",
              "xnix", "xniy", "xnox", "xnoy"):
        assert np.array_equal(getattr(h, k), getattr(g, k)), k
    assert h.ar == g.ar and h.dxi0 == g.dxi0


def test_inp_malformed(tmp_path):
    p = tmp_path / "INP.DAT"
    p.write_text("10 10 0.1 0.1\n0 0 2\n0 0 0 0\n1 2 3\n")
    with pytest.raises(ValueError):
        read_inp(p)
    p.write_text("x y\n")
    with pytest.raises(ValueError):
        read_inp(p)
