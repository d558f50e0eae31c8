"""CPU checks of the shallow-water oracle against the known answers the
reference's own tests assert (tests/test_coriolis.py, test_momentum.py,
test_vorticity.py), restated on the canonical 18x18 grid."""

import numpy as np

import oracle.fvx_oracle as O
from fixture_inputs import DX, DY, NX, NY, fields_2d, h_mask_2d


def _mask():
    return {k: np.asarray(v, np.float64) for k, v in O.mask2d_from_mask(h_mask_2d()).items()}


def test_coriolis_known_answers():
    z = np.zeros((NY, NX))
    one = np.ones((NY, NX))
    du, dv = O.coriolis2d(z, one, one)          # f = 1, v = 1: du = +1, dv = 0
    np.testing.assert_allclose(du[1:-1, 1:-1], 1.0, rtol=1e-12)
    np.testing.assert_allclose(dv, 0.0, atol=1e-15)
    du, dv = O.coriolis2d(one, z, one)          # f = 1, u = 1: dv = -1
    np.testing.assert_allclose(dv[1:-1, 1:-1], -1.0, rtol=1e-12)
    for a in (du, dv):                          # ghost ring zero
        assert not a[0].any() and not a[-1].any() and not a[:, 0].any() and not a[:, -1].any()
    m = _mask()
    du, dv = O.coriolis2d(one, one, one, m)
    assert not du[m["u"] == 0].any() and not dv[m["v"] == 0].any()


def test_momentum_known_answers():
    one = np.ones((NY, NX))
    for s in ("energy", "enstrophy", "al"):
        du, dv = O.momentum_advection(one, 2 * one, DX, DY, s)   # uniform flow: no tendency
        np.testing.assert_allclose(du, 0.0, atol=1e-12)
        np.testing.assert_allclose(dv, 0.0, atol=1e-12)
    F = fields_2d()
    e = O.momentum_advection(F["u"], F["v"], DX, DY, "energy")
    z = O.momentum_advection(F["u"], F["v"], DX, DY, "enstrophy")
    al = O.momentum_advection(F["u"], F["v"], DX, DY, "al")
    # the Arakawa-Lamb tendency blends the two (momentum.py:164-175)
    np.testing.assert_allclose(al[0], e[0] / 3 + 2 * z[0] / 3 + 0 * al[0], atol=1e-10)
    assert np.abs(e[0]).max() > 0 and not e[0][:2].any() and not e[0][:, -2:].any()


def test_vorticity_known_answers():
    F = fields_2d()
    one = np.ones((NY, NX))
    # solid body rotation u = -y, v = x: relative vorticity 2 everywhere inside
    yy, xx = np.meshgrid(np.arange(NY) * DY, np.arange(NX) * DX, indexing="ij")
    zeta = O.diff2d("curl", -yy, DX, DY, None, xx)
    np.testing.assert_allclose(zeta[1:-1, 1:-1], 2.0, rtol=1e-12)
    q = O.potential_vorticity_x(F["u"], F["v"], one, F["f"], DX, DY)
    assert np.isfinite(q).all()
    e = O.pv_flux(F["q"], F["u"], F["v"], "energy")
    s = O.pv_flux(F["q"], F["u"], F["v"], "enstrophy")
    al = O.pv_flux(F["q"], F["u"], F["v"], "al", alpha=0.25)
    np.testing.assert_allclose(al[1], 0.25 * e[1] + 0.75 * s[1], rtol=1e-12, atol=1e-15)
