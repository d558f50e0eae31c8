"""Pin the CPU oracle to the reference's own golden fixtures and known answers.

CPU-only: the oracle is checked against finitevolX's FP64 golden ``.npz``
outputs (copied into tests/golden/ref) at the reference's own tolerance
(rtol 1e-12, atol 1e-14; finitevolX tests/fixtures/_helpers.py:49-108), and
against known-answer tests restated from the reference's test suite.
"""

import pathlib

import numpy as np
import pytest

import oracle.fvx_oracle as O
from tests.fixture_inputs import DX, DY, fields_2d, h_mask_2d

GOLD = pathlib.Path(__file__).parent / "golden" / "ref"
RTOL, ATOL = 1e-12, 1e-14


def golden(op, method, variant):
    with np.load(GOLD / f"{op}__{method}__{variant}.npz") as d:
        return {k: np.asarray(d[k]) for k in d.files}


@pytest.fixture(scope="module")
def F():
    return fields_2d()


@pytest.fixture(scope="module")
def M():
    return O.mask2d_from_mask(h_mask_2d())


VARIANTS = ("unmasked", "masked")


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("method", ("upwind1", "weno5"))
def test_advection2d_golden(F, M, method, variant):
    mask = M if variant == "masked" else None
    out = O.advection2d(F["h"], F["u"], F["v"], DX, DY, method, mask)
    np.testing.assert_allclose(out, golden("Advection2D", f"__call___{method}", variant)["out"],
                               rtol=RTOL, atol=ATOL)


DIFF_SPECS = (("diff_x_T_to_U", "h"), ("diff_y_T_to_V", "h"), ("diff_y_U_to_X", "u"),
              ("diff_x_V_to_X", "v"), ("diff_y_X_to_U", "h"), ("diff_x_X_to_V", "h"),
              ("diff_x_U_to_T", "u"), ("diff_y_V_to_T", "v"), ("laplacian", "h"))


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("name,arg", DIFF_SPECS)
def test_difference2d_golden(F, M, name, arg, variant):
    mask = M if variant == "masked" else None
    out = O.diff2d(name, F[arg], DX, DY, mask)
    np.testing.assert_allclose(out, golden("Difference2D", name, variant)["out"], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("variant", VARIANTS)
def test_difference2d_compound_golden(F, M, variant):
    mask = M if variant == "masked" else None
    g = golden("Difference2D", "divergence", variant)["out"]
    np.testing.assert_allclose(O.diff2d("divergence", F["u"], DX, DY, mask, F["v"]), g, rtol=RTOL, atol=ATOL)
    g = golden("Difference2D", "curl", variant)["out"]
    np.testing.assert_allclose(O.diff2d("curl", F["u"], DX, DY, mask, F["v"]), g, rtol=RTOL, atol=ATOL)
    g = golden("Difference2D", "grad_perp", variant)
    u, v = O.diff2d("grad_perp", F["h"], DX, DY, mask)
    np.testing.assert_allclose(u, g["out0"], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(v, g["out1"], rtol=RTOL, atol=ATOL)


INTERP_SPECS = (("T_to_U", "h"), ("T_to_V", "h"), ("T_to_X", "h"), ("X_to_U", "q"), ("X_to_V", "q"),
                ("U_to_T", "u"), ("V_to_T", "v"), ("X_to_T", "q"), ("U_to_X", "u"), ("V_to_X", "v"),
                ("U_to_V", "u"), ("V_to_U", "v"))


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("name,arg", INTERP_SPECS)
def test_interpolation2d_golden(F, M, name, arg, variant):
    mask = M if variant == "masked" else None
    out = O.interp2d(name, F[arg], mask)
    np.testing.assert_allclose(out, golden("Interpolation2D", name, variant)["out"], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("variant", VARIANTS)
def test_diffusion2d_golden(F, M, variant):
    mask = M if variant == "masked" else None
    out = O.diffusion2d(F["h"], 1.0, DX, DY, mask)
    np.testing.assert_allclose(out, golden("Diffusion2D", "__call__", variant)["out"], rtol=RTOL, atol=ATOL)
    fx, fy = O.diffusion_fluxes(F["h"], 1.0, DX, DY, None if mask is None else M["u"],
                                None if mask is None else M["v"])
    g = golden("Diffusion2D", "fluxes", variant)
    np.testing.assert_allclose(fx, g["out0"], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(fy, g["out1"], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("variant", VARIANTS)
def test_biharmonic2d_golden(F, M, variant):
    mask = M if variant == "masked" else None
    out = O.biharmonic2d(F["h"], 1e-3, DX, DY, mask)
    g = golden("BiharmonicDiffusion2D", "__call__", variant)["out"]
    np.testing.assert_allclose(out, g, rtol=RTOL, atol=ATOL)


# ---------------------------------------------------------------------------
# Known-answer tests restated from the reference's suite
# ---------------------------------------------------------------------------


def test_pool_bool_docstring_examples():
    # mask/utils.py:120-137 doctest values
    h = np.array([True, True, False, True, True])
    assert O.pool_bool(h, (2,), 0.75).tolist() == [False, True, False, False, True]
    assert O.pool_bool(h, (2,), 0.75, "trailing").tolist() == [True, False, False, True, False]
    h2 = np.array([[True, True], [False, True]])
    assert O.pool_bool(h2, (2, 2), 1.0 / 8.0).all()


def test_count_contiguous_docstring_examples():
    # mask/utils.py:455-461
    h = np.array([True, True, False, True, True, True])
    assert O.count_contiguous(h, 0, True).tolist() == [2, 1, 0, 3, 2, 1]
    assert O.count_contiguous(h, 0, False).tolist() == [1, 2, 0, 1, 2, 3]


def test_dilate_mask_docstring_examples():
    # mask/utils.py:349-368
    m = np.zeros((5, 5), bool)
    m[2, 2] = True
    exp = np.zeros((5, 5), int)
    exp[1:4, 2] = 1
    exp[2, 1:4] = 1
    assert (O.dilate_mask(m).astype(int) == exp).all()
    m = np.zeros((4, 4), bool)
    m[0, 0] = True
    d = O.dilate_mask(m).astype(int)
    assert d.tolist() == [[1, 1, 0, 0], [1, 0, 0, 0], [0, 0, 0, 0], [0, 0, 0, 0]]


def test_make_sponge_docstring_examples():
    # mask/utils.py:521-536
    np.testing.assert_array_equal(O.make_sponge((6,), 2), np.array([0, .5, 1, 1, .5, 0], np.float32))
    s = O.make_sponge((5, 5), 1)
    exp = np.zeros((5, 5), np.float32)
    exp[1:4, 1:4] = 1
    np.testing.assert_array_equal(s, exp)
    np.testing.assert_array_equal(O.make_sponge((4,), 0), np.ones(4, np.float32))


def test_mask_classification_island():
    # tests/test_cgrid_mask.py island fixture: land=0, ocean classes present
    m = np.ones((20, 20), bool)
    m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = False
    m[8:12, 8:12] = False
    M = O.mask2d_from_mask(m)
    cls = M["classification"]
    assert (cls[~m] == 0).all()
    assert set(np.unique(cls[m]).tolist()) == {1, 2, 3}
    # the cells adjacent (cross) to land are coast
    assert cls[1, 5] == 1 and cls[2, 5] == 2 and cls[3, 5] == 3


def test_weno_constant_and_linear_exactness():
    # tests/test_weno.py:56-105 (constants) and :156-183 (linear exactness)
    c = np.full(7, 3.25)
    for f, n in ((O.weno3, 3), (O.weno5, 5), (O.wenoz5, 5), (O.weno7, 7)):
        np.testing.assert_allclose(f(*c[:n]), 3.25, rtol=1e-10)
    x = np.arange(9, dtype=float)  # cell averages of a linear function are exact
    np.testing.assert_allclose(O.weno5(*x[0:5]), 2.5, rtol=1e-10)
    np.testing.assert_allclose(O.weno5_right(*x[0:5]), 1.5, rtol=1e-10)
    np.testing.assert_allclose(O.weno7(*x[0:7]), 3.5, rtol=1e-10)
    np.testing.assert_allclose(O.weno9(*x[0:9]), 4.5, rtol=1e-10)
    np.testing.assert_allclose(O.weno9_right(*x[0:9]), 3.5, rtol=1e-10)


def test_weno_tables_match_published_values():
    # advection/weno.py:13 and :55 (optimal linear weights)
    np.testing.assert_allclose(O.WENO7_WEIGHTS, (1 / 35, 12 / 35, 18 / 35, 4 / 35), rtol=1e-15)
    np.testing.assert_allclose(O.WENO9_WEIGHTS, (1 / 126, 10 / 63, 10 / 21, 20 / 63, 5 / 126), rtol=1e-15)
    np.testing.assert_allclose(O.WENO7_COEFFS[0], (-1 / 4, 13 / 12, -23 / 12, 25 / 12), rtol=1e-15)
    np.testing.assert_allclose(O.WENO7_BETA[0][0, 0], 547.0 / 240.0, rtol=1e-15)
    np.testing.assert_allclose(O.WENO9_BETA[2][2, 2], 77051.0 / 1680.0, rtol=1e-15)


def test_limiters_known_values():
    # tests/test_limiters.py: phi(1)=1 for every limiter, phi(r<=0)=0
    for f in O.LIMITERS.values():
        assert f(np.array(1.0)) == pytest.approx(1.0)
        assert f(np.array(-1.0)) == 0.0


def test_jacobian_known_answers():
    # tests/test_jacobian.py:94-102 antisymmetry, J(f,f)=0, :187-196 J(x,y)=1
    rng = np.random.default_rng(0)
    f = rng.standard_normal((12, 10))
    g = rng.standard_normal((12, 10))
    np.testing.assert_allclose(O.arakawa_jacobian(f, g, 0.1, 0.2), -O.arakawa_jacobian(g, f, 0.1, 0.2), atol=1e-12)
    np.testing.assert_allclose(O.arakawa_jacobian(f, f, 0.1, 0.2), 0.0, atol=1e-12)
    x = np.linspace(0, 1, 10)
    y = np.linspace(0, 1, 12)
    X, Y = np.meshgrid(x, y)
    J = O.arakawa_jacobian(X, Y, x[1] - x[0], y[1] - y[0])
    np.testing.assert_allclose(J, 1.0, rtol=1e-12)


def test_rk3_order_on_linear_ode():
    # tests/test_timestepping.py:68-91 (order check on dy/dt = -y)
    errs = []
    for dt in (0.1, 0.05):
        y = np.array([1.0])
        for _ in range(int(round(1 / dt))):
            y = O.rk3_ssp_step(y, lambda z: -z, dt)
        errs.append(abs(y[0] - np.exp(-1.0)))
    assert 7.0 < errs[0] / errs[1] < 9.5


def test_dst_solver_exact_identity():
    # solve_helmholtz_dst: the solution satisfies the discrete 5-point
    # Dirichlet Helmholtz equation to rounding
    rng = np.random.default_rng(1)
    f = rng.standard_normal((24, 30))
    for lam in (0.0, 3.0):
        psi = O.solve_helmholtz_dst(f, 0.1, 0.07, lam)
        r = O.dirichlet_helmholtz_apply(psi, 0.1, 0.07, lam) - f
        assert np.abs(r).max() < 1e-10 * np.abs(f).max()


def test_dst_matrix_form_matches_fft_form():
    rng = np.random.default_rng(2)
    f = rng.standard_normal((16, 20))
    Sy, Sx = O.dst1_matrix(16), O.dst1_matrix(20)
    lam = 0.5
    den = O.dst1_eigenvalues(16, 0.3)[:, None] + O.dst1_eigenvalues(20, 0.2)[None, :] - lam
    psi = 4.0 / (17 * 21) * Sy @ ((Sy @ f @ Sx) / den) @ Sx
    np.testing.assert_allclose(psi, O.solve_helmholtz_dst(f, 0.2, 0.3, lam), rtol=1e-11, atol=1e-13)


def test_multigrid_pcg_converges():
    # tests/test_multigrid.py:318-334: MG-preconditioned CG converges
    n = 32
    m = np.ones((n, n))
    m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = 0
    m[10:16, 12:20] = 0
    mg = O.mg_build(m, 1.0 / n, 1.0 / n, lambda_=10.0)
    rng = np.random.default_rng(3)
    f = rng.standard_normal((n, n)) * m
    L = mg["levels"][0]
    x, info = O.pcg(lambda z: O.mg_apply(z, L), f,
                    precond=lambda r: O.mg_vcycle(mg, np.zeros_like(r), r), rtol=1e-10, atol=1e-10)
    assert info["converged"] and info["iterations"] < 30
    assert np.linalg.norm(O.mg_apply(x, L) - f) < 1e-8 * np.linalg.norm(f)


def test_multigrid_transfer_constant_preserving():
    # tests/test_multigrid.py:157-199
    m = np.ones((16, 16))
    c = np.full((8, 8), 2.5)
    np.testing.assert_allclose(O.mg_prolong(c, np.ones((8, 8)), m), 2.5)
    np.testing.assert_allclose(O.mg_restrict(np.full((16, 16), 1.5), m, np.ones((8, 8))), 1.5)


def test_vertical_modes_roundtrip():
    A = O.build_coupling_matrix([400.0, 1100.0, 2600.0], [9.81, 0.025, 0.0125])
    rr, l2m, m2l = O.decompose_vertical_modes(A, 1e-4)
    np.testing.assert_allclose(l2m @ m2l, np.eye(3), atol=1e-12)
    assert rr.shape == (3,)


# ---------------------------------------------------------------------------
# Shallow-water operators: Coriolis2D (operators/coriolis.py:86-133),
# Vorticity2D (operators/vorticity.py:60-235), MomentumAdvection2D
# (diffusion/momentum.py:108-216); goldens from finitevolX
# tests/fixtures/_gen_golden.py:477-547 (vorticity), :852-864 (momentum),
# :968-987 (Coriolis), f = 1 + 0.1 y (tests/fixtures/inputs.py:284-287).
# ---------------------------------------------------------------------------

def _pair(g):
    return g["out0"], g["out1"]


@pytest.mark.parametrize("variant", VARIANTS)
def test_coriolis2d_golden(F, M, variant):
    mask = M if variant == "masked" else None
    for got, ref in zip(O.coriolis2d(F["u"], F["v"], F["f"], mask), _pair(golden("Coriolis2D", "__call__", variant))):
        np.testing.assert_allclose(got, ref, rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("variant", VARIANTS)
def test_vorticity2d_golden(F, M, variant):
    mask = M if variant == "masked" else None
    g = golden("Vorticity2D", "relative_vorticity", variant)["out"]
    np.testing.assert_allclose(O.diff2d("curl", F["u"], DX, DY, mask, F["v"]), g, rtol=RTOL, atol=ATOL)
    g = golden("Vorticity2D", "potential_vorticity", variant)["out"]
    np.testing.assert_allclose(O.potential_vorticity_x(F["u"], F["v"], F["h"], F["f"], DX, DY, mask), g,
                               rtol=RTOL, atol=ATOL)
    for scheme, name in (("energy", "pv_flux_energy_conserving"), ("enstrophy", "pv_flux_enstrophy_conserving"),
                         ("al", "pv_flux_arakawa_lamb")):
        got = O.pv_flux(F["q"], F["u"], F["v"], scheme, mask=mask)
        for a, b in zip(got, _pair(golden("Vorticity2D", name, variant))):
            np.testing.assert_allclose(a, b, rtol=RTOL, atol=ATOL, err_msg=name)


@pytest.mark.parametrize("variant", VARIANTS)
def test_momentum_advection2d_golden(F, M, variant):
    mask = M if variant == "masked" else None
    got = O.momentum_advection(F["u"], F["v"], DX, DY, "energy", mask)
    for a, b in zip(got, _pair(golden("MomentumAdvection2D", "__call__", variant))):
        np.testing.assert_allclose(a, b, rtol=RTOL, atol=ATOL)
