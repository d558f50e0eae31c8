"""GPU parity: stencil operators and masks vs the oracle and the reference goldens.

Tolerances (stated per the parity bar):
  * FP64 kernels vs reference goldens: rtol 1e-12, atol 1e-14 (the
    reference's own golden tolerance);
  * FP64 kernels vs the FP64 oracle on seeded fields: max|a-b| <= 1e-12 *
    max|b| (normwise relative, max norm);
  * FP32 kernels vs the FP64 oracle: max|a-b| <= 1e-5 * max|b|;
  * masks, tier codes, classification, irregular-boundary lists: bit-exact.
"""

import pathlib

import numpy as np
import pytest
import torch

import finitevolx_b200 as fvx
import oracle.fvx_oracle as O
from tests.fixture_inputs import DX, DY, fields_2d, h_mask_2d

pytestmark = pytest.mark.gpu
GOLD = pathlib.Path(__file__).parent / "golden" / "ref"
METHODS = O.ADVECTION_METHODS


def golden(op, method, variant):
    with np.load(GOLD / f"{op}__{method}__{variant}.npz") as d:
        return {k: np.asarray(d[k]) for k in d.files}


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device="cuda")


def host(t):
    return t.detach().cpu().numpy().astype(np.float64)


def close_norm(a, b, rel):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max()
    assert err <= rel * scale, f"max err {err:.3e} > {rel:.0e} * {scale:.3e}"


@pytest.fixture(scope="module")
def F(cuda_ok):
    return fields_2d()


@pytest.fixture(scope="module")
def MG(cuda_ok):
    return fvx.Mask2D.from_mask(h_mask_2d())


@pytest.fixture(scope="module")
def MO():
    return O.mask2d_from_mask(h_mask_2d())


def island_mask(ny, nx, seed):
    rng = np.random.default_rng(seed)
    h = np.ones((ny, nx), bool)
    h[0, :] = h[-1, :] = h[:, 0] = h[:, -1] = False
    for _ in range(4):
        y, x = rng.integers(2, ny - 6), rng.integers(2, nx - 6)
        h[y:y + rng.integers(2, 6), x:x + rng.integers(2, 6)] = False
    return h


def rand_fields(ny, nx, seed):
    rng = np.random.default_rng(seed)
    h = O.kminus3_field(ny, nx, seed) + 2.0
    u = rng.standard_normal((ny, nx))
    v = rng.standard_normal((ny, nx))
    return h, u, v


# ---------------------------------------------------------------- goldens --
@pytest.mark.parametrize("variant", ("unmasked", "masked"))
@pytest.mark.parametrize("method", ("upwind1", "weno5"))
def test_advection_golden_fp64(F, MG, method, variant):
    grid = fvx.ArakawaCGrid2D.from_interior(16, 16, 1.0, 1.0)
    adv = fvx.Advection2D(grid, MG if variant == "masked" else None)
    out = adv(dev(F["h"]), dev(F["u"]), dev(F["v"]), method=method)
    g = golden("Advection2D", f"__call___{method}", variant)["out"]
    np.testing.assert_allclose(host(out), g, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("variant", ("unmasked", "masked"))
def test_difference_interp_golden_fp64(F, MG, variant):
    grid = fvx.ArakawaCGrid2D.from_interior(16, 16, 1.0, 1.0)
    m = MG if variant == "masked" else None
    D = fvx.Difference2D(grid, m)
    for name, arg in (("diff_x_T_to_U", "h"), ("diff_y_T_to_V", "h"), ("diff_y_U_to_X", "u"),
                      ("diff_x_V_to_X", "v"), ("diff_y_X_to_U", "h"), ("diff_x_X_to_V", "h"),
                      ("diff_x_U_to_T", "u"), ("diff_y_V_to_T", "v"), ("laplacian", "h")):
        out = getattr(D, name)(dev(F[arg]))
        np.testing.assert_allclose(host(out), golden("Difference2D", name, variant)["out"], rtol=1e-12,
                                   atol=1e-14, err_msg=name)
    np.testing.assert_allclose(host(D.divergence(dev(F["u"]), dev(F["v"]))),
                               golden("Difference2D", "divergence", variant)["out"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(host(D.curl(dev(F["u"]), dev(F["v"]))),
                               golden("Difference2D", "curl", variant)["out"], rtol=1e-12, atol=1e-14)
    u, v = D.grad_perp(dev(F["h"]))
    g = golden("Difference2D", "grad_perp", variant)
    np.testing.assert_allclose(host(u), g["out0"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(host(v), g["out1"], rtol=1e-12, atol=1e-14)
    I = fvx.Interpolation2D(grid, m)
    for name, arg in (("T_to_U", "h"), ("T_to_V", "h"), ("T_to_X", "h"), ("X_to_U", "q"), ("X_to_V", "q"),
                      ("U_to_T", "u"), ("V_to_T", "v"), ("X_to_T", "q"), ("U_to_X", "u"), ("V_to_X", "v"),
                      ("U_to_V", "u"), ("V_to_U", "v")):
        out = getattr(I, name)(dev(F[arg]))
        np.testing.assert_allclose(host(out), golden("Interpolation2D", name, variant)["out"], rtol=1e-12,
                                   atol=1e-14, err_msg=name)


@pytest.mark.parametrize("variant", ("unmasked", "masked"))
def test_diffusion_golden_fp64(F, MG, variant):
    grid = fvx.ArakawaCGrid2D.from_interior(16, 16, 1.0, 1.0)
    m = MG if variant == "masked" else None
    d = fvx.Diffusion2D(grid, m)
    np.testing.assert_allclose(host(d(dev(F["h"]), 1.0)), golden("Diffusion2D", "__call__", variant)["out"],
                               rtol=1e-12, atol=1e-14)
    fx, fy = d.fluxes(dev(F["h"]), 1.0)
    g = golden("Diffusion2D", "fluxes", variant)
    np.testing.assert_allclose(host(fx), g["out0"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(host(fy), g["out1"], rtol=1e-12, atol=1e-14)
    b = fvx.BiharmonicDiffusion2D(grid, m)
    np.testing.assert_allclose(host(b(dev(F["h"]), 1e-3)),
                               golden("BiharmonicDiffusion2D", "__call__", variant)["out"], rtol=1e-12, atol=1e-14)


# ------------------------------------------------------------------ masks --
MASK_KEYS = ("h", "u", "v", "xy_corner", "xy_corner_strict", "xy_corner_y_wall", "xy_corner_x_wall",
             "xy_corner_convex", "xy_corner_valid", "classification")


@pytest.mark.parametrize("case", ("fixture", "island", "random", "all_ocean", "all_land", "thin"))
def test_mask_build_bit_exact(cuda_ok, case):
    if case == "fixture":
        h = h_mask_2d()
    elif case == "island":
        h = island_mask(40, 52, 0)
    elif case == "random":
        h = np.random.default_rng(5).random((37, 61)) > 0.3
    elif case == "all_ocean":
        h = np.ones((12, 9), bool)
    elif case == "all_land":
        h = np.zeros((12, 9), bool)
    else:
        h = np.random.default_rng(6).random((3, 70)) > 0.2
    ref = O.mask2d_from_mask(h, sponge_width=3)
    got = fvx.Mask2D.from_mask(h, sponge_width=3)
    for k in MASK_KEYS:
        a = getattr(got, k).cpu().numpy()
        assert (a == ref[k]).all(), k
    sc = got.stencil_capability
    for k in ("x_pos", "x_neg", "y_pos", "y_neg"):
        assert (getattr(sc, k).cpu().numpy() == ref[k]).all(), k
    assert (got.xy_corner_strict_irrbound_rows.cpu().numpy() == ref["xy_corner_strict_irrbound_rows"]).all()
    assert (got.xy_corner_strict_irrbound_cols.cpu().numpy() == ref["xy_corner_strict_irrbound_cols"]).all()
    assert (got.sponge.cpu().numpy() == ref["sponge"]).all()
    for d, (p, n) in (("x", ("x_pos", "x_neg")), ("y", ("y_pos", "y_neg"))):
        hier = got.get_adaptive_masks(direction=d, stencil_sizes=(2, 4, 6, 8, 10))
        rh = O.adaptive_masks(ref[p], ref[n], (2, 4, 6, 8, 10))
        for s in rh:
            assert (hier[s].cpu().numpy() == rh[s]).all(), (d, s)


def test_mask_source_u_adaptive(cuda_ok):
    h = island_mask(30, 33, 2)
    ref = O.mask2d_from_mask(h)
    got = fvx.Mask2D.from_mask(h)
    hier = got.get_adaptive_masks(direction="x", source="u", stencil_sizes=(2, 4, 6))
    xp, xn = O.count_contiguous(ref["u"], 1, True), O.count_contiguous(ref["u"], 1, False)
    rh = O.adaptive_masks(xp, xn, (2, 4, 6))
    for s in rh:
        assert (hier[s].cpu().numpy() == rh[s]).all()


# -------------------------------------------------------------- advection --
@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("masked", (False, True))
def test_advection_all_methods_fp64(cuda_ok, method, masked):
    ny, nx = 40, 52
    h, u, v = rand_fields(ny, nx, 11)
    hm = island_mask(ny, nx, 3)
    mo = O.mask2d_from_mask(hm) if masked else None
    mg = fvx.Mask2D.from_mask(hm) if masked else None
    ref = O.advection2d(h, u, v, 0.3, 0.2, method, mo)
    grid = fvx.ArakawaCGrid2D(Nx=nx, Ny=ny, Lx=0.3 * (nx - 2), Ly=0.2 * (ny - 2), dx=0.3, dy=0.2)
    got = fvx.Advection2D(grid, mg)(dev(h), dev(u), dev(v), method=method)
    close_norm(host(got), ref, 1e-12)
    # structure: ghost plus the first interior ring stay exactly zero
    g = host(got)
    assert (g[:2] == 0).all() and (g[-2:] == 0).all() and (g[:, :2] == 0).all() and (g[:, -2:] == 0).all()


@pytest.mark.parametrize("method", ("weno5", "weno7", "weno9", "van_leer", "wenoz5", "upwind3"))
def test_advection_fp32_within_1e5(cuda_ok, method):
    ny, nx = 66, 130
    h = O.kminus3_field(ny, nx, 1) + 1.0
    psi = O.fourier_streamfunction(ny - 2, nx - 2, 1.0, 1.0, 2)
    u, v = O.diff2d("grad_perp", psi, 1.0, 1.0)
    ref = O.advection2d(h, u, v, 1.0, 1.0, method)
    got = fvx.Advection2D(fvx.ArakawaCGrid2D(nx, ny, nx - 2.0, ny - 2.0, 1.0, 1.0))(
        dev(h, torch.float32), dev(u, torch.float32), dev(v, torch.float32), method=method)
    assert got.dtype == torch.float32
    close_norm(host(got), ref, 1e-5)


@pytest.mark.parametrize("method", METHODS + ("wenoz3",))
def test_face_flux_fp64(cuda_ok, method):
    ny, nx = 21, 34
    h, u, v = rand_fields(ny, nx, 4)
    R = fvx.Reconstruction2D(fvx.ArakawaCGrid2D.from_interior(nx - 2, ny - 2, 1.0, 1.0))
    if method in O.LIMITERS:
        fe = R.tvd_x(dev(h), dev(u), limiter=method)
        fn_ = R.tvd_y(dev(h), dev(v), limiter=method)
    else:
        fe = getattr(R, f"{method}_x")(dev(h), dev(u))
        fn_ = getattr(R, f"{method}_y")(dev(h), dev(v))
    close_norm(host(fe), O.face_flux_x(h, u, method), 1e-12)
    close_norm(host(fn_), O.face_flux_y(h, v, method), 1e-12)


def test_upwind_flux_blend_matches_masked_path(cuda_ok):
    ny, nx = 30, 41
    h, u, v = rand_fields(ny, nx, 8)
    hm = island_mask(ny, nx, 9)
    mg = fvx.Mask2D.from_mask(hm)
    grid = fvx.ArakawaCGrid2D.from_interior(nx - 2, ny - 2, 1.0, 1.0)
    R = fvx.Reconstruction2D(grid)
    hier = mg.get_adaptive_masks(direction="x", stencil_sizes=(2, 4, 6))
    fe = fvx.upwind_flux(dev(h), dev(u), 1, {2: R.upwind1_x, 4: R.weno3_x, 6: R.weno5_x}, hier)
    mo = O.mask2d_from_mask(hm)
    hx = O.adaptive_masks(mo["x_pos"], mo["x_neg"], (2, 4, 6))
    ref = O.upwind_flux_x(h, u, hx, {2: "upwind1", 4: "weno3", 6: "weno5"})
    close_norm(host(fe), ref, 1e-12)
    close_norm(host(R.weno5_x_masked(dev(h), dev(u), mg)), ref, 1e-12)


def test_advection_edge_cases(cuda_ok):
    # minimum sizes, all-negative flow, all-land mask, constant field -> zero tendency
    for method, n in (("weno9", 8), ("weno9", 9), ("weno7", 6), ("weno5", 4), ("upwind1", 3),
                      ("minmod", 3)):
        for sign in (-1.0, 1.0):
            h, u, v = rand_fields(n, n + 3, 1)
            u, v = sign * np.abs(u), sign * np.abs(v)
            ref = O.advection2d(h, u, v, 1.0, 1.0, method)
            grid = fvx.ArakawaCGrid2D(Nx=n + 3, Ny=n, Lx=n + 1.0, Ly=n - 2.0, dx=1.0, dy=1.0)
            got = fvx.Advection2D(grid)(dev(h), dev(u), dev(v), method=method)
            close_norm(host(got), ref, 1e-12)
            fe, fn_ = fvx.uv_center_flux(dev(h), dev(u), dev(v), grid, method)
            close_norm(host(fe), O.face_flux_x(h, u, method), 1e-12)
            close_norm(host(fn_), O.face_flux_y(h, v, method), 1e-12)
    with pytest.raises(ValueError):
        fvx.Advection2D(fvx.ArakawaCGrid2D.from_interior(5, 5, 1.0, 1.0))(
            dev(np.ones((7, 7))), dev(np.ones((7, 7))), dev(np.ones((7, 7))), method="weno9")
    with pytest.raises(ValueError):
        fvx.Advection2D(fvx.ArakawaCGrid2D.from_interior(8, 8, 1.0, 1.0))(
            dev(np.ones((10, 10))), dev(np.ones((10, 10))), dev(np.ones((10, 10))), method="weno11")
    land = fvx.Mask2D.from_mask(np.zeros((12, 12), bool))
    out = fvx.Advection2D(fvx.ArakawaCGrid2D.from_interior(10, 10, 1.0, 1.0), land)(
        dev(np.random.rand(12, 12)), dev(np.ones((12, 12))), dev(np.ones((12, 12))), method="weno5")
    assert (host(out) == 0).all()
    c = fvx.Advection2D(fvx.ArakawaCGrid2D.from_interior(20, 20, 1.0, 1.0))(
        dev(np.full((22, 22), 3.0)), dev(np.ones((22, 22))), dev(np.ones((22, 22))), method="weno5")
    assert np.abs(host(c)).max() < 1e-12


# ------------------------------------------------- jacobian / bc / rk3 -----
def test_jacobian_fp64_and_batch(cuda_ok):
    rng = np.random.default_rng(0)
    f = rng.standard_normal((3, 2, 17, 23))
    g = rng.standard_normal((3, 2, 17, 23))
    got = fvx.arakawa_jacobian(dev(f), dev(g), 0.1, 0.3)
    assert tuple(got.shape) == (3, 2, 15, 21)
    close_norm(host(got), O.arakawa_jacobian(f, g, 0.1, 0.3), 1e-12)
    x = np.linspace(0, 1, 10)
    y = np.linspace(0, 1, 12)
    X, Y = np.meshgrid(x, y)
    J = fvx.arakawa_jacobian(dev(X), dev(Y), x[1] - x[0], y[1] - y[0])
    np.testing.assert_allclose(host(J), 1.0, rtol=1e-12)


def test_periodic_and_pad(cuda_ok):
    a = np.random.default_rng(1).standard_normal((2, 9, 13))
    got = fvx.enforce_periodic(dev(a))
    for b in range(2):
        np.testing.assert_array_equal(host(got)[b], O.enforce_periodic(a[b]))
        np.testing.assert_array_equal(host(fvx.pad_interior(dev(a[b]))), O.pad_interior_constant(a[b]))


def test_rk3_with_advection_fp64(cuda_ok):
    ny, nx = 34, 34
    h, u, v = rand_fields(ny, nx, 3)
    grid = fvx.ArakawaCGrid2D(Nx=nx, Ny=ny, Lx=nx - 2.0, Ly=ny - 2.0, dx=1.0, dy=1.0)
    adv = fvx.Advection2D(grid)
    ud, vd = dev(u), dev(v)
    got = fvx.rk3_ssp_step(dev(h), lambda q: adv(fvx.enforce_periodic(q), ud, vd, "weno5"), 0.05)
    ref = O.rk3_ssp_step(h, lambda q: O.advection2d(O.enforce_periodic(q), u, v, 1.0, 1.0, "weno5"), 0.05)
    close_norm(host(got), ref, 1e-12)
    got = fvx.heun_step({"q": dev(h)}, lambda s: {"q": adv(s["q"], ud, vd, "upwind1")}, 0.05)["q"]
    ref = O.heun_step(h, lambda q: O.advection2d(q, u, v, 1.0, 1.0, "upwind1"), 0.05)
    close_norm(host(got), ref, 1e-12)


def test_no_host_fallback_without_library(monkeypatch, cuda_ok):
    import finitevolx_b200._lib as L
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", pathlib.Path("/nonexistent/libfvx.so"))
    with pytest.raises(RuntimeError):
        fvx.enforce_periodic(dev(np.zeros((5, 5))))


# interior tiles: at 150 x 270 most 64 x 16 tiles lie at least the halo from
# every edge and take the kernels' branch-free interior bodies; the edge
# tiles keep the boundary ladders -- both against the oracle
@pytest.mark.parametrize("method", METHODS)
def test_advection_interior_tiles_fp64(cuda_ok, method):
    ny, nx = 150, 270
    h, u, v = rand_fields(ny, nx, 21)
    ref = O.advection2d(h, u, v, 0.3, 0.2, method)
    grid = fvx.ArakawaCGrid2D(Nx=nx, Ny=ny, Lx=0.3 * (nx - 2), Ly=0.2 * (ny - 2), dx=0.3, dy=0.2)
    close_norm(host(fvx.Advection2D(grid)(dev(h), dev(u), dev(v), method=method)), ref, 1e-12)


@pytest.mark.parametrize("method", ("weno5", "wenoz5", "weno7", "weno9", "van_leer", "upwind3"))
def test_advection_interior_tiles_fp32(cuda_ok, method):
    ny, nx = 150, 270
    h = O.kminus3_field(ny, nx, 2) + 1.0
    psi = O.fourier_streamfunction(ny - 2, nx - 2, 1.0, 1.0, 3)
    u, v = O.diff2d("grad_perp", psi, 1.0, 1.0)
    ref = O.advection2d(h, u, v, 1.0, 1.0, method)
    got = fvx.Advection2D(fvx.ArakawaCGrid2D(nx, ny, nx - 2.0, ny - 2.0, 1.0, 1.0))(
        dev(h, torch.float32), dev(u, torch.float32), dev(v, torch.float32), method=method)
    close_norm(host(got), ref, 1e-5)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-5)])
def test_biharmonic_jacobian_interior_tiles(cuda_ok, dtype, tol):
    ny, nx = 150, 270
    rng = np.random.default_rng(22)
    h = O.kminus3_field(ny, nx, 4)
    g = O.kminus3_field(ny, nx, 5)
    grid = fvx.ArakawaCGrid2D(Nx=nx, Ny=ny, Lx=0.3 * (nx - 2), Ly=0.2 * (ny - 2), dx=0.3, dy=0.2)
    got = fvx.BiharmonicDiffusion2D(grid)(dev(h, dtype), 1e-3)
    close_norm(host(got), O.biharmonic2d(h, 1e-3, 0.3, 0.2), tol)
    mask = rng.random((ny, nx)) > 0.2
    got = fvx.BiharmonicDiffusion2D(grid, fvx.Mask2D.from_mask(mask))(dev(h, dtype), 1e-3)
    close_norm(host(got), O.biharmonic2d(h, 1e-3, 0.3, 0.2, O.mask2d_from_mask(mask)), tol)
    got = fvx.arakawa_jacobian(dev(h, dtype), dev(g, dtype), 0.3, 0.2)
    close_norm(host(got), O.arakawa_jacobian(h, g, 0.3, 0.2), tol)
