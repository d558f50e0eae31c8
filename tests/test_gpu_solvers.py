"""GPU parity: multigrid, PCG, masked Laplacian, PV inversion, vertical modes.

Tolerances: MG hierarchy arrays exact to 1e-15 (FP64 host build, same
formulas); operator / V-cycle / solve FP64 vs the oracle 1e-11 (normwise
relative, max norm); PCG: 2-norm relative residual <= 1e-8 checked in FP64
(the config's target), solution vs oracle PCG 1e-6; PV inversion FP64 1e-12.
"""

import numpy as np
import pytest
import torch

import finitevolx_b200 as fvx
import oracle.fvx_oracle as O

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device="cuda")


def host(t):
    return t.detach().cpu().numpy().astype(np.float64)


def rel(a, b):
    return np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-300)


def basin(n, seed=0, land=0.3):
    """Seeded coastline mask: smooth random field thresholded, largest ocean kept."""
    from scipy import ndimage
    rng = np.random.default_rng(seed)
    g = ndimage.gaussian_filter(rng.standard_normal((n, n)), sigma=max(n / 50.0, 2.0), mode="wrap")
    m = g > np.quantile(g, land)
    lab, k = ndimage.label(m)
    if k > 1:
        sizes = ndimage.sum(m, lab, range(1, k + 1))
        m = lab == (1 + int(np.argmax(sizes)))
    m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = False
    return m.astype(np.float64)


def coeff(n, seed=1):
    from scipy import ndimage
    rng = np.random.default_rng(seed)
    g = ndimage.gaussian_filter(rng.standard_normal((n, n)), sigma=max(n / 50.0, 2.0), mode="wrap")
    g /= g.std()
    return np.exp(0.5 * g)


@pytest.fixture(scope="module")
def case64(cuda_ok):
    n = 64
    m = basin(n, 3)
    c = coeff(n, 4)
    lam = 2.0
    mg = fvx.build_multigrid_solver(m, 1.0 / n, 1.0 / n, lambda_=lam, coeff=c)
    ref = O.mg_build(m, 1.0 / n, 1.0 / n, lambda_=lam, coeff=c)
    return n, m, c, lam, mg, ref


def test_mg_hierarchy_matches_oracle(case64):
    n, m, c, lam, mg, ref = case64
    assert mg.n_levels == ref["n_levels"]
    for k in range(mg.n_levels):
        got = mg.level(k)
        R = ref["levels"][k]
        for a, b in (("mask", "mask"), ("cx", "cx"), ("cy", "cy"), ("inv_diagonal", "inv")):
            np.testing.assert_allclose(host(got[a]), R[b], rtol=1e-15, atol=0, err_msg=f"level {k} {a}")


def test_mg_apply_vcycle_solve_fp64(case64):
    n, m, c, lam, mg, ref = case64
    rng = np.random.default_rng(5)
    u = rng.standard_normal((n, n))
    f = rng.standard_normal((n, n)) * m
    L0 = ref["levels"][0]
    assert rel(host(mg.apply(dev(u))), O.mg_apply(u, L0)) < 1e-12
    assert rel(host(mg.v_cycle(None, dev(f))), O.mg_vcycle(ref, np.zeros_like(f), f)) < 1e-11
    assert rel(host(mg.v_cycle(dev(u), dev(f))), O.mg_vcycle(ref, u, f)) < 1e-11
    assert rel(host(mg(dev(f))), O.mg_solve(ref, f)) < 1e-11


def test_mg_fine_levels_host_driven_path(cuda_ok):
    # 512^2: levels 512, 256 run one launch per sweep, 128 .. 8 in the single-CTA kernel
    n = 512
    m = basin(n, 6)
    c = coeff(n, 7)
    mg = fvx.build_multigrid_solver(m, 1.0 / n, 1.0 / n, lambda_=0.0, coeff=c)
    ref = O.mg_build(m, 1.0 / n, 1.0 / n, lambda_=0.0, coeff=c)
    f = np.random.default_rng(8).standard_normal((n, n)) * m
    assert rel(host(mg.v_cycle(None, dev(f))), O.mg_vcycle(ref, np.zeros_like(f), f)) < 1e-10


@pytest.mark.parametrize("dtype,sweeps,bar", [(torch.float64, 12, 1e-10), (torch.float64, 16, 1e-10),
                                              (torch.float32, 12, 1e-5), (torch.float32, 16, 1e-5)])
def test_mg_vcycle_many_sweeps(cuda_ok, dtype, sweeps, bar):
    # 12 and 16 sweeps per leg widen each tile's region past what four rows
    # per thread cover: the legs run their eight-row thread layouts (FP64
    # 512 threads x 8 rows at 512^2, FP32 1024 x 8)
    n = 512
    m = basin(n, 21)
    c = coeff(n, 22)
    kw = dict(lambda_=0.5, coeff=c, n_pre=sweeps, n_post=sweeps)
    mg = fvx.build_multigrid_solver(m, 1.0 / n, 1.0 / n, dtype=dtype, **kw)
    ref = O.mg_build(m, 1.0 / n, 1.0 / n, **kw)
    f = np.random.default_rng(23).standard_normal((n, n)) * m
    if dtype == torch.float32:
        f = f.astype(np.float32).astype(np.float64)
    u = np.random.default_rng(24).standard_normal((n, n)) * m
    if dtype == torch.float32:
        u = u.astype(np.float32).astype(np.float64)
    assert rel(host(mg.v_cycle(None, dev(f, dtype))), O.mg_vcycle(ref, np.zeros_like(f), f)) < bar
    assert rel(host(mg.v_cycle(dev(u, dtype), dev(f, dtype))), O.mg_vcycle(ref, u, f)) < bar


def test_mg_fp32_plan_coarsest_solve_in_fp64(cuda_ok):
    # FP32 plans run the coarsest-grid solve (its 50 Jacobi sweeps) in FP64.
    # With no smoothing on the other levels a V-cycle is restriction ->
    # coarsest solve -> prolongation, so it matches the FP64 oracle up to the
    # FP32 rounding of the transfers
    n = 32
    m = basin(n, 17)
    c = coeff(n, 18)
    kw = dict(lambda_=1e-3, coeff=c, n_pre=0, n_post=0)
    mg = fvx.build_multigrid_solver(m, 1.0 / n, 1.0 / n, dtype=torch.float32, **kw)
    ref = O.mg_build(m, 1.0 / n, 1.0 / n, **kw)
    f = (np.random.default_rng(19).standard_normal((n, n)) * m).astype(np.float32).astype(np.float64)
    got = host(mg.v_cycle(None, dev(f, torch.float32)))
    assert rel(got, O.mg_vcycle(ref, np.zeros_like(f), f)) < 1e-6


def test_mg_shape_error(cuda_ok):
    with pytest.raises(ValueError):
        fvx.build_multigrid_solver(np.ones((24, 24)), 1.0, 1.0, n_levels=5)


def _oracle_pcg_iters(mg, f, tol=1e-8, maxit=200):
    """Iterations the oracle's MG-preconditioned CG needs for ||r||_2 <= tol ||b||_2."""
    L0 = mg["levels"][0]
    x = np.zeros_like(f)
    r = f.copy()
    z = O.mg_vcycle(mg, np.zeros_like(r), r)
    p = z.copy()
    g = np.vdot(r, z)
    for k in range(1, maxit + 1):
        Ap = O.mg_apply(p, L0)
        a = g / np.vdot(p, Ap)
        x = x + a * p
        r = r - a * Ap
        if np.linalg.norm(r) <= tol * np.linalg.norm(f):
            return k
        z = O.mg_vcycle(mg, np.zeros_like(r), r)
        gn = np.vdot(r, z)
        p = z + (gn / g) * p
        g = gn
    return maxit


# lambda > 0: with zero-flux coast faces the lambda = 0 operator is singular on
# each wet region.  lambda*dx^2 = 1.5e-4 (hard) and 0.0156 (Ld = 40 km at 5 km)
@pytest.mark.parametrize("lam", (10.0, 1022.36))
@pytest.mark.parametrize("dtype", (torch.float64, torch.float32))
def test_pcg_mg_reaches_1e8(cuda_ok, dtype, lam):
    n = 256
    m = basin(n, 9)
    c = coeff(n, 10)
    mg = fvx.build_multigrid_solver(m, 1.0 / n, 1.0 / n, lambda_=lam, coeff=c, dtype=dtype)
    f = O.kminus3_field(n, n, 11) * m
    pcg = fvx.MaskedHelmholtzPCG(mg)
    x, info = pcg.solve(dev(f, dtype), rtol=1e-8, precond="mg")
    assert info["converged"] and info["rel_residual"] <= 1e-8, info
    ref = O.mg_build(m, 1.0 / n, 1.0 / n, lambda_=lam, coeff=c)
    # FP64 work vectors track the FP64 oracle; so do FP32 work vectors with
    # the FP64 iterate, FP64 inner products and the residual recomputed in
    # FP64 every iteration
    it_ref = _oracle_pcg_iters(ref, f)
    bound = it_ref + 3
    assert info["iterations"] <= bound, (info, it_ref)
    fb = host(dev(f, dtype))  # the right-hand side the solver saw
    r = fb - O.mg_apply(host(x), ref["levels"][0])
    assert np.linalg.norm(r) <= 1.01e-8 * np.linalg.norm(fb)
    # unpreconditioned CG needs many more iterations on the same problem
    x2, info2 = pcg.solve(dev(f, dtype), rtol=1e-8, precond="none", max_iter=info["iterations"] + 20)
    assert info2["iterations"] > info["iterations"]


def test_pcg_callable_preconditioner_flexible(cuda_ok):
    n = 128
    m = basin(n, 12)
    mg = fvx.build_multigrid_solver(m, 1.0 / n, 1.0 / n, lambda_=1.0)
    f = O.kminus3_field(n, n, 13) * m
    pcg = fvx.MaskedHelmholtzPCG(mg)
    pc = fvx.make_multigrid_preconditioner(mg)
    x, info = pcg.solve(dev(f), rtol=1e-8, precond=pc, flexible=True)
    assert info["converged"], info


def test_solve_cg_generic_and_masked_laplacian(cuda_ok):
    n = 64
    m = basin(n, 14)
    mg = fvx.build_multigrid_solver(m, 1.0 / n, 1.0 / n, lambda_=3.0)
    ref = O.mg_build(m, 1.0 / n, 1.0 / n, lambda_=3.0)
    f = np.random.default_rng(15).standard_normal((n, n)) * m
    x, info = fvx.solve_cg(mg.apply, dev(f), preconditioner=fvx.make_multigrid_preconditioner(mg), rtol=1e-10,
                           atol=1e-10)
    xr, ir = O.pcg(lambda z: O.mg_apply(z, ref["levels"][0]), f,
                   precond=lambda r: O.mg_vcycle(ref, np.zeros_like(r), r), rtol=1e-10, atol=1e-10)
    assert info.converged and ir["converged"]
    assert rel(host(x), xr) < 1e-6
    assert abs(info.iterations - ir["iterations"]) <= 1
    psi = np.random.default_rng(16).standard_normal((n, n))
    got = fvx.masked_laplacian(dev(psi), dev(m), 0.1, 0.2, 1.5)
    assert rel(host(got), O.masked_laplacian(psi, m, 0.1, 0.2, 1.5)) < 1e-12


def test_pv_inversion_multilayer_modes(cuda_ok):
    H = [400.0, 1100.0, 2600.0]
    gp = [9.81, 0.025, 0.0125]
    f0 = 9.375e-5
    A = fvx.build_coupling_matrix(H, gp)
    np.testing.assert_allclose(A, O.build_coupling_matrix(H, gp), rtol=1e-15)
    rr, l2m, m2l = fvx.decompose_vertical_modes(A, f0)
    rro, l2mo, m2lo = O.decompose_vertical_modes(A, f0)
    np.testing.assert_allclose(rr, rro, rtol=1e-12)
    n = 64
    dx = 5.12e6 / n
    q = np.stack([O.kminus3_field(n, n, s, std=1e-5) for s in range(3)])
    qm = fvx.layer_to_mode(dev(q), l2m)
    np.testing.assert_allclose(host(qm), np.einsum("kl,lyx->kyx", l2m, q), rtol=1e-12, atol=1e-20)
    lam = np.where(np.isfinite(rr), 1.0 / np.where(np.isfinite(rr), rr, 1.0) ** 2, 0.0)
    psim = fvx.pv_inversion(qm, dx, dx, lam)
    ref = np.stack([O.solve_helmholtz_dst(np.einsum("kl,lyx->kyx", l2m, q)[k], dx, dx, lam[k]) for k in range(3)])
    assert rel(host(psim), ref) < 1e-12
    psi = fvx.mode_to_layer(psim, m2l)
    back = np.einsum("kl,lyx->kyx", m2l, ref)
    assert rel(host(psi), back) < 1e-12
    # scalar lambda, batched leading dims, FP32
    q4 = np.random.default_rng(1).standard_normal((2, 2, 64, 64))
    got = fvx.pv_inversion(dev(q4, torch.float32), 0.1, 0.1, 0.5)
    assert rel(host(got), O.solve_helmholtz_dst(q4, 0.1, 0.1, 0.5)) < 1e-4
    with pytest.raises(ValueError):
        fvx.pv_inversion(dev(q), dx, dx, lam[:2])
