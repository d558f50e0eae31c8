"""GPU parity: the Neumann (DCT-II) and periodic rectangular spectral
solvers on the tensor-core / FP64 transform chains, and the capacitance-
matrix masked solver, against the FP64 oracle.

Tolerances: FP64 chains 1e-12 (normwise relative, max norm); FP32 3xBF16
chains 1e-4 of max|psi| (the DST chain's bound); capacitance (FP64): the
solution vanishes on the inner-boundary points to 1e-10 (the reference's
own test tolerance) and matches the oracle to 1e-11.
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


SOLVERS = {"dct": (fvx.solve_helmholtz_dct, O.solve_helmholtz_dct),
           "fft": (fvx.solve_helmholtz_fft, O.solve_helmholtz_fft)}


@pytest.mark.parametrize("bc", ["dct", "fft"])
@pytest.mark.parametrize("shape,lam", [((8, 10), 0.0), ((8, 10), 3.0), ((37, 29), -1.0), ((64, 128), 0.0),
                                       ((256, 192), 2.5)])
def test_spectral_fp64(cuda_ok, bc, shape, lam):
    ny, nx = shape
    dx, dy = 1.0 / (nx - 1), 1.0 / (ny - 1)
    f = np.random.default_rng(ny + nx).standard_normal(shape)
    got = host(SOLVERS[bc][0](dev(f), dx, dy, lam))
    assert rel(got, SOLVERS[bc][1](f, dx, dy, lam)) < 1e-12
    if lam == 0.0:
        assert abs(got.mean()) < 1e-12 * np.abs(got).max()  # zero-mean gauge


@pytest.mark.parametrize("bc", ["dct", "fft"])
@pytest.mark.parametrize("shape,lam", [((64, 128), 0.0), ((256, 256), 4.0), ((512, 256), 0.0)])
def test_spectral_fp32_split_chain(cuda_ok, bc, shape, lam):
    # well-conditioned cases: with lambda ~ 1e-3 the near-null mean mode is
    # amplified ~1e3 times the FP32 rounding of the input's mean, beyond
    # what FP32 data resolves whatever the solver
    ny, nx = shape
    dx, dy = 1.0 / nx, 1.0 / ny
    f = O.kminus3_field(ny, nx, 7)
    f = f - f.mean()
    got = host(SOLVERS[bc][0](dev(f, torch.float32), dx, dy, lam))
    assert rel(got, SOLVERS[bc][1](f, dx, dy, lam)) < 1e-4


def test_spectral_batched_lambdas_and_wrappers(cuda_ok):
    ny, nx, dx = 48, 40, 0.05
    q = np.random.default_rng(3).standard_normal((3, ny, nx))
    lam = np.array([0.0, 1.0, 4.0])
    for bc in ("dct", "fft", "dst"):
        got = host(fvx.pv_inversion(dev(q), dx, dx, lam, bc=bc))
        ref = np.stack([O.spectral_solve(q[k], dx, dx, lam[k], bc) for k in range(3)])
        assert rel(got, ref) < 1e-12
    p = host(fvx.pressure_from_divergence(dev(q[0]), dx, dx))  # Neumann default
    assert rel(p, O.solve_helmholtz_dct(q[0], dx, dx, 0.0)) < 1e-12
    M = fvx.make_spectral_preconditioner(dx, dx, lambda_=1.0)  # periodic default
    assert rel(host(M(dev(q[1]))), O.solve_helmholtz_fft(q[1], dx, dx, 1.0)) < 1e-12
    with pytest.raises(ValueError):
        fvx.make_spectral_preconditioner(dx, dx, bc="neumann")


def _rect_mask(ny, nx):
    m = np.ones((ny, nx), bool)
    m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = False
    return m


@pytest.mark.parametrize("base_bc", ["fft", "dst", "dct"])
def test_capacitance_reference_case(cuda_ok, base_bc):
    # the reference's own case: 10 x 12 rectangle with a land border,
    # lambda = -1, rhs = sin(pi j / Ny) cos(pi i / Nx); psi = 0 on B
    ny, nx = 10, 12
    mask = _rect_mask(ny, nx)
    dx, dy = 1.0 / (nx - 1), 1.0 / (ny - 1)
    j, i = np.arange(ny)[:, None], np.arange(nx)[None, :]
    rhs = np.sin(np.pi * j / ny) * np.cos(np.pi * i / nx)
    solver = fvx.build_capacitance_solver(mask, dx, dy, lambda_=-1.0, base_bc=base_bc)
    psi = host(solver(dev(rhs)))
    jb, ib = O.inner_boundary_indices(mask)
    assert solver.n_boundary == len(jb)
    assert np.abs(psi[jb, ib]).max() < 1e-10
    assert rel(psi, O.capacitance_solve(rhs, mask, dx, dy, -1.0, base_bc)) < 1e-11
    got = host(fvx.streamfunction_from_vorticity(dev(rhs), dx, dy, method="capacitance", lambda_=-1.0,
                                                 capacitance_solver=solver))
    assert rel(got, psi) < 1e-14


def test_capacitance_coastline_fp32_and_batch(cuda_ok):
    # irregular island on a 64 x 64 periodic base; FP32 through the split chain
    n = 64
    mask = np.ones((n, n), bool)
    yy, xx = np.mgrid[:n, :n]
    mask[(yy - 30) ** 2 + (xx - 25) ** 2 < 64] = False
    mask[5:9, 40:60] = False
    dx = 1.0 / n
    rhs = np.random.default_rng(5).standard_normal((2, n, n))
    solver = fvx.build_capacitance_solver(mask, dx, dx, lambda_=50.0)
    jb, ib = O.inner_boundary_indices(mask)
    ref = np.stack([O.capacitance_solve(rhs[k], mask, dx, dx, 50.0) for k in range(2)])
    got64 = host(solver(dev(rhs)))
    assert rel(got64, ref) < 1e-11
    assert np.abs(got64[:, jb, ib]).max() < 1e-10 * np.abs(ref).max()
    got32 = host(solver(dev(rhs, torch.float32)))
    assert rel(got32, ref) < 1e-4


def test_capacitance_errors(cuda_ok):
    with pytest.raises(ValueError, match="No inner-boundary points"):
        fvx.build_capacitance_solver(np.ones((8, 10), bool), 0.1, 0.1)
    with pytest.raises(ValueError):
        fvx.build_capacitance_solver(_rect_mask(8, 10), 0.1, 0.1, base_bc="neumann")
    with pytest.raises(ValueError):
        fvx.streamfunction_from_vorticity(dev(np.zeros((8, 10))), 0.1, 0.1, method="capacitance")
