"""CPU: the oracle's Neumann / periodic spectral solvers and capacitance
solve, pinned by the discrete operators they invert and by the reference's
capacitance tests (tests/test_elliptic.py:483-545 of finitevolX), and the
Python host logic that needs no GPU (inner-boundary detection, argument
errors)."""

import numpy as np
import pytest

import oracle.fvx_oracle as O
from finitevolx_b200.solvers.capacitance import inner_boundary_mask


@pytest.mark.parametrize("lam", [0.0, 2.0, -1.0])
@pytest.mark.parametrize("shape", [(8, 10), (13, 7)])
def test_dct_and_fft_invert_their_operators(shape, lam):
    f = np.random.default_rng(1).standard_normal(shape)
    dx, dy = 1.0 / (shape[1] - 1), 1.0 / (shape[0] - 1)
    target = f - f.mean() if lam == 0.0 else f
    for solve, apply in ((O.solve_helmholtz_dct, O.neumann_helmholtz_apply),
                         (O.solve_helmholtz_fft, O.periodic_helmholtz_apply)):
        psi = solve(f, dx, dy, lam)
        assert np.abs(apply(psi, dx, dy, lam) - target).max() < 1e-12 * np.abs(f).max() / min(dx, dy) ** 2
        if lam == 0.0:
            assert abs(psi.mean()) < 1e-14


def test_eigenvalue_tables():
    n, d = 12, 0.3
    assert np.allclose(O.dct2_eigenvalues(n, d)[0], 0.0) and np.allclose(O.fft_eigenvalues(n, d)[0], 0.0)
    # periodic eigenvalues are symmetric in k <-> n - k (what lets a real
    # Hartley basis diagonalise the operator)
    e = O.fft_eigenvalues(n, d)
    assert np.allclose(e[1:], e[1:][::-1])


def test_inner_boundary_matches_reference_definition():
    from scipy.ndimage import binary_dilation
    rng = np.random.default_rng(2)
    for _ in range(5):
        m = rng.random((17, 23)) > 0.3
        struct = np.array([[0, 1, 0], [1, 1, 1], [0, 1, 0]], bool)
        ref = m & binary_dilation(~m, structure=struct)
        assert np.array_equal(inner_boundary_mask(m), ref)
        jb, ib = O.inner_boundary_indices(m)
        assert np.array_equal(np.argwhere(ref), np.stack([jb, ib], 1))


@pytest.mark.parametrize("base_bc", ["fft", "dst", "dct"])
def test_oracle_capacitance_reference_case(base_bc):
    ny, nx = 10, 12
    mask = np.ones((ny, nx), bool)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = False
    dx, dy = 1.0 / (nx - 1), 1.0 / (ny - 1)
    j, i = np.arange(ny)[:, None], np.arange(nx)[None, :]
    rhs = np.sin(np.pi * j / ny) * np.cos(np.pi * i / nx)
    psi = O.capacitance_solve(rhs, mask, dx, dy, -1.0, base_bc)
    jb, ib = O.inner_boundary_indices(mask)
    np.testing.assert_allclose(psi[jb, ib], 0.0, atol=1e-10)
    with pytest.raises(ValueError, match="No inner-boundary points"):
        O.capacitance_solve(rhs, np.ones((ny, nx), bool), dx, dy)
