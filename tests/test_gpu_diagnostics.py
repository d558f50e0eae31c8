"""GPU diagnostics against the FP64 oracle (operators/diagnostics.py):
FP64 1e-12 max-norm relative, FP32 1e-5; domain integrals 1e-12 / 1e-6.
The reference ships no golden arrays for these functions: parity rests on the
restated formulas (the oracle), with the ghost-ring conventions checked
explicitly."""

import numpy as np
import pytest
import torch

import finitevolx_b200.diagnostics as G
import oracle.fvx_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    return np.nanmax(np.abs(a - b)) / max(np.nanmax(np.abs(b)), 1e-300)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-5)])
def test_diagnostics_match_oracle(cuda_ok, dtype, tol):
    rng = np.random.default_rng(0)
    ny, nx = 70, 90
    u, v, h, H, f, w = (rng.standard_normal((ny, nx)) for _ in range(6))
    h = np.abs(h) + 0.5
    h[3, 4] = 0.0  # potential_vorticity's NaN branch
    dx, dy = 0.3, 0.2
    d = lambda a: torch.as_tensor(a, dtype=dtype, device="cuda")  # noqa: E731
    hst = lambda t: t.double().cpu().numpy()  # noqa: E731
    cases = [
        (G.kinetic_energy(d(u), d(v)), O.kinetic_energy(u, v)),
        (G.bernoulli_potential(d(h), d(u), d(v), 9.81), O.bernoulli_potential(h, u, v, 9.81)),
        (G.shear_strain(d(u), d(v), dx, dy), O.shear_strain(u, v, dx, dy)),
        (G.tensor_strain(d(u), d(v), dx, dy), O.tensor_strain(u, v, dx, dy)),
        (G.qg_potential_vorticity(d(w), 1e-4, 2e-11, dx, dy, d(H), 0.1),
         O.qg_potential_vorticity(w, 1e-4, 2e-11, dx, dy, H, 0.1)),
        (G.enstrophy(d(w)), O.enstrophy(w)),
        (G.potential_enstrophy(d(w), d(h)), O.potential_enstrophy(w, h)),
        (G.strain_magnitude_squared(d(u), d(v)), O.strain_magnitude_squared(u, v)),
        (G.okubo_weiss(d(u), d(v), d(w)), O.okubo_weiss(u, v, w)),
        (G.available_potential_energy(d(h), d(H), 0.02), O.available_potential_energy(h, H, 0.02)),
    ]
    for k, (got, ref) in enumerate(cases):
        assert rel(hst(got), ref) < tol, k
    pv = hst(G.potential_vorticity(d(w), d(f), d(h)))
    ref = O.potential_vorticity(w, f, h)
    assert np.isnan(pv[3, 4]) and np.isnan(ref[3, 4])
    assert rel(pv, ref) < tol
    ke, ape = O.kinetic_energy(u, v), O.available_potential_energy(h, H, 0.02)
    te = float(G.total_energy(d(ke), d(ape), dx, dy).item())
    assert abs(te - O.total_energy(ke, ape, dx, dy)) <= (1e-12 if dtype == torch.float64 else 1e-6) * abs(te)
    ens = O.enstrophy(w)
    tz = float(G.total_enstrophy(d(ens), dx, dy).item())
    assert abs(tz - O.total_enstrophy(ens, dx, dy)) <= (1e-12 if dtype == torch.float64 else 1e-6) * abs(tz)
    # relative vorticity is the C-grid curl with a zero ring
    rv = hst(G.relative_vorticity_cgrid(d(u), d(v), dx, dy))
    assert np.all(rv[0] == 0) and np.all(rv[:, -1] == 0)
