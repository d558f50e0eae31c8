"""GPU shallow-water operators (fused kernels) against the oracle's
composition of Interpolation2D / Difference2D: FP64 1e-13 (same arithmetic,
same order), FP32 1e-5; masked (the canonical cross-island mask) and
unmasked; ghost rings and dry faces exactly zero."""

import numpy as np
import pytest
import torch

import finitevolx_b200 as fvx
import oracle.fvx_oracle as O
from fixture_inputs import DX, DY, NX, NY, fields_2d, h_mask_2d

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    if np.isnan(b).any():
        assert np.array_equal(np.isnan(a), np.isnan(b))
        a, b = np.nan_to_num(a), np.nan_to_num(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("masked", (False, True))
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 1e-5)])
def test_sw_operators_match_oracle(cuda_ok, masked, dtype, tol):
    F = fields_2d()
    grid = fvx.ArakawaCGrid2D.from_interior(NX - 2, NY - 2, 1.0, 1.0)
    hm = h_mask_2d()
    mask = fvx.Mask2D.from_mask(hm) if masked else None
    om = {k: np.asarray(v, np.float64) for k, v in O.mask2d_from_mask(hm).items()} if masked else None
    d = lambda a: torch.as_tensor(a, dtype=dtype, device="cuda")  # noqa: E731
    h = lambda t: t.double().cpu().numpy()  # noqa: E731
    thick = 1.0 + 0.2 * F["h"]
    cor = fvx.Coriolis2D(grid, mask)(d(F["u"]), d(F["v"]), d(F["f"]))
    for g, r in zip(cor, O.coriolis2d(F["u"], F["v"], F["f"], om)):
        assert rel(h(g), r) < tol
    vort = fvx.Vorticity2D(grid, mask)
    pv = vort.potential_vorticity(d(F["u"]), d(F["v"]), d(thick), d(F["f"]))
    assert rel(h(pv), O.potential_vorticity_x(F["u"], F["v"], thick, F["f"], grid.dx, grid.dy, om)) < tol
    for scheme, meth in (("energy", vort.pv_flux_energy_conserving), ("enstrophy", vort.pv_flux_enstrophy_conserving)):
        for g, r in zip(meth(d(F["q"]), d(F["u"]), d(F["v"])), O.pv_flux(F["q"], F["u"], F["v"], scheme, mask=om)):
            assert rel(h(g), r) < tol, scheme
    for g, r in zip(vort.pv_flux_arakawa_lamb(d(F["q"]), d(F["u"]), d(F["v"]), alpha=0.3),
                    O.pv_flux(F["q"], F["u"], F["v"], "al", alpha=0.3, mask=om)):
        assert rel(h(g), r) < tol
    madv = fvx.MomentumAdvection2D(grid, mask)
    for scheme in ("energy", "enstrophy", "al"):
        got = madv(d(F["u"]), d(F["v"]), scheme)
        ref = O.momentum_advection(F["u"], F["v"], grid.dx, grid.dy, scheme, om)
        for g, r in zip(got, ref):
            assert rel(h(g), r) < tol, scheme
            assert not h(g)[:2].any() and not h(g)[-2:].any()  # writes [2:-2, 2:-2] only
    with pytest.raises(ValueError):
        madv(d(F["u"]), d(F["v"]), "bogus")


def test_sw_large_random_fp64(cuda_ok):
    rng = np.random.default_rng(3)
    ny, nx = 130, 97
    u, v, f, q = (rng.standard_normal((ny, nx)) for _ in range(4))
    grid = fvx.ArakawaCGrid2D.from_interior(nx - 2, ny - 2, 2.0, 3.0)
    d = lambda a: torch.as_tensor(a, device="cuda")  # noqa: E731
    got = fvx.MomentumAdvection2D(grid)(d(u), d(v), "al")
    ref = O.momentum_advection(u, v, grid.dx, grid.dy, "al")
    for g, r in zip(got, ref):
        assert rel(g.cpu().numpy(), r) < 1e-13
    got = fvx.Coriolis2D(grid)(d(u), d(v), d(f))
    for g, r in zip(got, O.coriolis2d(u, v, f)):
        assert rel(g.cpu().numpy(), r) < 1e-13


GOLD = __import__("pathlib").Path(__file__).parent / "golden" / "ref"


def _golden(op, method, variant):
    with np.load(GOLD / f"{op}__{method}__{variant}.npz") as z:
        return [np.asarray(z[k]) for k in sorted(z.files)]


@pytest.mark.parametrize("variant", ("unmasked", "masked"))
def test_sw_operators_match_reference_goldens(cuda_ok, variant):
    # finitevolX's own FP64 golden outputs (tests/fixtures/_gen_golden.py:477-547,
    # 852-864, 968-987) at its tolerance, rtol 1e-12 / atol 1e-14
    F = fields_2d()
    grid = fvx.ArakawaCGrid2D.from_interior(NX - 2, NY - 2, 1.0, 1.0)
    mask = fvx.Mask2D.from_mask(h_mask_2d()) if variant == "masked" else None
    d = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")  # noqa: E731

    def same(got, ref):
        got = [g.cpu().numpy() for g in (got if isinstance(got, tuple) else (got,))]
        assert len(got) == len(ref)
        for g, r in zip(got, ref):
            np.testing.assert_allclose(g, r, rtol=1e-12, atol=1e-14)

    same(fvx.Coriolis2D(grid, mask)(d(F["u"]), d(F["v"]), d(F["f"])), _golden("Coriolis2D", "__call__", variant))
    vort = fvx.Vorticity2D(grid, mask)
    same(vort.relative_vorticity(d(F["u"]), d(F["v"])), _golden("Vorticity2D", "relative_vorticity", variant))
    same(vort.potential_vorticity(d(F["u"]), d(F["v"]), d(F["h"]), d(F["f"])),
         _golden("Vorticity2D", "potential_vorticity", variant))
    q, u, v = d(F["q"]), d(F["u"]), d(F["v"])
    same(vort.pv_flux_energy_conserving(q, u, v), _golden("Vorticity2D", "pv_flux_energy_conserving", variant))
    same(vort.pv_flux_enstrophy_conserving(q, u, v), _golden("Vorticity2D", "pv_flux_enstrophy_conserving", variant))
    same(vort.pv_flux_arakawa_lamb(q, u, v), _golden("Vorticity2D", "pv_flux_arakawa_lamb", variant))
    same(fvx.MomentumAdvection2D(grid, mask)(u, v), _golden("MomentumAdvection2D", "__call__", variant))
