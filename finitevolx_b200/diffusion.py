"""Harmonic and biharmonic diffusion (finitevolX diffusion/diffusion.py:70-574).

``Diffusion2D`` applies the three-step intermediate-flux masking pattern of
the reference inside one kernel; ``BiharmonicDiffusion2D`` runs both
Laplacian passes in one kernel with the intermediate field held in shared
memory (the reference materialises it in HBM).
"""

from __future__ import annotations

import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import D, I, P, check, fn, sfx, stream_ptr
from finitevolx_b200.grid import ArakawaCGrid2D
from finitevolx_b200.mask import Mask2D


def _diffuse(h, kappa, dx, dy, mu=None, mv=None, mh=None, want_out=True, want_fluxes=False):
    h = L.as_field(h)
    if h.ndim != 2:
        raise ValueError(f"expected a [Ny, Nx] field, got shape {tuple(h.shape)}")
    ny, nx = h.shape
    kf = None
    kap = 0.0
    if isinstance(kappa, (int, float)):
        kap = float(kappa)
    else:
        kt = L.as_field(kappa, dtype=h.dtype)
        if kt.ndim == 0:
            kap = float(kt.item())
        elif kt.shape == h.shape:
            kf = kt
        else:
            raise ValueError(f"kappa must be a scalar or a {tuple(h.shape)} field")
    out = torch.empty_like(h) if want_out else None
    fx = torch.empty_like(h) if want_fluxes else None
    fy = torch.empty_like(h) if want_fluxes else None
    check(fn(f"fvx_diffusion2d_{sfx(h)}")(P(h), P(kf), D(kap), P(out), P(fx), P(fy), I(ny), I(nx), D(dx),
                                           D(dy), P(mu), P(mv), P(mh), stream_ptr()), "Diffusion2D")
    return out, fx, fy


def diffusion_2d(h, kappa, dx: float, dy: float) -> torch.Tensor:
    """Mask-free functional form (diffusion/diffusion.py:70-117)."""
    return _diffuse(h, kappa, dx, dy)[0]


class Diffusion2D:
    """Flux-form harmonic diffusion (diffusion/diffusion.py:208-330)."""

    def __init__(self, grid: ArakawaCGrid2D, mask: Mask2D | None = None):
        self.grid = grid
        self.mask = mask

    def _m(self):
        m = self.mask
        return (None, None, None) if m is None else (m.u, m.v, m.h)

    def __call__(self, h, kappa) -> torch.Tensor:
        mu, mv, mh = self._m()
        return _diffuse(h, kappa, self.grid.dx, self.grid.dy, mu, mv, mh)[0]

    def fluxes(self, h, kappa):
        mu, mv, _ = self._m()
        _, fx, fy = _diffuse(h, kappa, self.grid.dx, self.grid.dy, mu, mv, None, want_out=False,
                             want_fluxes=True)
        return fx, fy


class BiharmonicDiffusion2D:
    """-kappa * L(L(h)), inner Laplacian unmasked (diffusion/diffusion.py:462-574)."""

    def __init__(self, grid: ArakawaCGrid2D, mask: Mask2D | None = None):
        self.grid = grid
        self.mask = mask

    def __call__(self, h, kappa: float) -> torch.Tensor:
        h = L.as_field(h)
        if h.ndim != 2:
            raise ValueError(f"expected a [Ny, Nx] field, got shape {tuple(h.shape)}")
        ny, nx = h.shape
        out = torch.empty_like(h)
        mh = None if self.mask is None else self.mask.h
        check(fn(f"fvx_biharmonic2d_{sfx(h)}")(P(h), D(float(kappa)), P(out), I(ny), I(nx), D(self.grid.dx),
                                                D(self.grid.dy), P(mh), stream_ptr()), "BiharmonicDiffusion2D")
        return out
