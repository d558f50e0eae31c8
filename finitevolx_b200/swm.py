"""Shallow-water operators: Coriolis2D (operators/coriolis.py:34-133),
Vorticity2D (operators/vorticity.py:14-235) and MomentumAdvection2D
(diffusion/momentum.py:35-216).

Each method is one fused libfvx.so launch (``fvx_sw2d_*``) that recomputes
the staggered intermediates the reference materialises (interpolations,
curl, kinetic energy and its gradient), with the same arithmetic, zero ghost
rings and pass-down mask rules, so nothing but the outputs is written.
"""

from __future__ import annotations

import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import D, I, P, check, fn, sfx, stream_ptr
from finitevolx_b200.grid import ArakawaCGrid2D
from finitevolx_b200.mask import Mask2D
from finitevolx_b200.operators import cgrid_op

_CORIOLIS, _PV_E, _PV_Z, _PV_AL, _MOM_E, _MOM_Z, _MOM_AL, _PV = range(8)


def _sw(op, a, b, c=None, d=None, dx=1.0, dy=1.0, alpha=1.0 / 3.0, mask: Mask2D | None = None, two=True):
    a = L.as_field(a)
    fields = [a] + [None if t is None else L.as_field(t, dtype=a.dtype) for t in (b, c, d)]
    for t in fields[1:]:
        if t is not None and t.shape != a.shape:
            raise ValueError(f"shape mismatch {tuple(a.shape)} vs {tuple(t.shape)}")
    ny, nx = a.shape
    o1 = torch.empty_like(a)
    o2 = torch.empty_like(a) if two else None
    m = (None,) * 4 if mask is None else (mask.h, mask.u, mask.v, mask.xy_corner_strict)
    check(fn(f"fvx_sw2d_{sfx(a)}")(I(op), *[P(t) for t in fields], P(o1), P(o2), I(ny), I(nx), D(dx), D(dy),
                                   D(alpha), *[P(t) for t in m], stream_ptr()), "shallow-water operator")
    return (o1, o2) if two else o1


class Coriolis2D:
    """du = +f_on_u v_on_u, dv = -f_on_v u_on_v (coriolis.py:34-133)."""

    def __init__(self, grid: ArakawaCGrid2D, mask: Mask2D | None = None):
        self.grid, self.mask = grid, mask

    def __call__(self, u, v, f):
        return _sw(_CORIOLIS, u, v, f, mask=self.mask)


class Vorticity2D:
    """Relative / potential vorticity and PV fluxes (vorticity.py:14-235)."""

    def __init__(self, grid: ArakawaCGrid2D, mask: Mask2D | None = None):
        self.grid, self.mask = grid, mask

    def relative_vorticity(self, u, v):
        return cgrid_op("curl", u, v, self.grid.dx, self.grid.dy, self.mask)

    def potential_vorticity(self, u, v, h, f):
        return _sw(_PV, u, v, h, f, self.grid.dx, self.grid.dy, mask=self.mask, two=False)

    def pv_flux_energy_conserving(self, q, u, v):
        return _sw(_PV_E, q, u, v, mask=self.mask)

    def pv_flux_enstrophy_conserving(self, q, u, v):
        return _sw(_PV_Z, q, u, v, mask=self.mask)

    def pv_flux_arakawa_lamb(self, q, u, v, alpha: float = 1.0 / 3.0):
        return _sw(_PV_AL, q, u, v, alpha=alpha, mask=self.mask)


class MomentumAdvection2D:
    """Vector-invariant momentum advection, energy / enstrophy / Arakawa-Lamb
    vorticity fluxes (momentum.py:35-216); writes [2:-2, 2:-2]."""

    def __init__(self, grid: ArakawaCGrid2D, mask: Mask2D | None = None):
        self.grid, self.mask = grid, mask

    def __call__(self, u, v, scheme: str = "energy"):
        ops = {"energy": _MOM_E, "enstrophy": _MOM_Z, "al": _MOM_AL}
        if scheme not in ops:
            raise ValueError(f"Unknown scheme: {scheme!r}.  Choose 'energy', 'enstrophy', or 'al'.")
        return _sw(ops[scheme], u, v, dx=self.grid.dx, dy=self.grid.dy, mask=self.mask)
