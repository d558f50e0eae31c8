"""Advection2D, Reconstruction2D, upwind_flux and face-flux helpers.

Mirrors finitevolX advection/advection.py:283-420 (Advection2D),
advection/reconstruction.py:572-1306 (Reconstruction2D),
advection/flux.py:100-253 (upwind_flux) and advection/face_flux.py:36-186.
The tendency runs as one fused tile kernel per call (face fluxes and their
divergence never leave shared memory); masked, mask-dispatchable methods
select each face's tier from packed per-cell tier codes inside that kernel.
"""

from __future__ import annotations

import ctypes

import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import D, I, P, SCHEMES, check, fn, sfx, stream_ptr
from finitevolx_b200.grid import ArakawaCGrid2D
from finitevolx_b200.mask import Mask2D

TVD_LIMITERS = frozenset({"minmod", "van_leer", "superbee", "mc"})
MASK_DISPATCHABLE = frozenset({"weno3", "weno5", "wenoz5"}) | TVD_LIMITERS
ADVECTION_METHODS = ("naive", "upwind1", "upwind2", "upwind3", "weno3", "weno5", "wenoz5", "weno7",
                     "weno9", "minmod", "van_leer", "superbee", "mc")
_MIN_LEN = {"weno9": 8, "weno7": 6, "weno5": 4, "wenoz5": 4}


def _check_fields(*ts):
    shape, dtype = ts[0].shape, ts[0].dtype
    for t in ts:
        if t.shape != shape:
            raise ValueError(f"shape mismatch: {tuple(t.shape)} vs {tuple(shape)}")
        if t.dtype != dtype:
            raise ValueError(f"dtype mismatch: {t.dtype} vs {dtype}")
    if len(shape) != 2:
        raise ValueError(f"expected [Ny, Nx] fields, got shape {tuple(shape)}")


def advect(h, u, v, dx: float, dy: float, method: str = "upwind1", mask: Mask2D | None = None,
           out: torch.Tensor | None = None) -> torch.Tensor:
    """-div(h u) at T-points, output written only to [2:-2, 2:-2]."""
    if method not in SCHEMES or method == "wenoz3":
        raise ValueError(f"Unknown method: {method!r}")
    h, u, v = (L.as_field(x) for x in (h, u, v))
    _check_fields(h, u, v)
    ny, nx = h.shape
    need = _MIN_LEN.get(method, 3)
    if ny < need or nx < need:
        raise ValueError(f"method {method!r} needs at least {need} cells per axis, got {(ny, nx)}")
    if out is None:
        out = torch.empty_like(h)
    tiers = mh = None
    if mask is not None:
        mh = mask.h
        if tuple(mh.shape) != (ny, nx):
            raise ValueError("mask shape does not match the fields")
        if method in MASK_DISPATCHABLE:
            tiers = mask.tier_codes()
    check(fn(f"fvx_advect2d_{sfx(h)}")(P(h), P(u), P(v), P(out), I(ny), I(nx), D(dx), D(dy),
                                        I(SCHEMES[method]), P(tiers), P(mh), stream_ptr()),
          f"Advection2D({method})")
    return out


class Advection2D:
    """2-D advection operator (advection/advection.py:283-420)."""

    def __init__(self, grid: ArakawaCGrid2D, mask: Mask2D | None = None):
        self.grid = grid
        self.mask = mask
        self.recon = Reconstruction2D(grid)
        if mask is not None:
            mask.tier_codes()  # pre-built once, like the reference's hierarchy

    def __call__(self, h, u, v, method: str = "upwind1") -> torch.Tensor:
        return advect(h, u, v, self.grid.dx, self.grid.dy, method, self.mask)


def _face_flux(h, u, v, method, tiers=None, want=("x", "y")):
    h, u, v = (L.as_field(x) for x in (h, u, v))
    _check_fields(h, u, v)
    ny, nx = h.shape
    need = _MIN_LEN.get(method, 3)
    if ny < need or nx < need:
        raise ValueError(f"method {method!r} needs at least {need} cells per axis, got {(ny, nx)}")
    fe = torch.empty_like(h) if "x" in want else None
    fnn = torch.empty_like(h) if "y" in want else None
    check(fn(f"fvx_face_flux2d_{sfx(h)}")(P(h), P(u), P(v), P(fe), P(fnn), I(ny), I(nx), I(SCHEMES[method]),
                                           P(tiers), stream_ptr()), f"face flux ({method})")
    return fe, fnn


class Reconstruction2D:
    """Face fluxes h_face * velocity with zero ghost ring (reconstruction.py:572-1306)."""

    def __init__(self, grid: ArakawaCGrid2D):
        self.grid = grid

    def _x(self, h, u, m):
        hh = L.as_field(h)
        return _face_flux(hh, u, hh, m, want=("x",))[0]

    def _y(self, h, v, m):
        hh = L.as_field(h)
        return _face_flux(hh, hh, v, m, want=("y",))[1]

    def _xm(self, h, u, mask, m):
        hh = L.as_field(h)
        return _face_flux(hh, u, hh, m, tiers=mask.tier_codes(), want=("x",))[0]

    def _ym(self, h, v, mask, m):
        hh = L.as_field(h)
        return _face_flux(hh, hh, v, m, tiers=mask.tier_codes(), want=("y",))[1]


def _add_methods():
    for m in ("naive", "upwind1", "upwind2", "upwind3", "weno3", "wenoz3", "weno5", "wenoz5", "weno7",
              "weno9"):
        setattr(Reconstruction2D, f"{m}_x", (lambda mm: lambda self, h, u: self._x(h, u, mm))(m))
        setattr(Reconstruction2D, f"{m}_y", (lambda mm: lambda self, h, v: self._y(h, v, mm))(m))
    for m in ("weno3", "weno5", "wenoz5"):
        setattr(Reconstruction2D, f"{m}_x_masked",
                (lambda mm: lambda self, h, u, mask: self._xm(h, u, mask, mm))(m))
        setattr(Reconstruction2D, f"{m}_y_masked",
                (lambda mm: lambda self, h, v, mask: self._ym(h, v, mask, mm))(m))


_add_methods()


def _tvd_check(limiter):
    if limiter not in TVD_LIMITERS:
        raise ValueError(f"Unknown flux limiter {limiter!r}. Choose one of "
                         f"{['minmod', 'van_leer', 'superbee', 'mc']!r}.")


def _tvd_x(self, h, u, limiter="minmod"):
    _tvd_check(limiter)
    return self._x(h, u, limiter)


def _tvd_y(self, h, v, limiter="minmod"):
    _tvd_check(limiter)
    return self._y(h, v, limiter)


def _tvd_x_masked(self, h, u, mask, limiter="minmod"):
    _tvd_check(limiter)
    return self._xm(h, u, mask, limiter)


def _tvd_y_masked(self, h, v, mask, limiter="minmod"):
    _tvd_check(limiter)
    return self._ym(h, v, mask, limiter)


Reconstruction2D.tvd_x = _tvd_x
Reconstruction2D.tvd_y = _tvd_y
Reconstruction2D.tvd_x_masked = _tvd_x_masked
Reconstruction2D.tvd_y_masked = _tvd_y_masked


def upwind_flux(q, u, dim: int, rec_funcs: dict, mask_hierarchy: dict) -> torch.Tensor:
    """Blend tier fluxes by the upwind cell's tier (advection/flux.py:100-253)."""
    if not rec_funcs:
        raise ValueError("rec_funcs must not be empty")
    q = L.as_field(q)
    u = L.as_field(u)
    if not 0 <= dim < q.ndim:
        raise ValueError(f"dim={dim!r} is out of range for {q.ndim}-D input")
    if q.ndim != 2:
        raise ValueError("upwind_flux: 2-D fields only")
    if not mask_hierarchy:
        raise ValueError("mask_hierarchy must not be empty")
    sizes = sorted(rec_funcs)
    missing = set(sizes) - set(mask_hierarchy)
    if missing:
        raise ValueError("mask_hierarchy is missing masks for stencil sizes "
                         f"{sorted(missing)}; got keys {sorted(mask_hierarchy.keys())}")
    fluxes = [L.as_field(rec_funcs[s](q, u)).to(q.dtype) for s in sizes]
    masks = [L.as_mask(mask_hierarchy[s]) for s in sizes]
    ny, nx = q.shape
    out = torch.empty_like(q)
    n = len(sizes)
    fp = (ctypes.c_void_p * n)(*[t.data_ptr() for t in fluxes])
    mp = (ctypes.c_void_p * n)(*[t.data_ptr() for t in masks])
    check(fn(f"fvx_upwind_blend_{sfx(q)}")(fp, mp, I(n), P(u), P(out), I(ny), I(nx), I(dim), stream_ptr()),
          "upwind_flux")
    return out


def uv_center_flux(h, u, v, grid: ArakawaCGrid2D, method: str = "upwind1", mask: Mask2D | None = None):
    """(fe, fn) face fluxes of a T-point scalar (advection/face_flux.py:36-87, :130-186)."""
    if method not in ADVECTION_METHODS:
        raise ValueError(f"Unknown method: {method!r}")
    tiers = mask.tier_codes() if (mask is not None and method in MASK_DISPATCHABLE) else None
    return _face_flux(h, u, v, method, tiers=tiers)


def uv_node_flux(q, u, v, grid: ArakawaCGrid2D, method: str = "upwind1", mask: Mask2D | None = None):
    """Same reconstruction for a node-centred tracer (advection/face_flux.py:88-128)."""
    return uv_center_flux(q, u, v, grid, method, mask)
