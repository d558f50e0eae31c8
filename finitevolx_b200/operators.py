"""C-grid differences, interpolations and the Arakawa Jacobian.

Mirrors finitevolX operators/difference.py:165-520 (Difference2D),
operators/interpolation.py:104-275 (Interpolation2D) and
operators/jacobian.py:22-131 (arakawa_jacobian).  Each method is one
libfvx.so launch (``fvx_cgrid_op2d_*``, ``fvx_arakawa_jacobian_*``).
"""

from __future__ import annotations

import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import D, I, P, check, fn, sfx, stream_ptr
from finitevolx_b200.grid import ArakawaCGrid2D
from finitevolx_b200.mask import Mask2D

_OPS = {
    "diff_x_T_to_U": (0, "u"), "diff_y_T_to_V": (1, "v"), "diff_y_U_to_X": (2, "xy_corner_strict"),
    "diff_x_V_to_X": (3, "xy_corner_strict"), "diff_y_X_to_U": (4, "u"), "diff_x_X_to_V": (5, "v"),
    "diff_x_U_to_T": (6, "h"), "diff_y_V_to_T": (7, "h"), "laplacian": (8, "h"),
    "divergence": (9, "h"), "curl": (10, "xy_corner_strict"), "grad_perp": (11, "u"),
    "T_to_U": (16, "u"), "T_to_V": (17, "v"), "T_to_X": (18, "xy_corner_strict"), "X_to_U": (19, "u"),
    "X_to_V": (20, "v"), "U_to_T": (21, "h"), "V_to_T": (22, "h"), "X_to_T": (23, "h"),
    "U_to_X": (24, "xy_corner_strict"), "V_to_X": (25, "xy_corner_strict"), "U_to_V": (26, "v"),
    "V_to_U": (27, "u"),
}


def cgrid_op(name, a, b=None, dx=1.0, dy=1.0, mask: Mask2D | None = None, out=None):
    code, mk = _OPS[name]
    a = L.as_field(a)
    if a.ndim != 2:
        raise ValueError(f"{name}: expected a [Ny, Nx] field, got shape {tuple(a.shape)}")
    if b is not None:
        b = L.as_field(b, dtype=a.dtype)
        if b.shape != a.shape:
            raise ValueError(f"{name}: shape mismatch {tuple(a.shape)} vs {tuple(b.shape)}")
    ny, nx = a.shape
    out = torch.empty_like(a) if out is None else out
    out2 = torch.empty_like(a) if name == "grad_perp" else None
    m1 = None if mask is None else getattr(mask, mk)
    m2 = None if (mask is None or name != "grad_perp") else mask.v
    check(fn(f"fvx_cgrid_op2d_{sfx(a)}")(I(code), P(a), P(b), P(out), P(out2), I(ny), I(nx), D(dx), D(dy),
                                          P(m1), P(m2), stream_ptr()), name)
    return (out, out2) if name == "grad_perp" else out


class Difference2D:
    """Finite differences on the 2-D C-grid (operators/difference.py:165-520)."""

    def __init__(self, grid: ArakawaCGrid2D, mask: Mask2D | None = None):
        self.grid = grid
        self.mask = mask

    def _op(self, name, a, b=None):
        return cgrid_op(name, a, b, self.grid.dx, self.grid.dy, self.mask)

    def diff_x_T_to_U(self, h): return self._op("diff_x_T_to_U", h)
    def diff_y_T_to_V(self, h): return self._op("diff_y_T_to_V", h)
    def diff_y_U_to_X(self, u): return self._op("diff_y_U_to_X", u)
    def diff_x_V_to_X(self, v): return self._op("diff_x_V_to_X", v)
    def diff_y_X_to_U(self, q): return self._op("diff_y_X_to_U", q)
    def diff_x_X_to_V(self, q): return self._op("diff_x_X_to_V", q)
    def diff_x_U_to_T(self, u): return self._op("diff_x_U_to_T", u)
    def diff_y_V_to_T(self, v): return self._op("diff_y_V_to_T", v)
    def divergence(self, u, v): return self._op("divergence", u, v)
    def curl(self, u, v): return self._op("curl", u, v)
    def laplacian(self, h): return self._op("laplacian", h)
    def grad_perp(self, psi): return self._op("grad_perp", psi)


class Interpolation2D:
    """2- and 4-point averages on the 2-D C-grid (operators/interpolation.py:104-275)."""

    def __init__(self, grid: ArakawaCGrid2D, mask: Mask2D | None = None):
        self.grid = grid
        self.mask = mask

    def _op(self, name, a):
        return cgrid_op(name, a, None, 1.0, 1.0, self.mask)


for _n in ("T_to_U", "T_to_V", "T_to_X", "X_to_U", "X_to_V", "U_to_T", "V_to_T", "X_to_T", "U_to_X",
           "V_to_X", "U_to_V", "V_to_U"):
    setattr(Interpolation2D, _n, (lambda nn: lambda self, a: self._op(nn, a))(_n))


def divergence_2d(u, v, dx: float, dy: float):
    """operators/divergence.py:17-60 (unmasked functional form)."""
    return cgrid_op("divergence", u, v, dx, dy)


def arakawa_jacobian(f, g, dx: float, dy: float) -> torch.Tensor:
    """Arakawa (1966) J(f, g) on [..., Ny, Nx] -> [..., Ny-2, Nx-2] (jacobian.py:22-131)."""
    f = L.as_field(f)
    g = L.as_field(g, dtype=f.dtype)
    if f.shape != g.shape:
        raise ValueError(f"arakawa_jacobian: shape mismatch {tuple(f.shape)} vs {tuple(g.shape)}")
    if f.ndim < 2:
        raise ValueError("arakawa_jacobian: inputs need at least 2 dims")
    ny, nx = f.shape[-2:]
    lead = f.shape[:-2]
    batch = 1
    for s in lead:
        batch *= s
    out = torch.empty(lead + (ny - 2, nx - 2), dtype=f.dtype, device=f.device)
    check(fn(f"fvx_arakawa_jacobian_{sfx(f)}")(P(f), P(g), P(out), I(batch), I(ny), I(nx), D(dx), D(dy),
                                                stream_ptr()), "arakawa_jacobian")
    return out
