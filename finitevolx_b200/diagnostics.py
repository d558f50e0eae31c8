"""Diagnostics on the Arakawa C-grid (finitevolX operators/diagnostics.py).

Pointwise and 5-point quantities run in one library kernel selected by an
operator code; the domain integrals (``total_energy``, ``total_enstrophy``)
sum the interior in FP64 on the device with a deterministic reduction and
return a 0-d device tensor.  Ghost-ring conventions follow the reference:
quantities it returns through ``interior(...)`` have a zero ring, pointwise
ones are evaluated everywhere.
"""

from __future__ import annotations

import ctypes

import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import D, I, P, check, fn, sfx, stream_ptr

_OPS = {"kinetic_energy": 0, "bernoulli_potential": 1, "shear_strain": 2, "tensor_strain": 3,
        "qg_potential_vorticity": 4, "potential_vorticity": 5, "enstrophy": 6, "potential_enstrophy": 7,
        "strain_magnitude_squared": 8, "okubo_weiss": 9, "available_potential_energy": 10}


def _diag(name, a, b=None, c=None, p=(0.0, 0.0, 0.0, 0.0, 0.0)):
    a = L.as_field(a)
    b = None if b is None else L.as_field(b, dtype=a.dtype)
    c = None if c is None else L.as_field(c, dtype=a.dtype)
    for t in (b, c):
        if t is not None and t.shape != a.shape:
            raise ValueError(f"{name}: all fields must have shape {tuple(a.shape)}")
    ny, nx = a.shape
    out = torch.empty_like(a)
    check(fn(f"fvx_diag2d_{sfx(a)}")(I(_OPS[name]), P(a), P(b), P(c), P(out), I(ny), I(nx), *[D(x) for x in p],
                                     stream_ptr()), name)
    return out


def kinetic_energy(u, v):
    """0.5 (avg_x_bwd(u^2) + avg_y_bwd(v^2)) at T-points (diagnostics.py:35-73)."""
    return _diag("kinetic_energy", u, v)


def bernoulli_potential(h, u, v, gravity: float = 9.81):
    """ke + g h at T-points (diagnostics.py:76-112)."""
    return _diag("bernoulli_potential", h, u, v, (gravity, 0, 0, 0, 0))


def relative_vorticity_cgrid(u, v, dx: float, dy: float):
    """Curl at X-points (diagnostics.py:115-147, difference.py:47-59)."""
    from finitevolx_b200.operators import cgrid_op
    return cgrid_op("curl", L.as_field(u), L.as_field(v), dx=dx, dy=dy)


def shear_strain(u, v, dx: float, dy: float):
    """dv/dx + du/dy at X-points (diagnostics.py:184-213)."""
    return _diag("shear_strain", u, v, None, (dx, dy, 0, 0, 0))


def tensor_strain(u, v, dx: float, dy: float):
    """du/dx - dv/dy at T-points (diagnostics.py:216-245)."""
    return _diag("tensor_strain", u, v, None, (dx, dy, 0, 0, 0))


def strain_magnitude_squared(sn, ss):
    return _diag("strain_magnitude_squared", sn, ss)


def okubo_weiss(sn, ss, omega):
    """Sn^2 + Ss^2 - omega^2 (diagnostics.py:274-305)."""
    return _diag("okubo_weiss", sn, ss, omega)


def potential_vorticity(omega, f, h):
    """(omega + f) / h, NaN where h == 0 (diagnostics.py:150-181)."""
    return _diag("potential_vorticity", omega, f, h)


def enstrophy(omega):
    """0.5 omega^2 (diagnostics.py:308-329)."""
    return _diag("enstrophy", omega)


def potential_enstrophy(q, h):
    """0.5 q^2 h (diagnostics.py:332-360)."""
    return _diag("potential_enstrophy", q, h)


def available_potential_energy(h, H, g_prime: float):
    """0.5 g' (h - H)^2 (diagnostics.py:363-392)."""
    return _diag("available_potential_energy", h, H, None, (g_prime, 0, 0, 0, 0))


def qg_potential_vorticity(psi, f0: float, beta: float, dx: float, dy: float, y, y0: float):
    """lap(psi) / f0 + beta (y - y0) / f0 at T-points (diagnostics.py:395-452)."""
    return _diag("qg_potential_vorticity", psi, y, None, (f0, beta, dx, dy, y0))


_SUM_WORK = {}


def _interior_sum(a, b, scale):
    a = L.as_field(a)
    b = None if b is None else L.as_field(b, dtype=a.dtype)
    dev = a.device
    if dev not in _SUM_WORK:
        _SUM_WORK[dev] = (torch.empty(296, dtype=torch.float64, device=dev),
                          torch.zeros(1, dtype=torch.int32, device=dev))
    part, ticket = _SUM_WORK[dev]
    out = torch.empty((), dtype=torch.float64, device=dev)
    ny, nx = a.shape
    check(fn(f"fvx_interior_sum_{sfx(a)}")(P(a), P(b), I(ny), I(nx), D(scale), P(part), P(ticket), P(out),
                                           stream_ptr()), "interior sum")
    return out


def total_energy(ke, ape, dx: float, dy: float):
    """sum_interior(KE + APE) dx dy, FP64 device scalar (diagnostics.py:498-524)."""
    return _interior_sum(ke, ape, dx * dy)


def total_enstrophy(ens, dx: float, dy: float):
    """sum_interior(ens) dx dy, FP64 device scalar (diagnostics.py:527-555)."""
    return _interior_sum(ens, None, dx * dy)
