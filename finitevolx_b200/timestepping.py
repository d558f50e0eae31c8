"""Explicit Runge-Kutta steppers over pytrees of CUDA tensors.

Mirrors finitevolX timestepping/explicit_rk.py:22-121.  The stage
combinations run as one ``fvx_lincomb_*`` launch per leaf with the
reference's operation order, e.g. ``0.75*y + 0.25*y1 + (0.25*dt)*k2``.
For the fused QG step (all three stages of one kernel each, no separate
combination pass) see :mod:`finitevolx_b200.qg`.
"""

from __future__ import annotations

import torch

from finitevolx_b200._lib import D, I64, P, check, fn, sfx, stream_ptr


def _map(f, *trees):
    t0 = trees[0]
    if isinstance(t0, torch.Tensor):
        return f(*trees)
    if isinstance(t0, dict):
        return {k: _map(f, *(t[k] for t in trees)) for k in t0}
    if isinstance(t0, (list, tuple)):
        out = [_map(f, *(t[i] for t in trees)) for i in range(len(t0))]
        return type(t0)(out) if isinstance(t0, tuple) and not hasattr(t0, "_fields") else (
            type(t0)(*out) if hasattr(t0, "_fields") else out)
    raise TypeError(f"unsupported pytree node {type(t0)}")


def lincomb(a, x, b=0.0, y=None, c=0.0, z=None) -> torch.Tensor:
    """((a*x + b*y) + c*z) elementwise in x's dtype."""
    out = torch.empty_like(x)
    for t in (y, z):
        if t is not None and (t.shape != x.shape or t.dtype != x.dtype):
            raise ValueError("lincomb operands must share shape and dtype")
    check(fn(f"fvx_lincomb_{sfx(x)}")(I64(x.numel()), D(a), P(x), D(b), P(y), D(c), P(z), P(out),
                                       stream_ptr()), "lincomb")
    return out


def euler_step(state, rhs_fn, dt: float):
    k1 = rhs_fn(state)
    return _map(lambda y, f: lincomb(1.0, y, dt, f), state, k1)


def heun_step(state, rhs_fn, dt: float):
    """explicit_rk.py:43-71."""
    k1 = rhs_fn(state)
    ys = _map(lambda y, f: lincomb(1.0, y, dt, f), state, k1)
    k2 = rhs_fn(ys)
    # y + 0.5*dt*(k1 + k2): sum first, then the axpy
    return _map(lambda y, f1, f2: lincomb(1.0, y, 0.5 * dt, lincomb(1.0, f1, 1.0, f2)), state, k1, k2)


def rk3_ssp_step(state, rhs_fn, dt: float):
    """Shu-Osher SSP-RK3 (explicit_rk.py:74-121)."""
    k1 = rhs_fn(state)
    y1 = _map(lambda y, f: lincomb(1.0, y, dt, f), state, k1)
    k2 = rhs_fn(y1)
    y2 = _map(lambda y, a, f: lincomb(0.75, y, 0.25, a, 0.25 * dt, f), state, y1, k2)
    k3 = rhs_fn(y2)
    return _map(lambda y, a, f: lincomb(1.0 / 3.0, y, 2.0 / 3.0, a, (2.0 / 3.0) * dt, f), state, y2, k3)
