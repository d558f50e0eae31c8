"""Ghost-ring boundary fills (finitevolX boundary/boundary.py:17-75)."""

from __future__ import annotations

import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import I, P, check, fn, sfx, stream_ptr


def _batched(field):
    f = L.as_field(field)
    if f.ndim < 2:
        raise ValueError("expected [..., Ny, Nx]")
    ny, nx = f.shape[-2:]
    b = f.numel() // (ny * nx)
    return f, b, ny, nx


def enforce_periodic_(field: torch.Tensor) -> torch.Tensor:
    """In-place periodic ghost fill (S, N, W, E order; bc_set.py:54-66)."""
    f, b, ny, nx = _batched(field)
    if f.data_ptr() != field.data_ptr():
        raise ValueError("enforce_periodic_ needs a contiguous CUDA tensor")
    check(fn(f"fvx_fill_periodic_{sfx(f)}")(P(f), I(b), I(ny), I(nx), stream_ptr()), "enforce_periodic")
    return field


def enforce_periodic(field) -> torch.Tensor:
    """Copy of ``field`` with periodic ghost cells (boundary/boundary.py:52-75)."""
    f, b, ny, nx = _batched(field)
    out = f.clone()
    check(fn(f"fvx_fill_periodic_{sfx(out)}")(P(out), I(b), I(ny), I(nx), stream_ptr()), "enforce_periodic")
    return out


def pad_interior(field, mode: str = "constant") -> torch.Tensor:
    """Re-fill the ghost ring (boundary/boundary.py:17-49).

    ``"constant"`` (zero ghost ring, wall BCs) and ``"wrap"`` (periodic) are
    supported.
    """
    f, b, ny, nx = _batched(field)
    out = f.clone()
    if mode == "constant":
        check(fn(f"fvx_zero_ring_{sfx(out)}")(P(out), I(b), I(ny), I(nx), stream_ptr()), "pad_interior")
    elif mode == "wrap":
        check(fn(f"fvx_fill_periodic_{sfx(out)}")(P(out), I(b), I(ny), I(nx), stream_ptr()), "pad_interior")
    else:
        raise ValueError(f"pad_interior: mode {mode!r} not supported (use 'constant' or 'wrap')")
    return out
