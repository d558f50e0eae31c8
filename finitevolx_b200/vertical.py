"""Vertical modes for multi-layer QG (finitevolX vertical/vertical_modes.py:50-263).

The coupling matrix and its eigendecomposition are nl x nl set-up
computations (nl <= 8) done on the host in FP64; the layer <-> mode
transforms of fields run on the device (``fvx_layer_mix_*``).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import I, P, check, fn, sfx, stream_ptr


def build_coupling_matrix(H, g_prime) -> np.ndarray:
    """Tridiagonal stratification matrix A (vertical_modes.py:50-121)."""
    H = np.asarray(H, dtype=float)
    g = np.asarray(g_prime, dtype=float)
    nl = H.shape[0]
    A = np.zeros((nl, nl))
    if nl == 1:
        A[0, 0] = 1.0 / (H[0] * g[0])
        return A
    A[0, 0] = 1.0 / (H[0] * g[0]) + 1.0 / (H[0] * g[1])
    A[0, 1] = -1.0 / (H[0] * g[1])
    for i in range(1, nl - 1):
        A[i, i - 1] = -1.0 / (H[i] * g[i])
        A[i, i] = (1.0 / H[i]) * (1.0 / g[i + 1] + 1.0 / g[i])
        A[i, i + 1] = -1.0 / (H[i] * g[i + 1])
    A[-1, -1] = 1.0 / (H[nl - 1] * g[nl - 1])
    A[-1, -2] = -1.0 / (H[nl - 1] * g[nl - 1])
    return A


def decompose_vertical_modes(A, f0: float):
    """Rossby radii and layer<->mode transforms (vertical_modes.py:124-190).

    Like jnp.linalg.eigh's default, the input is symmetrised, (A + A^T)/2.
    """
    A = np.asarray(A, dtype=float)
    lam, R = np.linalg.eigh(0.5 * (A + A.T))
    pos = lam > 0
    safe = np.where(pos, lam, 1.0)
    rr = np.where(pos, 1.0 / (abs(f0) * np.sqrt(safe)), np.inf)
    return rr, R.T.copy(), R.copy()


def _mix(field, C) -> torch.Tensor:
    f = L.as_field(field)
    C = np.ascontiguousarray(np.asarray(C, dtype=np.float64))
    nl = C.shape[0]
    if f.shape[0] != nl and (f.ndim < 3 or f.shape[-3] != nl):
        raise ValueError(f"layer axis of length {nl} expected")
    if f.shape[0] == nl:
        plane = f.numel() // nl
        batch = 1
    else:
        plane = f.shape[-2] * f.shape[-1]
        batch = f.numel() // (nl * plane)
    out = torch.empty_like(f)
    check(fn(f"fvx_layer_mix_{sfx(f)}")(C.ctypes.data_as(ctypes.c_void_p), I(nl), P(f), P(out),
                                         ctypes.c_int64(plane), I(batch), stream_ptr()), "layer_mix")
    return out


def layer_to_mode(field, Cl2m) -> torch.Tensor:
    """mode = Cl2m @ layer along the leading axis (vertical_modes.py:193-227)."""
    return _mix(field, Cl2m)


def mode_to_layer(field, Cm2l) -> torch.Tensor:
    """layer = Cm2l @ mode (vertical_modes.py:230-263)."""
    return _mix(field, Cm2l)
