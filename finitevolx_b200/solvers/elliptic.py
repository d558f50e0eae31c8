"""Elliptic inversion wrappers (finitevolX solvers/elliptic.py:255-542).

``method="spectral"`` with ``bc="dst"`` runs the tensor-core DST solver with
one lambda per layer in a single batched call (the reference vmaps one
solve per layer).  ``method="cg"`` runs solve_cg on masked_laplacian with a
caller-supplied preconditioner.  The FFT / DCT spectral solvers and the
capacitance method are outside this package's scope.
"""

from __future__ import annotations

import numpy as np
import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200.mask import Mask2D
from finitevolx_b200.solvers.iterative import masked_laplacian, solve_cg
from finitevolx_b200.solvers.spectral import solve_helmholtz_dst


def _solve_one(rhs, dx, dy, lam, bc, method, mask, preconditioner):
    if method == "spectral":
        if bc != "dst":
            raise ValueError(f"bc must be 'fft', 'dst', or 'dct'; got {bc!r}" if bc not in ("fft", "dct")
                             else f"bc={bc!r} is not provided by finitevolx_b200 (only 'dst')")
        return solve_helmholtz_dst(rhs, dx, dy, lam)
    if method == "cg":
        if mask is None:
            raise ValueError("method='cg' requires a mask (array or Mask2D)")
        m = mask.xy_corner_strict.to(rhs.dtype) if isinstance(mask, Mask2D) else L.as_field(mask, dtype=rhs.dtype)
        if preconditioner is None:
            raise ValueError("method='cg' needs a preconditioner here (the FFT default is not provided)")
        x, _ = solve_cg(lambda z: masked_laplacian(z, m, dx, dy, lam), rhs * m, preconditioner=preconditioner)
        return x * m
    if method == "capacitance":
        raise ValueError("method='capacitance' is not provided by finitevolx_b200")
    raise ValueError(f"method must be 'spectral', 'cg', or 'capacitance'; got {method!r}")


def streamfunction_from_vorticity(zeta, dx, dy, bc="dst", lambda_=0.0, method="spectral", mask=None,
                                  capacitance_solver=None, preconditioner=None):
    """(nabla^2 - lambda) psi = zeta (elliptic.py:255-340)."""
    return _solve_one(L.as_field(zeta), dx, dy, float(lambda_), bc, method, mask, preconditioner)


def pv_inversion(pv, dx, dy, lambda_, bc="dst", method="spectral", mask=None, capacitance_solver=None,
                 preconditioner=None):
    """(nabla^2 - lambda) psi = q, batched / per-layer lambda (elliptic.py:390-542)."""
    pv = L.as_field(pv)
    lam = np.asarray(lambda_.cpu() if isinstance(lambda_, torch.Tensor) else lambda_, dtype=np.float64)
    if lam.ndim == 0:
        if method == "spectral":
            return _solve_one(pv, dx, dy, float(lam), bc, method, mask, preconditioner)
        flat = pv.reshape(-1, *pv.shape[-2:])
        out = torch.stack([_solve_one(f, dx, dy, float(lam), bc, method, mask, preconditioner) for f in flat])
        return out.reshape(pv.shape)
    if pv.ndim < 3:
        raise ValueError(f"pv must have at least 3 dims when lambda_ is an array, got shape {tuple(pv.shape)}")
    nl = lam.shape[0]
    if pv.shape[-3] != nl:
        raise ValueError(f"pv.shape[-3]={pv.shape[-3]} does not match lambda_ length {nl}")
    if method == "capacitance":
        raise ValueError("method='capacitance' does not support array-valued lambda_; solve each layer "
                         "separately or use method='spectral' or 'cg' for multi-layer problems.")
    if method == "spectral":
        if bc != "dst":
            raise ValueError(f"bc={bc!r} is not provided by finitevolx_b200 (only 'dst')")
        return solve_helmholtz_dst(pv, dx, dy, lam)
    flat = pv.reshape(-1, nl, *pv.shape[-2:])
    out = torch.stack([torch.stack([_solve_one(f[k], dx, dy, float(lam[k]), bc, method, mask, preconditioner)
                                    for k in range(nl)]) for f in flat])
    return out.reshape(pv.shape)
