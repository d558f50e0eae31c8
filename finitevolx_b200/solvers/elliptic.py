"""Elliptic inversion wrappers (finitevolX solvers/elliptic.py:195-542).

``method="spectral"`` runs the tensor-core rectangular solver for ``bc``
("dst" Dirichlet, "dct" Neumann, "fft" periodic) with one lambda per layer
in a single batched call (the reference vmaps one solve per layer).
``method="cg"`` runs solve_cg on masked_laplacian, preconditioned by default
with the periodic spectral solve as the reference does.
``method="capacitance"`` calls a pre-built CapacitanceSolver.
"""

from __future__ import annotations

import numpy as np
import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200.mask import Mask2D
from finitevolx_b200.solvers.iterative import masked_laplacian, solve_cg
from finitevolx_b200.solvers.spectral import make_spectral_preconditioner, spectral_solve


def _solve_one(rhs, dx, dy, lam, bc, method, mask, preconditioner, capacitance_solver=None):
    if method == "spectral":
        return spectral_solve(rhs, dx, dy, lam, bc)
    if method == "cg":
        if mask is None:
            raise ValueError("method='cg' requires a mask (array or Mask2D)")
        m = mask.xy_corner_strict.to(rhs.dtype) if isinstance(mask, Mask2D) else L.as_field(mask, dtype=rhs.dtype)
        if preconditioner is None:
            preconditioner = make_spectral_preconditioner(dx, dy, lambda_=lam, bc="fft")
        x, _ = solve_cg(lambda z: masked_laplacian(z, m, dx, dy, lam), rhs * m, preconditioner=preconditioner)
        return x * m
    if method == "capacitance":
        if capacitance_solver is None:
            raise ValueError("method='capacitance' requires a pre-built CapacitanceSolver "
                             "(see build_capacitance_solver)")
        return capacitance_solver(rhs)
    raise ValueError(f"method must be 'spectral', 'cg', or 'capacitance'; got {method!r}")


def streamfunction_from_vorticity(zeta, dx, dy, bc="dst", lambda_=0.0, method="spectral", mask=None,
                                  capacitance_solver=None, preconditioner=None):
    """(nabla^2 - lambda) psi = zeta (elliptic.py:276-340)."""
    return _solve_one(L.as_field(zeta), dx, dy, float(lambda_), bc, method, mask, preconditioner,
                      capacitance_solver)


def pressure_from_divergence(div_u, dx, dy, bc="dct", method="spectral", mask=None, capacitance_solver=None,
                             preconditioner=None):
    """nabla^2 p = div u, Neumann by default (elliptic.py:342-388)."""
    return _solve_one(L.as_field(div_u), dx, dy, 0.0, bc, method, mask, preconditioner, capacitance_solver)


def pv_inversion(pv, dx, dy, lambda_, bc="dst", method="spectral", mask=None, capacitance_solver=None,
                 preconditioner=None):
    """(nabla^2 - lambda) psi = q, batched / per-layer lambda (elliptic.py:390-542)."""
    pv = L.as_field(pv)
    lam = np.asarray(lambda_.cpu() if isinstance(lambda_, torch.Tensor) else lambda_, dtype=np.float64)
    if lam.ndim == 0:
        if method in ("spectral", "capacitance"):
            return _solve_one(pv, dx, dy, float(lam), bc, method, mask, preconditioner, capacitance_solver)
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
        return spectral_solve(pv, dx, dy, lam, bc)
    flat = pv.reshape(-1, nl, *pv.shape[-2:])
    out = torch.stack([torch.stack([_solve_one(f[k], dx, dy, float(lam[k]), bc, method, mask, preconditioner)
                                    for k in range(nl)]) for f in flat])
    return out.reshape(pv.shape)
