"""Capacitance-matrix solver for masked Helmholtz problems on a rectangular
spectral solver (finitevolX solvers/elliptic.py:146-183,
``build_capacitance_solver`` / ``CapacitanceSolver``).

Inner-boundary points B are the mask's True cells 4-connected to a False
cell.  Building the solver runs N_b rectangular solves of unit vectors
(batched on the tensor-core / FP64 chains), gathers C[k, l] = g_l(b_k) and
inverts C once in FP64 on the host (the reference's offline step).  A
solve is then two rectangular solves and one kernel between them:

    u = L^-1 f,   rhs2 = f - E_B (C^-1 u[B]),   psi = L^-1 rhs2,

so psi vanishes on B without storing the N_b x (Ny Nx) Green's-function
matrix that psi = u - G alpha would need.
"""

from __future__ import annotations

import numpy as np
import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import I, P, check, fn, stream_ptr
from finitevolx_b200.mask import Mask2D
from finitevolx_b200.solvers.spectral import KINDS, get_plan

I64 = __import__("ctypes").c_longlong


def inner_boundary_mask(mask) -> np.ndarray:
    """True cells 4-connected to a False cell (cells beyond the array edge do
    not count as land)."""
    m = np.asarray(mask, dtype=bool)
    land = ~m
    d = land.copy()
    d[1:, :] |= land[:-1, :]
    d[:-1, :] |= land[1:, :]
    d[:, 1:] |= land[:, :-1]
    d[:, :-1] |= land[:, 1:]
    return m & d


class CapacitanceSolver:
    """Callable masked solver: ``psi = solver(rhs)`` for rhs [..., Ny, Nx]
    (float32: the 3xBF16 tensor-core chain; float64: the FP64 chain)."""

    def __init__(self, mask, dx: float, dy: float, lambda_: float = 0.0, base_bc: str = "fft",
                 chunk: int = 64):
        L.require_cuda()
        if base_bc not in KINDS:
            raise ValueError(f"base_bc must be 'fft', 'dst', or 'dct'; got {base_bc!r}")
        if isinstance(mask, Mask2D):
            mask = mask.xy_corner_strict
        if isinstance(mask, torch.Tensor):
            mask = mask.detach().cpu().numpy()
        m = np.asarray(mask, dtype=bool)
        if m.ndim != 2:
            raise ValueError(f"mask must be 2-D, got shape {m.shape}")
        jb, ib = np.where(inner_boundary_mask(m))
        if len(jb) == 0:
            raise ValueError("No inner-boundary points found in mask")
        self.shape = m.shape
        self.dx, self.dy, self.lambda_, self.base_bc = float(dx), float(dy), float(lambda_), base_bc
        ny, nx = m.shape
        flat = (jb.astype(np.int64) * nx + ib.astype(np.int64))
        self.n_boundary = nb = len(flat)
        self.j_b, self.i_b = jb, ib
        self.idx = torch.as_tensor(flat, device="cuda")
        # C[k, l] = g_l(b_k), g_l = L^-1 e_{b_l}, in FP64
        chunk = max(1, min(int(chunk), nb))
        plan = get_plan(ny, nx, dx, dy, (lambda_,), chunk, bc=base_bc)
        C = torch.empty((nb, nb), dtype=torch.float64, device="cuda")
        e = torch.zeros((chunk, ny * nx), dtype=torch.float64, device="cuda")
        for l0 in range(0, nb, chunk):
            c = min(chunk, nb - l0)
            e.zero_()
            e[torch.arange(c, device="cuda"), self.idx[l0:l0 + c]] = 1.0
            g = plan.solve(e[:c].reshape(c, ny, nx))
            C[:, l0:l0 + c] = g.reshape(c, ny * nx)[:, self.idx].T
        cinv = np.linalg.inv(C.cpu().numpy())
        self.cinv = torch.as_tensor(cinv, device="cuda")

    def __call__(self, rhs) -> torch.Tensor:
        rhs = L.as_field(rhs)
        if tuple(rhs.shape[-2:]) != self.shape:
            raise ValueError(f"rhs shape {tuple(rhs.shape[-2:])} != mask shape {self.shape}")
        if rhs.dtype not in (torch.float32, torch.float64):
            raise TypeError(f"unsupported dtype {rhs.dtype}")
        ny, nx = self.shape
        b = int(np.prod(rhs.shape[:-2])) if rhs.ndim > 2 else 1
        plan = get_plan(ny, nx, self.dx, self.dy, (self.lambda_,), b, bc=self.base_bc)
        u = plan.solve(rhs)
        rhs2 = torch.empty_like(rhs)
        sfx = "f32" if rhs.dtype == torch.float32 else "f64"
        f3, u3, r3 = (t.reshape(b, ny * nx) for t in (rhs, u, rhs2))
        for k in range(b):
            check(fn(f"fvx_capacitance_rhs_{sfx}")(P(f3[k]), P(u3[k]), P(self.cinv), P(self.idx),
                                                   I(self.n_boundary), I64(ny * nx), P(r3[k]), stream_ptr()),
                  "capacitance rhs")
        return plan.solve(rhs2)


def build_capacitance_solver(mask, dx: float, dy: float, lambda_: float = 0.0,
                             base_bc: str = "fft") -> CapacitanceSolver:
    """Pre-compute the capacitance matrix (elliptic.py:146-183)."""
    return CapacitanceSolver(mask, dx, dy, lambda_, base_bc)
