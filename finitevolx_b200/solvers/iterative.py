"""CG solvers and the masked Laplacian (finitevolX solvers/iterative.py).

* ``solve_cg(matvec, rhs, ...)`` -- the generic API: any callables for the
  operator and preconditioner (each a device computation); vector updates
  and FP64-accumulated inner products run in libfvx.so.  Stopping rule as
  solve_cg delegates to lineax.CG: max|r| < atol + rtol * max|b|, residual
  recomputed every 10 steps.
* ``MaskedHelmholtzPCG`` -- the device-resident PCG for the multigrid
  operator (variable coefficient, masked): no host round trip per
  iteration, FP64 iterate and inner products, FP32 or FP64 work vectors,
  2-norm relative residual checked in FP64.
"""

from __future__ import annotations

import ctypes
from typing import NamedTuple

import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import D, I, P, check, fn, sfx, stream_ptr
from finitevolx_b200.mask import Mask2D
from finitevolx_b200.timestepping import lincomb


class CGInfo(NamedTuple):
    """iterative.py:32-41."""
    iterations: int
    residual_norm: float
    converged: bool


_PART = {}


def _dot(a, b) -> torch.Tensor:
    """FP64-accumulated inner product as a device scalar."""
    dev = a.device
    if dev not in _PART:
        _PART[dev] = torch.empty(296, dtype=torch.float64, device=dev)
    out = torch.empty((), dtype=torch.float64, device=dev)
    check(fn(f"fvx_dot_{sfx(a)}")(P(a), P(b), ctypes.c_int64(a.numel()), P(_PART[dev]), P(out), stream_ptr()),
          "dot")
    return out


def _maxabs(a) -> float:
    return float(a.abs().max().item())


def solve_cg(matvec, rhs, x0=None, preconditioner=None, rtol: float = 1e-6, atol: float = 1e-6,
             max_steps: int | None = 500):
    """PCG for a negative (semi)definite operator (iterative.py:48-136)."""
    b = L.as_field(rhs)
    x = torch.zeros_like(b) if x0 is None else L.as_field(x0, dtype=b.dtype).clone()
    M = (lambda r: r) if preconditioner is None else preconditioner  # noqa: E731
    r = lincomb(1.0, b, -1.0, matvec(x)) if x0 is not None else b.clone()
    z = M(r)
    p = z.clone()
    gamma = float(_dot(r, z).item())
    tol = atol + rtol * _maxabs(b)
    k = 0
    conv = _maxabs(r) < tol
    steps = max_steps if max_steps is not None else 1 << 30
    while not conv and k < steps and gamma != 0.0:
        Ap = matvec(p)
        pAp = float(_dot(p, Ap).item())
        alpha = gamma / pAp
        x = lincomb(1.0, x, alpha, p)
        k += 1
        if k % 10 == 0:
            r = lincomb(1.0, b, -1.0, matvec(x))
        else:
            r = lincomb(1.0, r, -alpha, Ap)
        conv = _maxabs(r) < tol
        if conv:
            break
        z = M(r)
        g_new = float(_dot(r, z).item())
        p = lincomb(1.0, z, g_new / gamma, p)
        gamma = g_new
    res = lincomb(1.0, matvec(x), -1.0, b)
    return x, CGInfo(iterations=k, residual_norm=float(torch.linalg.vector_norm(res.double()).item()),
                     converged=bool(conv))


def masked_laplacian(psi, mask, dx: float, dy: float, lambda_: float = 0.0) -> torch.Tensor:
    """(nabla^2 - lambda)(psi * m) * m with periodic roll (iterative.py:144-191)."""
    psi = L.as_field(psi)
    if isinstance(mask, Mask2D):
        m = mask.xy_corner_strict.to(psi.dtype)
    else:
        m = L.as_field(mask, dtype=psi.dtype)
    ny, nx = psi.shape
    out = torch.empty_like(psi)
    check(fn(f"fvx_masked_laplacian_{sfx(psi)}")(P(psi), P(m), P(out), I(ny), I(nx), D(dx), D(dy), D(lambda_),
                                                  stream_ptr()), "masked_laplacian")
    return out


PRECOND_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)


class MaskedHelmholtzPCG:
    """Device-resident PCG on a MultigridSolver's finest operator.

    ``solve(b, rtol, precond="mg"|"none"|callable, flexible=False)`` returns
    (x FP64, info).  A callable preconditioner gets the residual tensor and
    returns z = M r (any device computation); ``flexible`` selects the
    Polak-Ribiere beta for preconditioners that are not a fixed linear map.
    """

    def __init__(self, mg):
        self.mg = mg
        self._h = ctypes.c_void_p()
        check(fn("fvx_pcg_create")(mg.handle, ctypes.byref(self._h)), "pcg_create")
        self.rho = torch.empty(mg.shape, dtype=mg.dtype, device="cuda")
        self.z = torch.empty_like(self.rho)
        check(fn("fvx_pcg_bind_vectors")(self._h, P(self.rho), P(self.z)), "pcg_bind_vectors")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                fn("fvx_pcg_destroy")(h)
            except Exception:
                pass
            self._h = None

    def solve(self, b, rtol: float = 1e-8, max_iter: int = 500, precond="mg", flexible: bool = False,
              replace_every: int = 10, chunk: int = 4, x=None):
        b = L.as_field(b, dtype=self.mg.dtype)
        if tuple(b.shape) != self.mg.shape:
            raise ValueError("rhs shape does not match the multigrid operator")
        x = torch.empty(b.shape, dtype=torch.float64, device=b.device) if x is None else x
        info = (ctypes.c_double * 3)()
        cb = None
        if isinstance(precond, str):
            if precond not in ("none", "mg"):
                raise ValueError(f"unknown preconditioner {precond!r}")
            kind = {"none": 0, "mg": 1}[precond]
        else:
            kind = 2
            user = precond

            def _cb(ctx, rho, z, stream):
                try:
                    self.z.copy_(user(self.rho))
                    return 0
                except Exception:
                    return 6
            cb = PRECOND_FN(_cb)
        st = fn("fvx_pcg_solve")(self._h, P(b), P(x), I(max_iter), D(rtol), I(kind), cb, None, I(int(flexible)),
                                 I(replace_every), I(chunk), info, stream_ptr())
        if st not in (0, 5):
            check(st, "pcg_solve")
        return x, dict(iterations=int(info[0]), rel_residual=float(info[1]), converged=st == 0)
