"""Rectangular spectral Helmholtz solves by transform-matrix products on
the tensor cores.

``solve_helmholtz_dst(rhs, dx, dy, lambda_)`` is the drop-in for
spectraldiffx's ``solve_helmholtz_dst`` that finitevolX re-exports
(solvers/spectral.py:14-98): it solves (nabla^2 - lambda) psi = rhs on the
interior-only array ``rhs`` [..., Ny, Nx] with psi = 0 outside.
``solve_helmholtz_dct`` (Neumann, DCT-II) and ``solve_helmholtz_fft``
(periodic) are the other two solvers that finitevolX's ``_spectral_solve``
dispatches on (spectral.py:105-128); they take the whole [..., Ny, Nx]
array and return the zero-mean solution when the problem has a null mode
(lambda = 0).  The periodic solve uses the real Hartley transform pair, the
same linear map as the FFT solve on real data.

* float32 input: 3xBF16-split tcgen05 GEMM chain, FP32 accumulation
  (relative error ~1e-5 of the FP64 answer);
* float64 input: the FP64 SIMT chain (``method="fp64"``, default) or the
  split chain with FP64 iterative refinement (``method="refine"``) to a
  normwise backward error ``tol``.
``lambda_`` may be a scalar or one value per layer (shape [nl], matching
``rhs.shape[-3]``, as ``pv_inversion`` uses it).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import D, I, P, check, fn, stream_ptr

I64 = ctypes.c_longlong


KINDS = {"dst": 0, "dct": 1, "fft": 2}


class DSTHelmholtzPlan:
    """Pre-built transform matrices, eigenvalue grids and workspaces for one
    size and boundary condition (``bc``: "dst" Dirichlet, "dct" Neumann,
    "fft" periodic).

    Creating a plan allocates device memory once; ``solve`` allocates
    nothing on the device besides its output (pass ``out=`` to avoid that).
    """

    def __init__(self, ny: int, nx: int, dx: float, dy: float, lambdas=(0.0,), batch_max: int = 1,
                 fp64: bool = True, bc: str = "dst"):
        L.require_cuda()
        if bc not in KINDS:
            raise ValueError(f"bc must be 'fft', 'dst', or 'dct'; got {bc!r}")
        lam = np.atleast_1d(np.asarray(lambdas, dtype=np.float64))
        self.ny, self.nx, self.dx, self.dy = int(ny), int(nx), float(dx), float(dy)
        self.bc = bc
        self.lambdas = lam
        self.batch_max = int(batch_max)
        self._h = ctypes.c_void_p()
        lam_c = (ctypes.c_double * len(lam))(*lam.tolist())
        check(fn("fvx_spectral_plan_create")(I(KINDS[bc]), I(self.ny), I(self.nx), D(self.dx), D(self.dy),
                                             I(self.batch_max), lam_c, I(len(lam)), I(int(fp64)),
                                             ctypes.byref(self._h)),
              "SpectralHelmholtzPlan")
        self.split_ok = (self.nx % 8 == 0) and (self.ny % 8 == 0)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                fn("fvx_dst_plan_destroy")(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    def _views(self, rhs):
        if rhs.shape[-2:] != (self.ny, self.nx):
            raise ValueError(f"rhs interior shape {tuple(rhs.shape[-2:])} != plan {(self.ny, self.nx)}")
        b = int(np.prod(rhs.shape[:-2])) if rhs.ndim > 2 else 1
        if b > self.batch_max:
            raise ValueError(f"batch {b} exceeds the plan's batch_max {self.batch_max}")
        return b

    def solve(self, rhs, out=None, method: str = "fp64") -> torch.Tensor:
        rhs = L.as_field(rhs)
        b = self._views(rhs)
        out = torch.empty_like(rhs) if out is None else out
        plane = self.ny * self.nx
        if rhs.dtype == torch.float32:
            check(fn("fvx_dst_solve_f32")(self._h, P(rhs), I64(plane), I64(self.nx), P(out), I64(plane),
                                          I64(self.nx), I(b), stream_ptr()), "solve_helmholtz_dst")
        elif rhs.dtype == torch.float64:
            m = {"fp64": 0, "refine": 1}[method]
            info = (ctypes.c_double * 3)()
            check(fn("fvx_dst_solve_f64")(self._h, P(rhs), I64(plane), I64(self.nx), P(out), I64(plane),
                                          I64(self.nx), I(b), I(m), D(1e-12), I(8), info, stream_ptr()),
                  "solve_helmholtz_dst")
        else:
            raise TypeError(f"unsupported dtype {rhs.dtype}")
        return out

    def solve_refined(self, rhs, tol: float = 1e-12, max_iter: int = 8, out=None):
        """Split-BF16 solve + FP64 iterative refinement (Dirichlet plans).

        Returns (psi, info) with info = {passes, backward_error, rel_residual};
        backward_error = ||r|| / (||A|| ||psi|| + ||rhs||).
        """
        if self.bc != "dst":
            raise ValueError("iterative refinement is provided for the Dirichlet (DST) plan only")
        rhs = L.as_field(rhs, dtype=torch.float64)
        b = self._views(rhs)
        out = torch.empty_like(rhs) if out is None else out
        plane = self.ny * self.nx
        info = (ctypes.c_double * 3)()
        st = fn("fvx_dst_solve_f64")(self._h, P(rhs), I64(plane), I64(self.nx), P(out), I64(plane), I64(self.nx),
                                     I(b), I(1), D(tol), I(max_iter), info, stream_ptr())
        res = dict(passes=int(info[0]), backward_error=float(info[1]), rel_residual=float(info[2]),
                   converged=st == 0)
        if st not in (0, 5):
            check(st, "solve_helmholtz_dst (refined)")
        return out, res

    def check_device(self):
        """Raises if a bounded device wait of the plan's products gave up
        since the last check (the flag is cleared once reported)."""
        check(fn("fvx_dst_plan_check")(self._h, stream_ptr()), "DST kernels")

    def set_wait_limit(self, cycles: int) -> None:
        """Bound, in SM clock cycles, on each barrier wait of the products."""
        check(fn("fvx_dst_plan_set_wait_limit")(self._h, ctypes.c_longlong(int(cycles))), "wait limit")


_CACHE: dict = {}


SpectralHelmholtzPlan = DSTHelmholtzPlan


def get_plan(ny, nx, dx, dy, lambdas, batch, fp64=True, bc: str = "dst") -> DSTHelmholtzPlan:
    lam = tuple(np.atleast_1d(np.asarray(lambdas, dtype=np.float64)).tolist())
    key = (bc, ny, nx, float(dx), float(dy), lam, torch.cuda.current_device())
    p = _CACHE.get(key)
    if p is None or p.batch_max < batch:
        p = DSTHelmholtzPlan(ny, nx, dx, dy, lam, batch_max=max(batch, 1), fp64=fp64, bc=bc)
        _CACHE[key] = p
    return p


def _solve(rhs, dx, dy, lambda_, method, bc):
    rhs = L.as_field(rhs)
    if rhs.ndim < 2:
        raise ValueError("rhs must be at least 2-D")
    lam = np.atleast_1d(np.asarray(lambda_.cpu() if isinstance(lambda_, torch.Tensor) else lambda_,
                                   dtype=np.float64))
    if lam.size > 1 and (rhs.ndim < 3 or rhs.shape[-3] != lam.size):
        raise ValueError(f"rhs.shape[-3] must match the {lam.size} lambda values")
    ny, nx = rhs.shape[-2:]
    b = int(np.prod(rhs.shape[:-2])) if rhs.ndim > 2 else 1
    return get_plan(ny, nx, dx, dy, lam, b, bc=bc).solve(rhs, method=method)


def solve_helmholtz_dct(rhs, dx: float, dy: float, lambda_=0.0) -> torch.Tensor:
    """(nabla^2 - lambda) psi = rhs with homogeneous Neumann walls (cell-centred,
    DCT-II); zero-mean psi when lambda = 0."""
    return _solve(rhs, dx, dy, lambda_, "fp64", "dct")


def solve_helmholtz_fft(rhs, dx: float, dy: float, lambda_=0.0) -> torch.Tensor:
    """(nabla^2 - lambda) psi = rhs on a doubly periodic grid; zero-mean psi
    when lambda = 0."""
    return _solve(rhs, dx, dy, lambda_, "fp64", "fft")


def solve_poisson_dct(rhs, dx: float, dy: float) -> torch.Tensor:
    return solve_helmholtz_dct(rhs, dx, dy, 0.0)


def solve_poisson_fft(rhs, dx: float, dy: float) -> torch.Tensor:
    return solve_helmholtz_fft(rhs, dx, dy, 0.0)


def spectral_solve(rhs, dx: float, dy: float, lambda_, bc: str) -> torch.Tensor:
    """The rectangular solver for ``bc`` (spectral.py:105-128 ``_spectral_solve``)."""
    if bc not in KINDS:
        raise ValueError(f"base_bc must be 'fft', 'dst', or 'dct'; got {bc!r}")
    return _solve(rhs, dx, dy, lambda_, "fp64", bc)


def make_spectral_preconditioner(dx: float, dy: float, lambda_: float = 0.0, bc: str = "fft"):
    """M_inv(r) = the rectangular spectral solve of (nabla^2 - lambda)
    (preconditioners.py:44-84); default periodic."""
    if bc not in KINDS:
        raise ValueError(f"bc must be 'fft', 'dst', or 'dct'; got {bc!r}")
    return lambda r: spectral_solve(r, dx, dy, lambda_, bc)


def dct2_eigenvalues(n: int, d: float) -> np.ndarray:
    k = np.arange(n)
    return -4.0 / d ** 2 * np.sin(np.pi * k / (2 * n)) ** 2


def fft_eigenvalues(n: int, d: float) -> np.ndarray:
    k = np.arange(n)
    return -4.0 / d ** 2 * np.sin(np.pi * k / n) ** 2


def solve_helmholtz_dst(rhs, dx: float, dy: float, lambda_=0.0, method: str = "fp64") -> torch.Tensor:
    """(nabla^2 - lambda) psi = rhs with psi = 0 outside the interior array."""
    rhs = L.as_field(rhs)
    if rhs.ndim < 2:
        raise ValueError("rhs must be at least 2-D")
    lam = np.atleast_1d(np.asarray(lambda_.cpu() if isinstance(lambda_, torch.Tensor) else lambda_,
                                   dtype=np.float64))
    if lam.size > 1 and (rhs.ndim < 3 or rhs.shape[-3] != lam.size):
        raise ValueError(f"rhs.shape[-3] must match the {lam.size} lambda values")
    ny, nx = rhs.shape[-2:]
    b = int(np.prod(rhs.shape[:-2])) if rhs.ndim > 2 else 1
    return get_plan(ny, nx, dx, dy, lam, b).solve(rhs, method=method)


def solve_poisson_dst(rhs, dx: float, dy: float) -> torch.Tensor:
    return solve_helmholtz_dst(rhs, dx, dy, 0.0)


def dst1_eigenvalues(n: int, d: float) -> np.ndarray:
    k = np.arange(n)
    return -4.0 / d ** 2 * np.sin(np.pi * (k + 1) / (2 * (n + 1))) ** 2
