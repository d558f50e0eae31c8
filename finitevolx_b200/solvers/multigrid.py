"""Geometric multigrid for (div(c grad) - lambda) on masked domains.

Mirrors finitevolX solvers/multigrid.py (build_multigrid_solver :905-1062,
MultigridSolver :601-897) and make_multigrid_preconditioner
(solvers/preconditioners.py:207-244).  The level hierarchy is built once in
FP64 inside libfvx.so (the reference builds it offline in NumPy); V-cycles
run on the device: one launch per leg (all of its sweeps plus the transfer)
on the fine levels, one single-CTA launch for every level at or below 32 x 32.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import D, I, P, check, fn, stream_ptr
from finitevolx_b200.mask import Mask2D


class MultigridSolver:
    """V-cycle solver; ``dtype`` float32 or float64 for the level arrays."""

    def __init__(self, mask, dx, dy, lambda_=0.0, coeff=None, n_levels=None, n_pre=6, n_post=6, n_coarse=50,
                 omega=0.95, n_cycles=5, dtype=torch.float64):
        L.require_cuda()
        if isinstance(mask, Mask2D):
            m = mask.xy_corner_strict.double().cpu().numpy()
        elif isinstance(mask, torch.Tensor):
            m = mask.double().cpu().numpy()
        else:
            m = np.asarray(mask, dtype=np.float64)
        m = np.ascontiguousarray(m, dtype=np.float64)
        ny, nx = m.shape
        c = None
        if coeff is not None:
            c = np.ascontiguousarray(coeff.double().cpu().numpy() if isinstance(coeff, torch.Tensor)
                                     else np.asarray(coeff, dtype=np.float64))
        nl = 0 if n_levels is None else int(n_levels)
        if nl > 0:
            fac = 2 ** (nl - 1)
            if ny % fac or nx % fac:
                raise ValueError(f"Grid shape ({ny}, {nx}) is not divisible by 2^(n_levels-1) = {fac}.  "
                                 "Choose a different n_levels or pad the grid.")
        self.shape = (ny, nx)
        self.dtype = dtype
        self.n_cycles = int(n_cycles)
        self.lambda_ = float(lambda_)
        self.dx, self.dy = float(dx), float(dy)
        self._h = ctypes.c_void_p()
        dt = 0 if dtype == torch.float32 else 1
        check(fn("fvx_mg_create")(m.ctypes.data_as(ctypes.c_void_p),
                                  None if c is None else c.ctypes.data_as(ctypes.c_void_p), I(ny), I(nx), D(dx),
                                  D(dy), D(lambda_), I(nl), I(n_pre), I(n_post), I(n_coarse), D(omega), I(dt),
                                  ctypes.byref(self._h)), "build_multigrid_solver")
        self.n_levels = fn("fvx_mg_num_levels")(self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                fn("fvx_mg_destroy")(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    def _field(self, x):
        t = L.as_field(x, dtype=self.dtype)
        if tuple(t.shape) != self.shape:
            raise ValueError(f"expected shape {self.shape}, got {tuple(t.shape)}")
        return t

    def level(self, k: int) -> dict:
        """mask, cx, cy, inv_diagonal of level k as device tensors (views)."""
        ny, nx, dx2 = I(), I(), D()
        ptrs = [ctypes.c_void_p() for _ in range(4)]
        check(fn("fvx_mg_level")(self._h, I(k), ctypes.byref(ny), ctypes.byref(nx), ctypes.byref(dx2),
                                 *[ctypes.byref(p) for p in ptrs]), "level")
        es = 4 if self.dtype == torch.float32 else 8
        out = {}
        for name, p in zip(("mask", "cx", "cy", "inv_diagonal"), ptrs):
            buf = torch.empty((ny.value, nx.value), dtype=self.dtype, device="cuda")
            check(fn("fvx_lincomb_" + ("f32" if es == 4 else "f64"))(
                ctypes.c_int64(ny.value * nx.value), D(1.0), p, D(0.0), None, D(0.0), None, P(buf), stream_ptr()),
                "copy level")
            out[name] = buf
        return out

    def apply(self, u, level: int = 0):
        """_apply_operator: A u at a level."""
        u = L.as_field(u, dtype=self.dtype)
        out = torch.empty_like(u)
        check(fn("fvx_mg_apply")(self._h, I(level), P(u), P(out), stream_ptr()), "apply_operator")
        return out

    def v_cycle(self, u, rhs):
        """One V-cycle from initial guess u (None = zeros)."""
        f = self._field(rhs)
        out = torch.empty_like(f)
        uu = None if u is None else self._field(u)
        check(fn("fvx_mg_vcycle")(self._h, P(uu), P(f), P(out), stream_ptr()), "v_cycle")
        return out

    def __call__(self, rhs):
        """n_cycles V-cycles from zero (MultigridSolver.__call__ forward pass)."""
        f = self._field(rhs)
        out = torch.empty_like(f)
        check(fn("fvx_mg_solve")(self._h, P(f), P(out), I(self.n_cycles), stream_ptr()), "multigrid solve")
        return out

    solve_unrolled = __call__
    solve_onestep = __call__


def build_multigrid_solver(mask, dx, dy, lambda_=0.0, coeff=None, n_levels=None, n_pre=6, n_post=6, n_coarse=50,
                           omega=0.95, n_cycles=5, dtype=torch.float64) -> MultigridSolver:
    """build_multigrid_solver (multigrid.py:905-1062)."""
    return MultigridSolver(mask, dx, dy, lambda_, coeff, n_levels, n_pre, n_post, n_coarse, omega, n_cycles, dtype)


def make_multigrid_preconditioner(mg: MultigridSolver):
    """One V-cycle from zero (preconditioners.py:207-244)."""
    def _pc(r):
        return mg.v_cycle(None, r)
    _pc.mg = mg
    return _pc
