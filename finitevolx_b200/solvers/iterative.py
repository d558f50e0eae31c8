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


def _next_chunk(rr_prev, rr, done, tol2, chunk_max):
    """Iterations the last chunk's residual reduction predicts are still
    needed (1 .. chunk_max), so few iterations run after convergence."""
    import math
    if not (rr > 0.0 and rr_prev > 0.0) or rr >= rr_prev or done < 1:
        return chunk_max
    per_it = math.log(rr / rr_prev) / done
    need = math.log(tol2 / rr) / per_it
    return max(1, min(chunk_max, 1 if need <= 1.0 else math.ceil(need)))


PRECOND_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)


class MaskedHelmholtzPCG:
    """Device-resident PCG on a MultigridSolver's finest operator.

    ``solve(b, rtol, precond=..., flexible=False, graph=False)`` returns
    (x FP64, info).  ``precond`` is "mg" (one V-cycle, the reference's
    make_multigrid_preconditioner), "none", a Python callable (gets the
    residual tensor, returns z = M r), or an object with a ``c_precond()``
    method returning (C function address, context) of an fvx_precond_fn --
    e.g. the learned preconditioner in finitevolx_b200.learned.
    ``flexible`` selects the Polak-Ribiere beta for preconditioners that are
    not a fixed linear map.  ``graph=True`` captures one PCG iteration
    (preconditioner included) in a CUDA graph and replays it, reading the
    device convergence flag every ``chunk`` iterations; it needs a C-level
    preconditioner ("mg", "none" or ``c_precond``).
    """

    def __init__(self, mg):
        self.mg = mg
        self._h = ctypes.c_void_p()
        check(fn("fvx_pcg_create")(mg.handle, ctypes.byref(self._h)), "pcg_create")
        self.rho = torch.empty(mg.shape, dtype=mg.dtype, device="cuda")
        self.z = torch.empty_like(self.rho)
        check(fn("fvx_pcg_bind_vectors")(self._h, P(self.rho), P(self.z)), "pcg_bind_vectors")
        self._graphs = {}
        self._gb = None
        self._gx = None

    def __del__(self):
        self._graphs = {}
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                fn("fvx_pcg_destroy")(h)
            except Exception:
                pass
            self._h = None

    def _precond_args(self, precond):
        """(kind, C function pointer, context, keep-alive) for the C entry points."""
        if isinstance(precond, str):
            if precond not in ("none", "mg"):
                raise ValueError(f"unknown preconditioner {precond!r}")
            return {"none": 0, "mg": 1}[precond], None, None, None
        if hasattr(precond, "c_precond"):
            addr, ctx = precond.c_precond()
            return 2, ctypes.c_void_p(addr), ctypes.c_void_p(ctx), precond
        user = precond

        def _cb(ctx, rho, z, stream):
            try:
                self.z.copy_(user(self.rho))
                return 0
            except Exception:
                return 6
        cb = PRECOND_FN(_cb)
        return 2, cb, None, cb

    def solve(self, b, rtol: float = 1e-8, max_iter: int = 500, precond="mg", flexible: bool = False,
              replace_every: int | None = None, chunk: int = 8, x=None, graph: bool = False):
        # a learned preconditioner whose calibration found it slower than
        # the multigrid one on its operator hands the solve to MG-PCG
        if getattr(precond, "use_fallback", False):
            precond, flexible = "mg", False
        # float32 work vectors: the recursively updated residual drifts from
        # b - A x by ~eps32 * cond(A) |b|, so recompute it from the FP64
        # iterate (in FP64) every iteration; float64: every 10
        if replace_every is None:
            replace_every = 1 if self.mg.dtype == torch.float32 else 10
        b = L.as_field(b, dtype=self.mg.dtype)
        if tuple(b.shape) != self.mg.shape:
            raise ValueError("rhs shape does not match the multigrid operator")
        kind, cfn, ctx, keep = self._precond_args(precond)
        if graph:
            if kind == 2 and isinstance(cfn, PRECOND_FN):
                raise ValueError("graph=True needs a C-level preconditioner")
            return self._solve_graph(b, rtol, max_iter, kind, cfn, ctx, keep, flexible, replace_every, chunk, x)
        x = torch.empty(b.shape, dtype=torch.float64, device=b.device) if x is None else x
        info = (ctypes.c_double * 3)()
        st = fn("fvx_pcg_solve")(self._h, P(b), P(x), I(max_iter), D(rtol), I(kind), cfn, ctx, I(int(flexible)),
                                 I(replace_every), I(chunk), info, stream_ptr())
        if st not in (0, 5):
            check(st, "pcg_solve")
        return x, dict(iterations=int(info[0]), rel_residual=float(info[1]), converged=st == 0)

    def _solve_graph(self, b, rtol, max_iter, kind, cfn, ctx, keep, flexible, replace_every, chunk, x_out):
        if self._gb is None:
            self._gb = torch.empty_like(self.rho)
            self._gx = torch.empty(self.mg.shape, dtype=torch.float64, device=self.rho.device)
        self._gb.copy_(b)
        bb = ctypes.c_double()
        check(fn("fvx_pcg_begin")(self._h, P(self._gb), P(self._gx), D(rtol), I(kind), cfn, ctx, ctypes.byref(bb),
                                  stream_ptr()), "pcg_begin")
        # the preconditioner object (kept alive by the cache) and its version
        # identify what the graph captured
        key = (kind, id(keep) if keep is not None else None, getattr(keep, "_version", 0), bool(flexible),
               replace_every)
        if key not in self._graphs:
            # one iteration per replay: the iteration counter, the buffer
            # ping-pong and the residual-replacement schedule live on the
            # device, so the same launches serve every iteration
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                check(fn("fvx_pcg_iterate")(self._h, P(self._gb), P(self._gx), I(0), I(1), I(kind), cfn, ctx,
                                            I(int(flexible)), I(replace_every), stream_ptr()), "pcg_iterate")
            self._graphs[key] = ([g], keep)
            # capture does not run the work: restart from the begin state
            check(fn("fvx_pcg_begin")(self._h, P(self._gb), P(self._gx), D(rtol), I(kind), cfn, ctx,
                                      ctypes.byref(bb), stream_ptr()), "pcg_begin")
        gs = self._graphs[key][0]
        status = (ctypes.c_double * 3)()
        it = 0
        conv = bb.value == 0.0
        rr_prev = bb.value
        tol2 = rtol * rtol * bb.value
        m = min(chunk, 2)
        while not conv and it < max_iter:
            m = min(m, max_iter - it)
            for _ in range(m):
                gs[0].replay()
                it += 1
            check(fn("fvx_pcg_status")(self._h, status, stream_ptr()), "pcg_status")
            conv = status[0] != 0.0
            m = _next_chunk(rr_prev, status[2], m, tol2, chunk)
            rr_prev = status[2]
        rel = ctypes.c_double()
        check(fn("fvx_pcg_finish")(self._h, P(self._gb), P(self._gx), D(bb.value), ctypes.byref(rel), stream_ptr()),
              "pcg_finish")
        x = self._gx.clone() if x_out is None else x_out.copy_(self._gx)
        iters = int(status[1]) if bb.value != 0.0 else 0
        return x, dict(iterations=iters, rel_residual=rel.value, converged=rel.value <= rtol)
