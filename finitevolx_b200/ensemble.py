"""Ensembles of multi-layer QG models with uneven grid sizes and layer counts.

Each member is an nl-layer QG model (nl <= 3) on an n x n interior with one
ghost ring: PV inverted through the vertical modes of
``build_coupling_matrix(H[:nl], g'[:nl])`` (vertical/vertical_modes.py:50-263,
solvers/elliptic.py:390-542) and every layer stepped with the 1.5-layer
tendency (scripts/qg_1p5_layer.py:454-487) in rk3_ssp_step.  One call to
``step`` advances every member; on the device a step is, per RK stage, one
batched tensor-core DST chain per grid size and one persistent fused-stage
launch over all tiles of all members (an atomic work queue), so a whole run
can be captured in a single CUDA graph (``capture``).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import I, P, SCHEMES, check, fn, require_cuda, stream_ptr
from finitevolx_b200.vertical import build_coupling_matrix, decompose_vertical_modes

H_DEFAULT = (400.0, 1100.0, 2600.0)
GPRIME_DEFAULT = (9.81, 0.025, 0.0125)


class QGEnsemble:
    """``members``: sequence of (n, nl).  Grid spacing dx = Lx / n, time step
    dt = cfl * dx / umax per member; beta, f0 shared."""

    def __init__(self, members, Lx: float = 5.12e6, beta: float = 1.7e-11, f0: float = 9.375e-5,
                 H=H_DEFAULT, gprime=GPRIME_DEFAULT, method: str = "weno5", cfl: float = 0.5, umax: float = 1.0,
                 refine_passes: int = 1):
        require_cuda()
        self.members = [(int(n), int(nl)) for n, nl in members]
        self.Lx, self.beta, self.f0, self.method = float(Lx), float(beta), float(f0), method
        ns, nls, l2m, m2l, lam, dxs, dts = [], [], [], [], [], [], []
        self.modes = []
        for n, nl in self.members:
            A = build_coupling_matrix(H[:nl], gprime[:nl])
            rr, a2m, m2a = decompose_vertical_modes(A, f0)
            lm = np.where(np.isfinite(rr), 1.0 / np.where(np.isfinite(rr), rr, 1.0) ** 2, 0.0)
            dx = self.Lx / n
            ns.append(n)
            nls.append(nl)
            l2m.extend(np.asarray(a2m, np.float64).ravel())
            m2l.extend(np.asarray(m2a, np.float64).ravel())
            lam.extend(lm)
            dxs.append(dx)
            dts.append(cfl * dx / umax)
            self.modes.append((np.asarray(a2m, np.float64), np.asarray(m2a, np.float64), lm))
        self.dx = dxs
        self.dt = dts
        arr = lambda v, t: (t * len(v))(*v)  # noqa: E731
        self._h = ctypes.c_void_p()
        check(fn("fvx_ens_create")(I(len(ns)), arr(ns, ctypes.c_int), arr(nls, ctypes.c_int),
                                   arr(l2m, ctypes.c_double), arr(m2l, ctypes.c_double), arr(lam, ctypes.c_double),
                                   arr(dxs, ctypes.c_double), arr(dxs, ctypes.c_double),
                                   arr(dts, ctypes.c_double), ctypes.c_double(beta), I(SCHEMES[method]),
                                   ctypes.byref(self._h)), "ensemble create")
        self._graph = None
        self.set_refine(refine_passes)

    def set_refine(self, passes: int) -> None:
        """FP64-residual refinement passes after the DST solves of the weakly
        screened modes (lambda (n dx)^2 < 2000: single-layer members with a
        deformation radius above ~L/45, every barotropic mode): the split
        tensor-core chain carries its intermediates in 16 bits (about 1e-5
        relative error in psi), which the velocity differences amplify past
        the FP32 step bar for those modes; one pass brings psi to FP32
        rounding.  Strongly screened modes skip it."""
        check(fn("fvx_ens_set_refine")(self._h, I(int(passes))), "ensemble refine")
        self.refine_passes = int(passes)
        self._graph = None

    def __del__(self):
        self._graph = None
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                fn("fvx_ens_destroy")(h)
            except Exception:
                pass
            self._h = None

    @property
    def launches_per_step(self) -> int:
        return fn("fvx_ens_launches_per_step")(self._h)

    def cells_per_step(self) -> int:
        """Interior layer-cells advanced by one step of the whole ensemble."""
        return sum(n * n * nl for n, nl in self.members)

    def set_layer(self, member: int, layer: int, q) -> None:
        n = self.members[member][0]
        t = L.as_field(q, dtype=torch.float32)
        if tuple(t.shape) != (n + 2, n + 2):
            raise ValueError(f"member {member}: expected ({n + 2}, {n + 2}), got {tuple(t.shape)}")
        check(fn("fvx_ens_io")(self._h, I(member), I(layer), P(t), None, stream_ptr()), "ensemble set")
        torch.cuda.current_stream().synchronize()

    def get_layer(self, member: int, layer: int) -> torch.Tensor:
        n = self.members[member][0]
        out = torch.empty((n + 2, n + 2), dtype=torch.float32, device="cuda")
        check(fn("fvx_ens_io")(self._h, I(member), I(layer), None, P(out), stream_ptr()), "ensemble get")
        return out

    def set_blocks_per_sm(self, k: int) -> None:
        """Persistent stage grid size (0 = as many CTAs as fit per SM)."""
        check(fn("fvx_ens_set_blocks_per_sm")(self._h, I(k)), "ensemble blocks")
        self._graph = None

    def step(self, n_steps: int = 1) -> None:
        """Advance every member by n_steps RK3-SSP steps (stream-ordered launches)."""
        check(fn("fvx_ens_step")(self._h, I(n_steps), stream_ptr()), "ensemble step")

    def capture(self, n_steps: int):
        """A CUDA graph of n_steps steps of the whole ensemble; ``.replay()`` runs it."""
        self.step(1)  # first call resolves kernel attributes outside capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.step(n_steps)
        torch.cuda.current_stream().wait_stream(s)
        self._graph = g
        return g
