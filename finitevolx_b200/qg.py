"""QG 1.5-layer model step on the device (scripts/qg_1p5_layer.py:380-561).

The tendency is the reference script's:
    psi   = solve_helmholtz_dst(q[1:-1, 1:-1], dx, dy, 1/Ld^2), zero ghost ring
    u, v  = geostrophic velocity (T_to_X then diff_y_X_to_U / diff_x_X_to_V)
    dq/dt = Advection2D(q, u, v, method) - beta V_to_T(v)
            + forcing - drag laplacian(psi) + viscosity laplacian(q)
stepped with rk3_ssp_step, the ghost ring refilled by the boundary condition
(periodic, or zero for walls) before each tendency and after the step.

``QGModel.step`` runs each RK stage as one DST solve (four tensor-core
products) plus one fused stage kernel; ``QGModel.step_unfused`` runs the
same mathematics as the reference's sequence of separate array operations
(one kernel per operator, every intermediate through HBM) and is the
baseline the fused form is measured against.
"""

from __future__ import annotations

import ctypes

import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import D, I, P, SCHEMES, check, fn, sfx, stream_ptr
from finitevolx_b200.grid import ArakawaCGrid2D
from finitevolx_b200.solvers.spectral import DSTHelmholtzPlan

I64 = ctypes.c_longlong
_FUSED = ("upwind1", "upwind3", "weno3", "weno5", "wenoz5", "weno7", "weno9", "van_leer", "minmod")
# rk3_ssp_step stage weights (explicit_rk.py:110-121): out = a*q_n + b*q_s + (c*dt)*rhs
RK3 = ((0.0, 1.0, 1.0), (0.75, 0.25, 0.25), (1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0))


class QGModel:
    def __init__(self, grid: ArakawaCGrid2D, beta: float, lambda_: float, method: str = "weno5",
                 bc: str = "periodic", drag: float = 0.0, viscosity: float = 0.0, forcing=None,
                 dtype=torch.float32, dst_refine: int = 0):
        if method not in _FUSED:
            raise ValueError(f"QGModel: method {method!r} not supported (choose from {_FUSED})")
        if bc not in ("periodic", "wall"):
            raise ValueError("bc must be 'periodic' or 'wall'")
        self.grid, self.beta, self.lam = grid, float(beta), float(lambda_)
        self.method, self.bc, self.drag, self.visc = method, bc, float(drag), float(viscosity)
        self.dtype = dtype
        dev = L.require_cuda()
        ny, nx = grid.Ny, grid.Nx
        self.plan = DSTHelmholtzPlan(ny - 2, nx - 2, grid.dx, grid.dy, (self.lam,), batch_max=1,
                                     fp64=(dtype == torch.float64) or (nx - 2) % 8 != 0 or (ny - 2) % 8 != 0)
        self.psi = torch.zeros((ny - 2, nx - 2), dtype=dtype, device=dev)
        self.y1 = torch.empty((ny, nx), dtype=dtype, device=dev)
        self.y2 = torch.empty((ny, nx), dtype=dtype, device=dev)
        self.forcing = None if forcing is None else L.as_field(forcing, dtype=dtype)
        hi, lo = ctypes.c_void_p(), ctypes.c_void_p()
        self._fused_split = dtype == torch.float32 and self.plan.split_ok
        self._layout = 0
        if self._fused_split:
            check(fn("fvx_dst_workspace")(self.plan.handle, ctypes.byref(hi), ctypes.byref(lo)), "workspace")
            self._layout = fn("fvx_dst_operand_layout")(self.plan.handle)
        self._w1 = (hi, lo)
        # FP64: the stage kernel writes its output's interior straight into
        # the FP64 chain's input workspace, so the next solve skips its copy
        self._v1 = ctypes.c_void_p()
        self._fused_copy64 = (dtype == torch.float64 and
                              fn("fvx_dst_workspace_f64")(self.plan.handle, ctypes.byref(self._v1)) == 0)
        # FP64-residual refinement passes after each FP32 DST solve (the
        # split chain's ~1e-5 relative psi error, amplified by the velocity
        # differences, exceeds the FP32 step bar in weakly screened fields:
        # small lambda dx^2; one pass brings psi to FP32 rounding)
        self.dst_refine = int(dst_refine) if (dtype == torch.float32 and self.plan.split_ok) else 0
        self.kernel_launches = 0
        # the stage kernel writes the next DST operand split (False: a
        # separate split pass per solve); finitevolx_b200.autotune picks it
        self.fuse_split = True

    # -- pieces --------------------------------------------------------------
    def _dst_from(self, q):
        """psi <- DST solve of q's interior (strided view, no copy)."""
        ny, nx = self.grid.Ny, self.grid.Nx
        view = q.view(-1)[nx + 1:]
        plane = (ny - 2) * (nx - 2)
        if q.dtype == torch.float32:
            check(fn("fvx_dst_solve_f32")(self.plan.handle, P(view), I64(plane), I64(nx), P(self.psi), I64(plane),
                                          I64(nx - 2), I(1), stream_ptr()), "DST solve")
            self._refine(q)
        else:
            check(fn("fvx_dst_solve_f64")(self.plan.handle, P(view), I64(plane), I64(nx), P(self.psi), I64(plane),
                                          I64(nx - 2), I(1), I(0), D(0.0), I(1), None, stream_ptr()), "DST solve")
        self.kernel_launches += 5

    def _dst_presplit(self, q):
        check(fn("fvx_dst_solve_presplit_f32")(self.plan.handle, P(self.psi), I64(self.psi.numel()),
                                               I64(self.grid.Nx - 2), I(1), stream_ptr()), "DST solve")
        self.kernel_launches += 4
        self._refine(q)

    def _dst_presplit64(self):
        check(fn("fvx_dst_solve_presplit_f64")(self.plan.handle, P(self.psi), I64(self.psi.numel()),
                                               I64(self.grid.Nx - 2), I(1), stream_ptr()), "DST solve")
        self.kernel_launches += 4

    def _refine(self, q):
        if not self.dst_refine:
            return
        nx = self.grid.Nx
        view = q.view(-1)[nx + 1:]
        check(fn("fvx_dst_refine_f32")(self.plan.handle, P(view), I64(self.psi.numel()), I64(nx), P(self.psi),
                                       I64(self.psi.numel()), I64(nx - 2), I(1), I(self.dst_refine), stream_ptr()),
              "DST refinement")
        self.kernel_launches += 5 * self.dst_refine

    def _stage(self, qs, qn, out, a, b, c, split, write_ghost):
        g = self.grid
        hi, lo = self._w1 if split else (ctypes.c_void_p(0), ctypes.c_void_p(0))
        if split and self._fused_copy64:
            hi = self._v1  # FP64: the interior copy for the FP64 chain
        check(fn(f"fvx_qg_stage_{sfx(qs)}")(P(qs), P(qn), P(self.psi), P(self.forcing), P(out), hi, lo,
                                            I(self._layout if split else 0), I(g.Ny),
                                            I(g.Nx), D(g.dx), D(g.dy), D(self.beta), D(self.drag), D(self.visc),
                                            D(a), D(b), D(c), I(SCHEMES[self.method]),
                                            I(1 if self.bc == "periodic" else 0), I(int(write_ghost)),
                                            stream_ptr()), "QG stage")
        self.kernel_launches += 1

    # -- public --------------------------------------------------------------
    def tendency(self, q) -> torch.Tensor:
        """dq/dt at T-points (interior; ghost ring left zero)."""
        q = L.as_field(q, dtype=self.dtype)
        self._dst_from(q)
        out = torch.zeros_like(q)
        self._stage(q, None, out, 0.0, 0.0, 1.0, False, False)
        return out

    def step(self, q, dt: float, out=None, presplit: bool = False) -> torch.Tensor:
        """One fused rk3_ssp_step; returns q_{n+1} with its ghost ring refilled.

        ``presplit``: the caller guarantees the DST operand workspace already
        holds q's interior split into bf16 hi/lo (true after a previous
        ``step`` whose output is this ``q``), so the first solve skips the
        split pass.
        """
        q = L.as_field(q, dtype=self.dtype)
        out = torch.empty_like(q) if out is None else out
        split = self._fused_split and self.fuse_split
        copy64 = self._fused_copy64 and self.fuse_split
        presplit = presplit and (split or copy64)
        stages = ((q, self.y1), (self.y1, self.y2), (self.y2, out))
        for s, ((a, b, c), (qs, qo)) in enumerate(zip(RK3, stages)):
            # the stage kernel before this one left qs's interior (split, or
            # as FP64) in the workspace
            if split and (s > 0 or presplit):
                self._dst_presplit(qs)
            elif copy64 and (s > 0 or presplit):
                self._dst_presplit64()
            else:
                self._dst_from(qs)
            # the layout argument stays 0 for FP64 (_layout is 0 there)
            self._stage(qs, None if s == 0 else q, qo, a, b, c * dt, split or copy64, s == 2)
        return out

    # -- unfused baseline: the reference's operator sequence ------------------
    def step_unfused(self, q, dt: float) -> torch.Tensor:
        from finitevolx_b200 import advection as A
        from finitevolx_b200 import boundary as B
        from finitevolx_b200 import operators as O
        from finitevolx_b200.timestepping import lincomb

        g = self.grid

        def bc(x):
            return B.enforce_periodic(x) if self.bc == "periodic" else B.pad_interior(x, "constant")

        def rhs_fn(y):
            qb = bc(y)
            rhs_int = qb[1:-1, 1:-1].contiguous()
            psi_int = self.plan.solve(rhs_int)
            psi = torch.zeros_like(qb)
            psi[1:-1, 1:-1] = psi_int
            px = O.cgrid_op("T_to_X", psi)
            u = lincomb(-1.0, O.cgrid_op("diff_y_X_to_U", px, dx=g.dx, dy=g.dy))
            v = O.cgrid_op("diff_x_X_to_V", px, dx=g.dx, dy=g.dy)
            fe, fnn = A._face_flux(qb, u, v, self.method)
            adv = torch.empty_like(qb)
            check(fn(f"fvx_flux_divergence2d_{sfx(qb)}")(P(fe), P(fnn), P(adv), I(g.Ny), I(g.Nx), D(g.dx), D(g.dy),
                                                         None, stream_ptr()), "divergence")
            vc = O.cgrid_op("V_to_T", v)
            r = lincomb(1.0, adv, -self.beta, vc)
            if self.forcing is not None:
                r = lincomb(1.0, r, 1.0, self.forcing)
            if self.drag:
                r = lincomb(1.0, r, -self.drag, O.cgrid_op("laplacian", psi, dx=g.dx, dy=g.dy))
            if self.visc:
                r = lincomb(1.0, r, self.visc, O.cgrid_op("laplacian", qb, dx=g.dx, dy=g.dy))
            return r

        q = L.as_field(q, dtype=self.dtype)
        k1 = rhs_fn(q)
        y1 = lincomb(1.0, q, dt, k1)
        k2 = rhs_fn(y1)
        y2 = lincomb(0.75, q, 0.25, y1, 0.25 * dt, k2)
        k3 = rhs_fn(y2)
        return bc(lincomb(1.0 / 3.0, q, 2.0 / 3.0, y2, (2.0 / 3.0) * dt, k3))


class QGPipeline:
    """Steps a stream of host-resident states through one QGModel with the
    transfers hidden behind the arithmetic.

    Each state is uploaded from pinned host memory, advanced by one fused
    RK3 step (a CUDA graph replay) and downloaded.  Three CUDA streams run
    the upload of state k+1, the step of state k and the download of state
    k-1 at once (device buffers double-buffered, ordered by events), so a
    run of K states takes about K steps when the step is longer than either
    copy.  This is the serving / ensemble-of-requests form of the step; a
    single trajectory keeps its state on the device instead.
    """

    def __init__(self, model: QGModel, dt: float):
        self.model, self.dt = model, float(dt)
        g = model.grid
        self.din = [torch.zeros((g.Ny, g.Nx), dtype=model.dtype, device="cuda") for _ in range(2)]
        self.dout = [torch.empty_like(self.din[0]) for _ in range(2)]
        self.s_up, self.s_step, self.s_down = (torch.cuda.Stream() for _ in range(3))
        for i in range(2):  # resolves kernel attributes outside capture
            model.step(self.din[i], self.dt, out=self.dout[i])
        torch.cuda.synchronize()
        self.graphs = []
        self.s_step.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(self.s_step):
            for i in range(2):
                gph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(gph, stream=self.s_step):
                    model.step(self.din[i], self.dt, out=self.dout[i])
                self.graphs.append(gph)
        torch.cuda.current_stream().wait_stream(self.s_step)
        self._ev = {k: [torch.cuda.Event() for _ in range(2)] for k in ("up", "step", "down")}

    def run(self, host_in, host_out, n=None, between_steps=None) -> None:
        """Step state ``host_in[k % len(host_in)]`` into ``host_out[k % len(host_out)]``
        for k < n (default len(host_in)).  Host tensors must be pinned and
        [.., Ny, Nx] of the model's dtype.  ``between_steps``: optional
        callable enqueued on the step stream before every step.  Returns
        when everything is enqueued; the current stream waits for the last
        download."""
        n = len(host_in) if n is None else int(n)
        cur = torch.cuda.current_stream()
        for s in (self.s_up, self.s_step, self.s_down):
            s.wait_stream(cur)
        ev = self._ev
        for k in range(n):
            i = k % 2
            with torch.cuda.stream(self.s_up):
                if k >= 2:
                    self.s_up.wait_event(ev["step"][i])  # step k-2 has read din[i]
                self.din[i].copy_(host_in[k % len(host_in)], non_blocking=True)
                ev["up"][i].record(self.s_up)
            with torch.cuda.stream(self.s_step):
                self.s_step.wait_event(ev["up"][i])
                if k >= 2:
                    self.s_step.wait_event(ev["down"][i])  # download k-2 has read dout[i]
                if between_steps is not None:
                    between_steps()
                self.graphs[i].replay()
                ev["step"][i].record(self.s_step)
            with torch.cuda.stream(self.s_down):
                self.s_down.wait_event(ev["step"][i])
                host_out[k % len(host_out)].copy_(self.dout[i], non_blocking=True)
                ev["down"][i].record(self.s_down)
        for s in (self.s_up, self.s_step, self.s_down):
            cur.wait_stream(s)


def geostrophic_velocity(psi, grid: ArakawaCGrid2D):
    """(u, v) from a T-point streamfunction (qg_1p5_layer.py:115-145)."""
    from finitevolx_b200 import operators as O
    from finitevolx_b200.timestepping import lincomb
    px = O.cgrid_op("T_to_X", psi)
    u = lincomb(-1.0, O.cgrid_op("diff_y_X_to_U", px, dx=grid.dx, dy=grid.dy))
    v = O.cgrid_op("diff_x_X_to_V", px, dx=grid.dx, dy=grid.dy)
    return u, v
