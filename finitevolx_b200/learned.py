"""Learned coarse-grid preconditioner for the masked Helmholtz PCG.

finitevolX preconditions its masked, variable-coefficient Helmholtz CG with
one multigrid V-cycle (solvers/preconditioners.py:207-244).  This module
adds a learned alternative: the V-cycle's fine legs (weighted Jacobi,
restriction, prolongation on levels 0 .. lvl-1) around a small U-Net that
replaces the whole coarse part of the cycle at level ``lvl``:

    e_lvl = s * sigma * m_lvl * net([f_lvl / s, m_lvl, log c_lvl])

with s the RMS of the restricted residual f_lvl over wet cells (so the
preconditioner is positively homogeneous) and sigma a fixed output scale.
The network is not a fixed linear map, so it runs inside flexible PCG
(Polak-Ribiere beta); every solve still stops on the same FP64-checked
relative residual as MG-PCG, which stays available as the fallback.

Training pairs (f_lvl, e_lvl) come from the package's own multigrid:
random fine-grid right-hand sides are pushed down the V-cycle's downward
leg to level lvl, and e_lvl is the multigrid solution of A_lvl e = f_lvl
(many independent coarse solves at once, one CTA each).  Forward, backward,
Adam and inference run in libfvx.so (finitevolx_b200/csrc/unet.cu): BF16
weights, FP32 accumulation and activations.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from finitevolx_b200 import _lib as L
from finitevolx_b200._lib import D, I, P, check, fn, stream_ptr
from finitevolx_b200.solvers.multigrid import MultigridSolver

_I64 = ctypes.c_longlong

# (cin, cout) of the eight 3x3 conv layers, in parameter order
LAYERS = ((3, 16), (16, 16), (16, 32), (32, 32), (32, 32), (32, 16), (16, 16), (16, 1))


def _num_params() -> int:
    f = fn("fvx_unet_num_params")
    f.restype = _I64
    return int(f())


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights (fan-in Cin * 9), zero biases, output layer x 0.1."""
    rng = np.random.default_rng(seed)
    parts = []
    for k, (ci, co) in enumerate(LAYERS):
        bound = math.sqrt(6.0 / (ci * 9)) * (0.1 if k == len(LAYERS) - 1 else 1.0)
        parts.append(rng.uniform(-bound, bound, co * ci * 9))
        parts.append(np.zeros(co))
    return np.concatenate(parts).astype(np.float32)


class UNet:
    """Handle on the library's 4-level U-Net (16/16/32/32 channels).

    ``h, w``: grid of the level the network runs on (multiples of 8);
    ``batch_max``: training batch capacity.
    """

    def __init__(self, h: int, w: int, batch_max: int = 32, seed: int = 0):
        L.require_cuda()
        self.h, self.w, self.batch_max = int(h), int(w), int(batch_max)
        self._h = ctypes.c_void_p()
        check(fn("fvx_unet_create")(I(h), I(w), I(batch_max), ctypes.byref(self._h)), "unet_create")
        self.n_params = _num_params()
        self.step = 0
        self.set_params(init_params(seed))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                fn("fvx_unet_destroy")(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    def _io(self, which, offset, count, src=None, dst=None):
        check(fn("fvx_unet_io")(self._h, I(which), _I64(offset), _I64(count), src, dst, stream_ptr()), "unet_io")

    def set_params(self, theta) -> None:
        t = L.as_field(np.ascontiguousarray(theta, np.float32) if not isinstance(theta, torch.Tensor) else theta,
                       dtype=torch.float32)
        if t.numel() != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {t.numel()}")
        self._io(0, 0, self.n_params, src=P(t))
        check(fn("fvx_unet_sync_params")(self._h, stream_ptr()), "unet_sync_params")
        self.step = 0

    def params(self) -> torch.Tensor:
        out = torch.empty(self.n_params, dtype=torch.float32, device="cuda")
        self._io(0, 0, self.n_params, dst=P(out))
        return out

    def grad(self) -> torch.Tensor:
        out = torch.empty(self.n_params, dtype=torch.float32, device="cuda")
        self._io(1, 0, self.n_params, dst=P(out))
        return out

    def _load_x(self, x: torch.Tensor) -> int:
        x = L.as_field(x, dtype=torch.float32)
        B = x.shape[0]
        if tuple(x.shape[1:]) != (3, self.h, self.w) or not 1 <= B <= self.batch_max:
            raise ValueError(f"x must be [1..{self.batch_max}, 3, {self.h}, {self.w}], got {tuple(x.shape)}")
        self._io(2, 0, x.numel(), src=P(x))
        return B

    def forward(self, x) -> torch.Tensor:
        """y = net(x), x [B, 3, h, w] -> y [B, 1, h, w]."""
        B = self._load_x(x)
        check(fn("fvx_unet_forward")(self._h, I(B), stream_ptr()), "unet_forward")
        y = torch.empty((B, 1, self.h, self.w), dtype=torch.float32, device="cuda")
        self._io(3, 0, y.numel(), dst=P(y))
        return y

    def backward(self, x, dy) -> torch.Tensor:
        """dL/dparams for dL/dy = dy at input x (runs the forward pass too)."""
        B = self._load_x(x)
        dy = L.as_field(dy, dtype=torch.float32)
        check(fn("fvx_unet_forward")(self._h, I(B), stream_ptr()), "unet_forward")
        check(fn("fvx_unet_backward")(self._h, I(B), P(dy), stream_ptr()), "unet_backward")
        return self.grad()

    def check_device(self) -> None:
        """Raises if a grid-barrier wait of the single-launch inference gave
        up since the last check (the barrier state is then reset)."""
        check(fn("fvx_unet_check")(self._h), "unet inference")

    def set_wait_limit(self, cycles: int) -> None:
        """Bound, in SM clock cycles, on each grid-barrier wait of the
        single-launch inference."""
        check(fn("fvx_unet_set_wait_limit")(self._h, _I64(int(cycles))), "unet wait limit")

    def train_step(self, x, target, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, loss_out=None) -> None:
        """One Adam step on the masked MSE (mask = channel 1 of x)."""
        B = self._load_x(x)
        t = L.as_field(target, dtype=torch.float32)
        self.step += 1
        check(fn("fvx_unet_train_step")(self._h, I(B), P(t), D(lr), D(beta1), D(beta2), D(eps), I(self.step),
                                        P(loss_out), stream_ptr()), "unet_train_step")


def _level_features(mg: MultigridSolver, lvl: int):
    """(mask, log c) of level lvl: c the mean of the cell's wet face coefficients."""
    lev = mg.level(lvl)
    m = lev["mask"].float()
    cx, cy = lev["cx"].float(), lev["cy"].float()
    cxw = torch.nn.functional.pad(cx[:, :-1], (1, 0))
    cys = torch.nn.functional.pad(cy[:-1, :], (0, 0, 1, 0))
    s = cx + cxw + cy + cys
    k = (cx > 0).float() + (cxw > 0).float() + (cy > 0).float() + (cys > 0).float()
    c = torch.where(k > 0, s / k.clamp(min=1.0), torch.ones_like(s))
    return m.contiguous(), (torch.log(c) * m).contiguous()


def _rms(f, m):
    """Per-sample RMS over wet cells, f [B, h, w], m [h, w]."""
    return torch.sqrt((f.double() ** 2 * m).sum(dim=(1, 2)) / m.sum().clamp(min=1.0)).float()


def generate_pairs(mg: MultigridSolver, lvl: int, n_pairs: int, n_pre: int = 2, seed: int = 0,
                   n_cycles: int = 10, batch: int = 512):
    """MG-generated training pairs at level lvl.

    Each pair starts from a random fine-grid right-hand side r (white noise
    for half the pairs, a smooth field -- one V-cycle applied to white
    noise -- for the other half, both masked), takes f = the level-lvl
    restricted residual after ``n_pre`` sweeps per level (the downward leg
    the preconditioner runs), and solves A_lvl e = f by ``n_cycles``
    multigrid cycles.  Returns (f [N, h, w], e [N, h, w]) FP32 tensors.
    """
    if mg.dtype != torch.float32:
        raise ValueError("the learned preconditioner runs on a float32 MultigridSolver")
    lev0 = mg.level(0)
    m0 = lev0["mask"]
    h, w = mg.level(lvl)["mask"].shape
    gen = torch.Generator(device="cuda").manual_seed(int(seed))
    F = torch.empty((n_pairs, h, w), dtype=torch.float32, device="cuda")
    E = torch.empty_like(F)
    f_lvl = fn("fvx_mg_restrict_residual")
    work_n = fn("fvx_mg_level_work")
    work_n.restype = _I64
    wpb = int(work_n(mg.handle, I(lvl)))
    for k in range(n_pairs):
        r = torch.randn(mg.shape, generator=gen, device="cuda", dtype=torch.float32) * m0
        if k % 2:
            r = mg.v_cycle(None, r) * m0
        check(f_lvl(mg.handle, P(r), I(lvl), I(n_pre), P(F[k]), stream_ptr()), "restrict_residual")
    for a in range(0, n_pairs, batch):
        b = min(n_pairs, a + batch)
        work = torch.empty((b - a) * wpb, dtype=torch.float32, device="cuda")
        check(fn("fvx_mg_solve_level_batched")(mg.handle, I(lvl), I(b - a), P(F[a:b]), P(E[a:b]), I(n_cycles),
                                               P(work), stream_ptr()), "solve_level_batched")
    return F, E


class LearnedPreconditioner:
    """Hybrid V-cycle with a trained U-Net as the level-``lvl`` solver.

    ``mg`` must be a float32 MultigridSolver.  Use ``fit`` (or ``train`` on
    pairs from ``generate_pairs``), then pass the object as ``precond`` to
    MaskedHelmholtzPCG.solve with ``flexible=True``.  ``coarse=False``
    drops the network (zero coarse correction) -- the same method without
    the learned part; ``coarse="mg"`` solves the level-lvl problem by
    ``mg_cycles`` multigrid cycles instead (the exact-coarse-solve limit).
    ``scale`` multiplies the coarse correction d by the energy-optimal
    omega = (d . f) / (d . A d), so it never increases the level-lvl error;
    ``n_smooth`` Jacobi sweeps at level lvl follow it.  Changing these
    attributes takes effect after ``rebuild()``.
    """

    def __init__(self, mg: MultigridSolver, lvl: int | None = None, n_pre: int = 2, n_post: int = 2,
                 batch_max: int = 32, seed: int = 0, coarse=True, mg_cycles: int = 10, n_smooth: int = 0,
                 scale: bool = True):
        if mg.dtype != torch.float32:
            raise ValueError("the learned preconditioner runs on a float32 MultigridSolver")
        self.mg = mg
        if lvl is None:  # the first level at or below 128 x 128 cells
            lvl = max(1, next(k for k in range(mg.n_levels) if mg.level(k)["mask"].numel() <= 128 * 128))
        if not 1 <= lvl < mg.n_levels:
            raise ValueError(f"level {lvl} outside 1 .. {mg.n_levels - 1}")
        self.lvl, self.n_pre, self.n_post, self.n_smooth = int(lvl), int(n_pre), int(n_post), int(n_smooth)
        self.scale = bool(scale)
        self._version = 0
        self.m_lvl, self.logc = _level_features(mg, self.lvl)
        h, w = self.m_lvl.shape
        if h % 8 or w % 8:
            raise ValueError(f"level {lvl} grid {h}x{w} is not a multiple of 8")
        self.net = UNet(h, w, batch_max, seed)
        self.sigma = 1.0
        self.mode = "net" if coarse is True else ("mg" if coarse == "mg" else "none")
        self._ls = ctypes.c_void_p()
        if self.mode == "mg":
            check(fn("fvx_levelsolve_create")(mg.handle, I(self.lvl), I(mg_cycles), ctypes.byref(self._ls)),
                  "levelsolve_create")
        self._hy = ctypes.c_void_p()
        self.use_fallback = False  # set by calibrate(): MG-PCG is the faster method here
        self.calibration = None
        self._make_hybrid()

    def _make_hybrid(self):
        if self._hy.value:
            fn("fvx_hybrid_destroy")(self._hy)
            self._hy = ctypes.c_void_p()
        if self.mode == "net":
            coarse, ctx = ctypes.cast(fn("fvx_unet_coarse"), ctypes.c_void_p), self.net.handle
        elif self.mode == "mg":
            coarse, ctx = ctypes.cast(fn("fvx_levelsolve_coarse"), ctypes.c_void_p), self._ls
        else:
            coarse, ctx = None, None
        check(fn("fvx_hybrid_create")(self.mg.handle, I(self.lvl), I(self.n_pre), I(self.n_post), I(self.n_smooth),
                                      I(int(self.scale and self.mode != "none")), coarse, ctx,
                                      ctypes.byref(self._hy)), "hybrid_create")
        self._version += 1

    def rebuild(self):
        """Apply changed n_pre / n_post / n_smooth / scale."""
        self._make_hybrid()

    def __del__(self):
        for name, dtor in (("_hy", "fvx_hybrid_destroy"), ("_ls", "fvx_levelsolve_destroy")):
            h = getattr(self, name, None)
            if h is not None and h.value:
                try:
                    fn(dtor)(h)
                except Exception:
                    pass
                setattr(self, name, None)

    # -- training -----------------------------------------------------------
    def make_inputs(self, F, E=None):
        """Normalised network inputs [N, 3, h, w] (and targets [N, 1, h, w])."""
        s = _rms(F, self.m_lvl).clamp(min=1e-30)
        N = F.shape[0]
        X = torch.empty((N, 3) + tuple(self.m_lvl.shape), dtype=torch.float32, device="cuda")
        X[:, 0] = F / s[:, None, None]
        X[:, 1] = self.m_lvl
        X[:, 2] = self.logc
        if E is None:
            return X
        T = (E / (s[:, None, None] * self.sigma))[:, None].contiguous()
        return X, T

    def train(self, F, E, epochs: int = 20, batch: int = 32, lr: float = 2e-3, seed: int = 0,
              lr_final: float = 1e-4):
        """Adam on (F, E) pairs; sigma is fixed first from the data.  Returns
        the mean loss of each epoch."""
        ratio = _rms(E, self.m_lvl) / _rms(F, self.m_lvl).clamp(min=1e-30)
        self.sigma = float(ratio.median().item())
        X, T = self.make_inputs(F, E)
        N = X.shape[0]
        batch = min(batch, self.net.batch_max, N)
        gen = torch.Generator(device="cuda").manual_seed(int(seed))
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        hist = []
        steps = epochs * (N // batch)
        k = 0
        for ep in range(epochs):
            perm = torch.randperm(N, generator=gen, device="cuda")
            acc = torch.zeros((), dtype=torch.float64, device="cuda")
            nb = N // batch
            for j in range(nb):
                idx = perm[j * batch:(j + 1) * batch]
                # cosine decay from lr to lr_final
                lr_k = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * k / max(steps, 1)))
                self.net.train_step(X[idx], T[idx], lr=lr_k, loss_out=loss)
                acc += loss[0]
                k += 1
            hist.append(float(acc.item()) / max(nb, 1))
        self.activate()
        return hist

    def fit(self, n_pairs: int = 2048, epochs: int = 20, batch: int = 32, lr: float = 2e-3, seed: int = 0,
            n_cycles: int = 10):
        F, E = generate_pairs(self.mg, self.lvl, n_pairs, self.n_pre, seed, n_cycles)
        return self.train(F, E, epochs, batch, lr, seed)

    def calibrate(self, pcg, b, rtol: float = 1e-8, reps: int = 3) -> dict:
        """Time flexible PCG with this preconditioner against MG-PCG (the
        multigrid V-cycle, its fallback) on a calibration right-hand side
        ``b`` and the solver ``pcg`` (a MaskedHelmholtzPCG on the same
        operator); when MG-PCG is faster, later solves given this object use
        MG-PCG (``use_fallback``).  Both reach ``rtol`` checked in FP64.
        Returns the two times (median of ``reps``, ms) and iteration counts."""
        import statistics

        def timed(**kw):
            pcg.solve(b, rtol=rtol, graph=True, **kw)
            ts, info = [], None
            for _ in range(reps):
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                _, info = pcg.solve(b, rtol=rtol, graph=True, **kw)
                e1.record()
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            return statistics.median(ts), info

        self.use_fallback = False
        t_net, i_net = timed(precond=self, flexible=True, max_iter=500)
        t_mg, i_mg = timed(precond="mg")
        self.use_fallback = (not i_net["converged"]) or t_mg < t_net
        self.calibration = {"learned_ms": t_net, "learned_iterations": i_net["iterations"], "mg_ms": t_mg,
                            "mg_iterations": i_mg["iterations"], "use_fallback": self.use_fallback}
        return self.calibration

    def activate(self):
        """Point the inference path at this level's mask, coefficient and sigma."""
        check(fn("fvx_unet_set_level")(self.net.handle, P(self.m_lvl), P(self.logc), D(self.sigma), stream_ptr()),
              "unet_set_level")

    # -- inference ----------------------------------------------------------
    def coarse_solve(self, f_lvl, fused: bool = False) -> torch.Tensor:
        """The network's approximation of A_lvl^{-1} f_lvl: one launch per
        layer (``fused=True``: the same solve as one cooperative launch)."""
        f = L.as_field(f_lvl, dtype=torch.float32)
        u = torch.empty_like(f)
        name = "fvx_unet_coarse_fused" if fused else "fvx_unet_coarse"
        check(fn(name)(self.net.handle, P(f), P(u), stream_ptr()), "unet_coarse")
        return u

    def __call__(self, r) -> torch.Tensor:
        """z = M r (the hybrid cycle)."""
        r = L.as_field(r, dtype=torch.float32)
        z = torch.empty_like(r)
        check(fn("fvx_hybrid_precond")(self._hy, P(r), P(z), stream_ptr()), "hybrid_precond")
        return z

    def c_precond(self):
        """(address of fvx_hybrid_precond, context) for MaskedHelmholtzPCG."""
        return ctypes.cast(fn("fvx_hybrid_precond"), ctypes.c_void_p).value, self._hy.value
