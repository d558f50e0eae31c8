"""Failure detection without a GPU fault.

* A bounded device wait that runs out: the DST plan's fault-injection hook
  makes the products' producers issue no loads, so each MMA warp waits on a
  barrier nothing completes; with a short wait limit (about 1 ms) the wait
  gives up, the CTA ends without trapping, the plan reports status 7 once,
  and the same plan then solves correctly (the context stays usable).
  The U-Net's single-launch inference does the same with a grid barrier that
  one CTA never reaches.
* Non-convergence is a result, not an exception (finitevolX's
  CGInfo.converged, solvers/iterative.py:32-41,129-136): PCG on a NaN
  right-hand side and on an indefinite operator (lambda < 0 beyond the
  Laplacian's spectrum) returns converged=False.
"""

import ctypes

import numpy as np
import pytest
import torch

import finitevolx_b200 as fvx
import oracle.fvx_oracle as O
from finitevolx_b200._lib import FvxError, fn
from finitevolx_b200.solvers import DSTHelmholtzPlan

pytestmark = pytest.mark.gpu


def test_dst_wait_timeout_reports_status_and_recovers(cuda_ok):
    n = 256  # the even/odd single-CTA products
    f = O.kminus3_field(n, n, 21)
    ref = O.solve_helmholtz_dst(f, 0.05, 0.05, 1.0)
    plan = DSTHelmholtzPlan(n, n, 0.05, 0.05, (1.0,))
    rhs = torch.as_tensor(f, dtype=torch.float32, device="cuda")
    plan.solve(rhs)
    plan.check_device()  # a clean solve first
    plan.set_wait_limit(2_000_000)  # ~1 ms
    assert fn("fvx_dst_plan_inject_stall")(plan.handle, 1) == 0
    try:
        plan.solve(rhs)  # the call itself returns normally
        torch.cuda.synchronize()
        rc = fn("fvx_dst_plan_check")(plan.handle, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 7
    finally:
        fn("fvx_dst_plan_inject_stall")(plan.handle, 0)
    # reported once, then cleared; the same plan and context still work
    plan.check_device()
    got = plan.solve(rhs).double().cpu().numpy()
    plan.check_device()
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-4
    with pytest.raises(FvxError):
        plan.set_wait_limit(10)  # below the accepted minimum


def test_unet_barrier_timeout_reports_status_and_recovers(cuda_ok):
    """The U-Net's single-launch inference: with CTA 0 held back from the first
    grid barrier and a ~1 ms wait limit, the other CTAs give up, the launch
    ends, fvx_unet_check reports status 7 once and resets the barrier, and
    the next solve is bit-identical to one before the fault."""
    from finitevolx_b200._lib import D, P, check, stream_ptr
    from finitevolx_b200.learned import UNet

    h = w = 32
    rng = np.random.default_rng(7)
    m = np.ones((h, w), np.float32)
    m[:, :3] = 0.0
    f = torch.from_numpy((rng.standard_normal((h, w)) * m).astype(np.float32)).cuda()
    net = UNet(h, w, batch_max=1)
    mt = torch.from_numpy(m).cuda()
    lt = torch.zeros_like(mt)
    check(fn("fvx_unet_set_level")(net.handle, P(mt), P(lt), D(1.0), stream_ptr()), "set_level")

    def solve():
        u = torch.empty_like(f)
        check(fn("fvx_unet_coarse_fused")(net.handle, P(f), P(u), stream_ptr()), "unet_coarse_fused")
        return u

    u0 = solve()
    net.check_device()
    net.set_wait_limit(2_000_000)  # ~1 ms
    assert fn("fvx_unet_inject_stall")(net.handle, 1) == 0
    try:
        solve()  # the call itself returns normally
        assert fn("fvx_unet_check")(net.handle) == 7
    finally:
        fn("fvx_unet_inject_stall")(net.handle, 0)
    net.check_device()
    u1 = solve()
    net.check_device()
    assert torch.equal(u0, u1)


def _basin(n=128, seed=3):
    rng = np.random.default_rng(seed)
    m = np.zeros((n, n))
    m[4:-4, 4:-4] = 1.0
    m[40:60, 30:90] = 0.0
    c = np.exp(0.3 * rng.standard_normal((n, n)))
    f = rng.standard_normal((n, n)) * m
    return m, c, f


@pytest.mark.parametrize("graph", (False, True))
def test_pcg_nan_rhs_not_converged(cuda_ok, graph):
    m, c, f = _basin()
    dx = 1.0 / 128
    mg = fvx.build_multigrid_solver(m, dx, dx, lambda_=100.0, coeff=c, dtype=torch.float32)
    pcg = fvx.MaskedHelmholtzPCG(mg)
    f[60, 60] = np.nan
    x, info = pcg.solve(torch.as_tensor(f, dtype=torch.float32, device="cuda"), rtol=1e-8, max_iter=20,
                        graph=graph)
    assert info["converged"] is False
    assert info["iterations"] <= 20


def test_pcg_indefinite_operator_not_converged(cuda_ok):
    m, c, f = _basin()
    dx = 1.0 / 128
    # lambda = -4/dx^2 shifts the (negative) spectrum of the variable-
    # coefficient Laplacian across zero: an indefinite operator
    mg = fvx.build_multigrid_solver(m, dx, dx, lambda_=-4.0 / dx ** 2, coeff=np.ones_like(c),
                                    dtype=torch.float64)
    pcg = fvx.MaskedHelmholtzPCG(mg)
    x, info = pcg.solve(torch.as_tensor(f, device="cuda"), rtol=1e-8, max_iter=30, precond="none")
    assert info["converged"] is False
    assert info["iterations"] <= 30


def test_solve_cg_nan_not_converged(cuda_ok):
    n = 64
    b = torch.ones((n, n), dtype=torch.float64, device="cuda")
    b[3, 3] = float("nan")
    x, info = fvx.solve_cg(lambda v: fvx.masked_laplacian(v, torch.ones_like(v), 1.0, 1.0, 1.0), b,
                           max_steps=15)
    assert info.converged is False
    assert info.iterations <= 15
