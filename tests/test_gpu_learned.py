"""GPU checks of the learned preconditioner.

* U-Net forward, gradients (backward) and one Adam step against the FP64
  NumPy oracle with the same BF16-rounded weights.  Tolerances: forward 2e-5
  normwise relative (FP32 accumulation over <= 288-term sums), gradients 1e-4
  normwise per layer, Adam 1e-6 absolute on lr = 1e-3 steps.
* The hybrid cycle's pieces (downward leg, batched level solves, zero-
  correction cycle) against the oracle in FP32: 1e-5 normwise.
* Training lowers the loss; flexible PCG with the trained network reaches the
  FP64-checked 1e-8 relative residual and needs fewer iterations than the same
  cycle without the network.
"""

import numpy as np
import pytest
import torch

import finitevolx_b200 as fvx
import oracle.fvx_oracle as O
import oracle.unet_oracle as U
from finitevolx_b200._lib import P
from finitevolx_b200.learned import LearnedPreconditioner, UNet, generate_pairs

from test_gpu_solvers import basin, coeff

pytestmark = pytest.mark.gpu


def nrel(a, b):
    a = np.asarray(a, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _net_case(seed=0, B=2, h=32, w=32):
    rng = np.random.default_rng(seed)
    theta = U.init_params(seed)
    # non-zero biases so every bias gradient path is exercised
    off = 0
    for ci, co, *_ in U.LAYERS:
        off += co * ci * 9
        theta[off:off + co] = rng.uniform(-0.1, 0.1, co)
        off += co
    x = rng.standard_normal((B, 3, h, w)).astype(np.float32)
    x[:, 1] = (rng.random((B, h, w)) > 0.25).astype(np.float32)
    t = rng.standard_normal((B, 1, h, w)).astype(np.float32)
    return theta, x, t


def test_unet_forward_matches_oracle(cuda_ok):
    theta, x, _ = _net_case()
    net = UNet(32, 32, batch_max=4)
    net.set_params(theta)
    y = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    ref = U.forward(theta.astype(np.float64), x)[8]
    assert nrel(y, ref) < 2e-5


def test_unet_gradients_match_oracle(cuda_ok):
    theta, x, t = _net_case(1, B=3, h=32, w=48)
    Lr, gref, acts = U.loss_and_grad(theta.astype(np.float64), x, t)
    m = x[:, 1:2].astype(np.float64)
    N = t.shape[0] * t.shape[2] * t.shape[3]
    dy = (2.0 * (acts[8] - t) * m * m / N).astype(np.float32)
    net = UNet(32, 48, batch_max=3)
    net.set_params(theta)
    g = net.backward(torch.from_numpy(x).cuda(), torch.from_numpy(dy).cuda()).cpu().numpy()
    off = 0
    for k, (ci, co, *_r) in enumerate(U.LAYERS):
        n = co * ci * 9 + co
        assert nrel(g[off:off + n], gref[off:off + n]) < 1e-4, f"layer {k}"
        off += n


def test_unet_gradients_match_oracle_many_items(cuda_ok):
    # 8 samples at 128^2: the full-resolution layers have 512 (sample, tile)
    # items, more than the weight-gradient kernel's partial rows, so its
    # blocks accumulate several items each; and the result is run-to-run
    # identical (fixed-order partial sums).  In this case one pre-activation
    # of layer 6 lies within FP32 rounding of zero, so the FP32 pass and the
    # FP64 oracle disagree on its ReLU; that pixel moves the gradients of the
    # layers below (0-2) by ~2e-4 relative, whatever the summation order, so
    # those take 1e-3 and the rest 1e-4.
    theta, x, t = _net_case(5, B=8, h=128, w=128)
    Lr, gref, acts = U.loss_and_grad(theta.astype(np.float64), x, t)
    m = x[:, 1:2].astype(np.float64)
    N = t.shape[0] * t.shape[2] * t.shape[3]
    dy = (2.0 * (acts[8] - t) * m * m / N).astype(np.float32)
    net = UNet(128, 128, batch_max=8)
    net.set_params(theta)
    xd, dyd = torch.from_numpy(x).cuda(), torch.from_numpy(dy).cuda()
    g = net.backward(xd, dyd).cpu().numpy()
    np.testing.assert_array_equal(net.backward(xd, dyd).cpu().numpy(), g)
    off = 0
    for k, (ci, co, *_r) in enumerate(U.LAYERS):
        n = co * ci * 9 + co
        assert nrel(g[off:off + n], gref[off:off + n]) < (1e-3 if k <= 2 else 1e-4), f"layer {k}"
        off += n


def test_unet_train_step_loss_and_adam(cuda_ok):
    theta, x, t = _net_case(2, B=2, h=16, w=16)
    net = UNet(16, 16, batch_max=2)
    net.set_params(theta)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    net.train_step(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), lr=1e-3, loss_out=loss)
    Lr, gref, _ = U.loss_and_grad(theta.astype(np.float64), x, t)
    assert abs(loss.item() - Lr) <= 1e-5 * Lr
    g = net.grad().cpu().numpy().astype(np.float64)
    th1, _, _ = U.adam(theta.astype(np.float64), g, 0.0, 0.0, 1, lr=1e-3)
    np.testing.assert_allclose(net.params().cpu().numpy(), th1, atol=1e-6, rtol=0)


def _set_level(net, m, logc, sigma):
    from finitevolx_b200._lib import D, P, check, fn, stream_ptr
    mt = torch.from_numpy(m).cuda()
    lt = torch.from_numpy(logc).cuda()
    check(fn("fvx_unet_set_level")(net.handle, P(mt), P(lt), D(sigma), stream_ptr()), "set_level")
    torch.cuda.synchronize()


def _coarse(net, f, fused=False):
    from finitevolx_b200._lib import P, check, fn, stream_ptr
    ft = torch.from_numpy(f).cuda()
    u = torch.empty_like(ft)
    name = "fvx_unet_coarse_fused" if fused else "fvx_unet_coarse"
    check(fn(name)(net.handle, P(ft), P(u), stream_ptr()), name)
    return u


@pytest.mark.parametrize("h,w", [(64, 64), (40, 56), (128, 128)])
def test_unet_coarse_single_launch_matches_oracle(cuda_ok, h, w):
    """The coarse solve (per-layer launches, and the same in one cooperative
    launch) against the oracle's s sigma m net([f / s, m, log c]);
    40 x 56 leaves partial tiles on every level."""
    theta, _, _ = _net_case(5, B=1, h=h, w=w)
    rng = np.random.default_rng(6)
    m = (rng.random((h, w)) > 0.3).astype(np.float32)
    logc = (0.3 * rng.standard_normal((h, w)) * m).astype(np.float32)
    f = (rng.standard_normal((h, w)) * m).astype(np.float32)
    net = UNet(h, w, batch_max=1)
    net.set_params(theta)
    sigma = 0.37
    _set_level(net, m, logc, sigma)
    u = _coarse(net, f, fused=True)
    u2 = _coarse(net, f, fused=True)
    ul = _coarse(net, f)
    net.check_device()
    fd, md = f.astype(np.float64), m.astype(np.float64)
    s = np.sqrt((fd * fd * md).sum() / max(md.sum(), 1.0))
    x = np.stack([fd / s, md, logc.astype(np.float64)])[None]
    ref = s * sigma * md * U.forward(theta.astype(np.float64), x)[8][0, 0]
    got = u.cpu().numpy()
    assert nrel(got, ref) < 2e-5
    assert nrel(ul.cpu().numpy(), ref) < 2e-5
    assert nrel(got, ul.cpu().numpy()) < 1e-6
    assert torch.equal(u, u2)  # fixed reduction order: run-to-run identical
    assert np.all(got[m == 0] == 0)


@pytest.mark.parametrize("h,w", [(128, 128), (40, 56)])
def test_unet_coarse_fused_layers_equal_generic_forward(cuda_ok, h, w):
    """The coarse solve's fused first-two and last-two layer kernels give
    exactly the generic per-layer forward pass on x = [f * (1/s), m, log c],
    scaled by (s sigma) and masked as the output hook does."""
    theta, _, _ = _net_case(9, B=1, h=h, w=w)
    rng = np.random.default_rng(10)
    m = (rng.random((h, w)) > 0.3).astype(np.float32)
    logc = (0.3 * rng.standard_normal((h, w)) * m).astype(np.float32)
    f = (rng.standard_normal((h, w)) * m).astype(np.float32)
    net = UNet(h, w, batch_max=1)
    net.set_params(theta)
    sigma = 0.61
    _set_level(net, m, logc, sigma)
    u = _coarse(net, f)
    sc = torch.empty(2, dtype=torch.float32, device="cuda")
    net._io(4, 0, 2, dst=P(sc))
    torch.cuda.synchronize()
    ft, mt = torch.from_numpy(f).cuda(), torch.from_numpy(m).cuda()
    x = torch.stack([ft * sc[1], mt, torch.from_numpy(logc).cuda()])[None]
    y = net.forward(x)[0, 0]
    ref = (y * (sc[0] * torch.tensor(sigma, dtype=torch.float32, device="cuda"))) * mt
    assert torch.equal(u, ref)


@pytest.fixture(scope="module")
def problem128(cuda_ok):
    n = 128
    m = basin(n, 21)
    c = coeff(n, 22)
    lam = 0.0156 * n * n  # lambda dx^2 = 0.0156 (deformation radius 8 cells)
    mg = fvx.build_multigrid_solver(m, 1.0 / n, 1.0 / n, lambda_=lam, coeff=c, dtype=torch.float32)
    ref = O.mg_build(m, 1.0 / n, 1.0 / n, lambda_=lam, coeff=c)
    return n, m, c, lam, mg, ref


def test_hybrid_pieces_match_oracle(problem128):
    n, m, c, lam, mg, ref = problem128
    rng = np.random.default_rng(23)
    f = (rng.standard_normal((n, n)) * m).astype(np.float32)
    lvl = 2
    from finitevolx_b200._lib import I, P, check, fn, stream_ptr
    h = n >> lvl
    fl = torch.empty((h, h), dtype=torch.float32, device="cuda")
    check(fn("fvx_mg_restrict_residual")(mg.handle, P(torch.from_numpy(f).cuda()), I(lvl), I(2), P(fl),
                                         stream_ptr()), "restrict")
    _, fs = O.mg_restrict_residual(ref, f.astype(np.float64), lvl, 2)
    assert nrel(fl.cpu().numpy(), fs[lvl]) < 1e-5
    F, E = generate_pairs(mg, lvl, 4, n_pre=2, seed=3, n_cycles=6)
    for k in range(4):
        e_ref = O.mg_level_solve(ref, lvl, F[k].double().cpu().numpy(), 6)
        assert nrel(E[k].cpu().numpy(), e_ref) < 1e-5
    pc0 = LearnedPreconditioner(mg, lvl=lvl, coarse=False)
    z = pc0(torch.from_numpy(f).cuda()).cpu().numpy()
    assert nrel(z, O.mg_hybrid(ref, f.astype(np.float64), lvl, 2, 2)) < 1e-5


def test_learned_pcg_gain(problem128):
    n, m, c, lam, mg, ref = problem128
    pc = LearnedPreconditioner(mg, lvl=2, n_pre=2, n_post=2, batch_max=32, seed=0)
    hist = pc.fit(n_pairs=1024, epochs=12, batch=32, lr=2e-3, seed=1)
    assert hist[-1] < 0.5 * hist[0], hist
    pcg = fvx.MaskedHelmholtzPCG(mg)
    f = O.kminus3_field(n, n, 24) * m
    b = torch.from_numpy(f).float().cuda()
    x, info = pcg.solve(b, rtol=1e-8, precond=pc, flexible=True, max_iter=300)
    assert info["converged"] and info["rel_residual"] <= 1e-8, info
    # FP64 check of the returned iterate against the oracle operator
    fb = b.double().cpu().numpy()
    r = fb - O.mg_apply(x.cpu().numpy(), ref["levels"][0])
    assert np.linalg.norm(r) <= 1.01e-8 * np.linalg.norm(fb)
    pc0 = LearnedPreconditioner(mg, lvl=2, n_pre=2, n_post=2, coarse=False)
    x0, info0 = pcg.solve(b, rtol=1e-8, precond=pc0, flexible=True, max_iter=300)
    assert info0["converged"], info0
    assert info["iterations"] < info0["iterations"], (info, info0)
    # graph replay gives the same iterations and tolerance
    xg, infog = pcg.solve(b, rtol=1e-8, precond=pc, flexible=True, max_iter=300, graph=True)
    assert infog["converged"] and abs(infog["iterations"] - info["iterations"]) <= 1, (infog, info)
    # calibration against MG-PCG: the faster method is kept, and with the
    # fallback set a solve given the preconditioner runs MG-PCG itself
    cal = pc.calibrate(pcg, torch.from_numpy(O.kminus3_field(n, n, 25) * m).float().cuda(), reps=1)
    assert pc.use_fallback == (cal["mg_ms"] < cal["learned_ms"]), cal
    pc.use_fallback = True
    xf, infof = pcg.solve(b, rtol=1e-8, precond=pc, flexible=True, max_iter=300, graph=True)
    xm, infom = pcg.solve(b, rtol=1e-8, precond="mg", max_iter=300, graph=True)
    assert infof["iterations"] == infom["iterations"] and torch.equal(xf, xm)
    pc.use_fallback = False
