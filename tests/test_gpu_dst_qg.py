"""GPU parity: DST Helmholtz (tensor-core split chain, FP64 chain, refinement)
and the QG RK3 step (fused and unfused) vs the FP64 oracle.

Tolerances: FP64 chain 1e-12 (normwise relative, max norm); FP32 3xBF16
chain 1e-4 of max|psi| (measured ~1e-5); refinement: normwise backward
error <= 1e-12 and 1e-10 of max|psi| vs the oracle; FP32 QG step: 1e-5
relative on q_{n+1} (the stated FP32-step bar); FP64 QG step: 1e-12.
"""

import numpy as np
import pytest
import torch

import finitevolx_b200 as fvx
import oracle.fvx_oracle as O
from finitevolx_b200.qg import QGModel
from finitevolx_b200.solvers import DSTHelmholtzPlan, solve_helmholtz_dst

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device="cuda")


def host(t):
    return t.detach().cpu().numpy().astype(np.float64)


def rel_err(a, b):
    return np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-300)


# (256, 512), (512, 256): multiples of 256, the even/odd (half-work) products
@pytest.mark.parametrize("shape,lam", [((128, 128), 0.0), ((256, 128), 3.0), ((64, 192), 50.0),
                                       ((256, 512), 2.0), ((512, 256), 0.0)])
def test_dst_split_bf16_chain(cuda_ok, shape, lam):
    ny, nx = shape
    f = O.kminus3_field(ny, nx, 3)
    ref = O.solve_helmholtz_dst(f, 0.05, 0.07, lam)
    got = solve_helmholtz_dst(dev(f, torch.float32), 0.05, 0.07, lam)
    plan = DSTHelmholtzPlan(ny, nx, 0.05, 0.07, (lam,))
    plan.check_device()
    from finitevolx_b200._lib import fn
    assert fn("fvx_dst_operand_layout")(plan.handle) == int(ny % 256 == 0 and nx % 256 == 0)
    e = rel_err(host(got), ref)
    assert e < 1e-4, e


@pytest.mark.parametrize("shape", [(256, 512), (512, 256), (768, 512), (2048, 2048)])
def test_dst_product_forms_agree(cuda_ok, shape):
    # the even/odd products on single CTAs (64- and 32-element K blocks) and
    # on CTA pairs (cta_group::2, B blocks shared by the pair): the same
    # 3xBF16 sums in another k order.  All within the chain's 1e-4 of the
    # oracle; against each other within 5e-5: an intermediate that differs
    # by one FP32 ulp can round to another bf16 hi/lo pair, which moves it by
    # up to 2^-16 relative (~1e-5 after the chain)
    from finitevolx_b200.autotune import DST_KERNELS, set_dst_kernel
    from finitevolx_b200._lib import fn
    ny, nx = shape
    f = O.kminus3_field(ny, nx, 4)
    ref = O.solve_helmholtz_dst(f, 0.05, 0.07, 1.0)
    outs = []
    try:
        for k, name in enumerate(DST_KERNELS):
            set_dst_kernel(name)
            assert fn("fvx_dst_kernel_config")(-1) == k
            plan = DSTHelmholtzPlan(ny, nx, 0.05, 0.07, (1.0,))
            outs.append(host(plan.solve(dev(f, torch.float32))))
            plan.check_device()
    finally:
        set_dst_kernel("single64")
    for o in outs:
        assert rel_err(o, ref) < 1e-4
    for o in outs[1:]:
        assert rel_err(o, outs[0]) < 5e-5


# The FP64 products take 16-, 32- or 64-element output tiles by problem size
# (the largest giving at least 148 tiles): the first three shapes run on
# 16-tiles, (420, 388) on 32-tiles and (790, 780) on 64-tiles, both with
# partial edge tiles.
@pytest.mark.parametrize("shape", [(40, 56), (37, 29), (128, 128), (420, 388), (790, 780)])
def test_dst_fp64_chain(cuda_ok, shape):
    ny, nx = shape
    f = np.random.default_rng(1).standard_normal((ny, nx))
    ref = O.solve_helmholtz_dst(f, 0.1, 0.2, 1.5)
    got = solve_helmholtz_dst(dev(f), 0.1, 0.2, 1.5)
    assert rel_err(host(got), ref) < 1e-12


def test_dst_fp64_chain_tile_size_keeps_result(cuda_ok):
    # one 128^2 right-hand side runs the FP64 products on 16 x 16 tiles
    # (128-long k-blocks); a batch of ten on 32 x 32 tiles (16-long
    # k-blocks).  Every output's FMA chain over k keeps its order in both, so
    # the results are bit-identical
    n = 128
    f = np.random.default_rng(9).standard_normal((n, n))
    one = host(solve_helmholtz_dst(dev(f), 0.1, 0.2, 1.5))
    batch = host(solve_helmholtz_dst(dev(np.stack([f] * 10)), 0.1, 0.2, 1.5))
    for k in range(10):
        np.testing.assert_array_equal(batch[k], one)
    assert rel_err(one, O.solve_helmholtz_dst(f, 0.1, 0.2, 1.5)) < 1e-12


def test_dst_odd_size_fp32_uses_fp64_chain(cuda_ok):
    f = np.random.default_rng(2).standard_normal((37, 29))
    ref = O.solve_helmholtz_dst(f, 0.1, 0.2, 0.0)
    got = solve_helmholtz_dst(dev(f, torch.float32), 0.1, 0.2, 0.0)
    assert rel_err(host(got), ref) < 1e-6


@pytest.mark.parametrize("lam", [0.0, 1.0 / 4e4 ** 2, 1.0 / 1e4 ** 2])
def test_dst_refinement_reaches_1e12(cuda_ok, lam):
    n = 256
    dx = 5.12e6 / n
    f = O.kminus3_field(n, n, 7, std=1e-5)
    plan = DSTHelmholtzPlan(n, n, dx, dx, (lam,))
    psi, info = plan.solve_refined(dev(f), tol=1e-12)
    assert info["converged"] and info["backward_error"] <= 1e-12, info
    ref = O.solve_helmholtz_dst(f, dx, dx, lam)
    assert rel_err(host(psi), ref) < 1e-10
    r = O.dirichlet_helmholtz_apply(host(psi), dx, dx, lam) - f
    assert np.linalg.norm(r) <= 1e-9 * np.linalg.norm(f) or lam == 0.0


def test_dst_batched_per_layer_lambda(cuda_ok):
    rng = np.random.default_rng(4)
    f = rng.standard_normal((2, 3, 64, 64))
    lam = np.array([0.0, 2.0, 10.0])
    got = solve_helmholtz_dst(dev(f, torch.float32), 0.1, 0.1, lam)
    ref = O.solve_helmholtz_dst(f, 0.1, 0.1, lam)
    assert rel_err(host(got), ref) < 1e-4
    got64 = solve_helmholtz_dst(dev(f), 0.1, 0.1, lam)
    assert rel_err(host(got64), ref) < 1e-12


def qg_setup(n, dtype, seed=0):
    L = 5.12e6
    grid = fvx.ArakawaCGrid2D.from_interior(n, n, L, L)
    q = np.zeros((n + 2, n + 2))
    q[1:-1, 1:-1] = O.kminus3_field(n, n, seed, std=1e-5)
    q = O.enforce_periodic(q)
    return grid, q


# 64^2: every tile touches the boundary; 256^2 (and 320 x 256) also has
# interior tiles, which the stage kernel runs without boundary handling
@pytest.mark.parametrize("method,n", [("weno5", 64), ("upwind1", 64), ("weno7", 64), ("van_leer", 64),
                                      ("weno5", 256), ("weno9", 256), ("van_leer", 256), ("wenoz5", 256)])
def test_qg_tendency_fp64(cuda_ok, method, n):
    grid, q = qg_setup(n, torch.float64)
    lam = 1.0 / 4e4 ** 2
    m = QGModel(grid, 1.7e-11, lam, method=method, dtype=torch.float64, drag=1e-7, viscosity=50.0)
    got = m.tendency(dev(q))
    ref = O.qg_tendency(q, grid.dx, grid.dy, 1.7e-11, lam, method, drag=1e-7, viscosity=50.0)
    g, r = host(got)[1:-1, 1:-1], ref[1:-1, 1:-1]
    assert rel_err(g, r) < 1e-11


@pytest.mark.parametrize("bc", ("periodic", "wall"))
def test_qg_step_fp64_fused_and_unfused(cuda_ok, bc):
    n = 64
    grid, q = qg_setup(n, torch.float64, 1)
    lam, beta, dt = 1.0 / 4e4 ** 2, 1.7e-11, 0.5 * (5.12e6 / n)
    m = QGModel(grid, beta, lam, method="weno5", bc=bc, dtype=torch.float64)
    ref = O.qg_step(q, grid.dx, grid.dy, beta, lam, dt, "weno5", bc)
    got = m.step(dev(q), dt)
    assert rel_err(host(got), ref) < 1e-12
    dq_ref = ref - q
    assert rel_err(host(got) - q, dq_ref) < 1e-8
    got_u = m.step_unfused(dev(q), dt)
    assert rel_err(host(got_u), ref) < 1e-12


def test_qg_step_fp32_within_1e5(cuda_ok):
    n = 256
    grid, q = qg_setup(n, torch.float32, 2)
    lam, beta, dt = 1.0 / 4e4 ** 2, 1.7e-11, 0.5 * (5.12e6 / n)
    m = QGModel(grid, beta, lam, method="weno5", dtype=torch.float32)
    ref = O.qg_step(q, grid.dx, grid.dy, beta, lam, dt, "weno5")
    got = m.step(dev(q, torch.float32), dt)
    assert rel_err(host(got), ref) < 1e-5
    # repeated steps keep the split workspace consistent (presplit path)
    q1 = m.step(dev(q, torch.float32), dt)
    q2a = m.step(q1, dt, presplit=True)
    q2b = m.step(q1.clone(), dt, presplit=False)
    np.testing.assert_array_equal(host(q2a), host(q2b))
    m.plan.check_device()


@pytest.mark.parametrize("method", ("weno7", "weno9"))
def test_qg_step_fp32_wide_schemes_within_1e5(cuda_ok, method):
    # the stage kernel's wide WENO faces (evaluated through calls) in FP32:
    # one step at 256^2 within the FP32 bar of the FP64 oracle
    n = 256
    grid, q = qg_setup(n, torch.float32, 15)
    lam, beta, dt = 1.0 / 4e4 ** 2, 1.7e-11, 0.5 * (5.12e6 / n)
    m = QGModel(grid, beta, lam, method=method, dtype=torch.float32)
    ref = O.qg_step(q.astype(np.float32).astype(np.float64), grid.dx, grid.dy, beta, lam, dt, method)
    got = m.step(dev(q, torch.float32), dt)
    assert rel_err(host(got), ref) < 1e-5


def test_autotuner_choices_keep_results(cuda_ok, tmp_path, monkeypatch):
    # every tile shape and both split placements give the same step (FP32,
    # 1e-6 relative: only accumulation order may differ), and the tuner
    # caches its choice
    from finitevolx_b200 import autotune
    monkeypatch.setenv("FVX_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    n = 256
    grid, q = qg_setup(n, torch.float32, 5)
    lam, beta, dt = 1.0 / 4e4 ** 2, 1.7e-11, 0.5 * (5.12e6 / n)
    m = QGModel(grid, beta, lam, method="weno5", dtype=torch.float32)
    qd = dev(q, torch.float32)
    outs = []
    for cfg in range(len(autotune._TILES)):
        autotune.set_stage_tile("weno5", torch.float32, cfg)
        outs.append(host(m.step(qd, dt)))
    m.fuse_split = False
    outs.append(host(m.step(qd, dt)))
    m.fuse_split = True
    for o in outs[1:]:
        assert rel_err(o, outs[0]) < 1e-6
    r1 = autotune.tune_qg_stage(m, qd, dt)
    assert r1["tile"] in autotune._TILES and len(r1["ms"]) == len(autotune._TILES)
    r2 = autotune.tune_qg_split(m, qd, dt)
    assert set(r2["ms"]) == {"fused", "unfused"}
    assert autotune.tune_qg_stage(m, qd, dt) == r1  # from the cache
    r3 = autotune.tune_dst_kernel(m, qd, dt)
    assert set(r3["ms"]) == set(autotune.DST_KERNELS) and r3["kernel"] in autotune.DST_KERNELS
    autotune.set_stage_tile("weno5", torch.float32, 0)
    autotune.set_dst_kernel("single64")


@pytest.mark.parametrize("method", ("wenoz5", "weno5"))
def test_qg_step_fp32_register_window_interior(cuda_ok, method):
    # 320^2: interior tiles take the register-window WENO path (packed f32x2
    # face pairs, u and v from psi differences), edge tiles the shared-memory
    # one; both must sit within the FP32 bar of the oracle
    n = 320
    grid, q = qg_setup(n, torch.float32, 6)
    lam, beta, dt = 1.0 / 4e4 ** 2, 1.7e-11, 0.5 * (5.12e6 / n)
    m = QGModel(grid, beta, lam, method=method, dtype=torch.float32)
    ref = O.qg_step(q, grid.dx, grid.dy, beta, lam, dt, method)
    assert rel_err(host(m.step(dev(q, torch.float32), dt)), ref) < 1e-5


def qg_setup_rect(ny, nx, seed, bc="periodic"):
    L = 5.12e6
    grid = fvx.ArakawaCGrid2D.from_interior(nx, ny, L * nx / 256, L * ny / 256)
    q = np.zeros((ny + 2, nx + 2))
    q[1:-1, 1:-1] = O.kminus3_field(ny, nx, seed, std=1e-5)
    q = O.enforce_periodic(q) if bc == "periodic" else O.pad_interior_constant(q)
    return grid, q


# FP32 stage-kernel fallbacks, each against the FP64 oracle at the FP32-step
# bar (1e-5 relative on q_{n+1}):
#  - odd total width (Nx = 203): rows are not 8-byte aligned, so the tile
#    loads fall back to 4-byte copies (and the DST to the FP64 chain);
#  - wall boundaries (zero ghosts, no periodic refill);
#  - forcing, bottom drag and viscosity: interior tiles leave the fast
#    column-walk tendency for the general per-cell loop.
@pytest.mark.parametrize("ny,nx,bc,method", [(256, 201, "periodic", "weno5"), (192, 201, "wall", "wenoz5"),
                                             (256, 256, "wall", "weno5"), (320, 256, "wall", "weno7")])
def test_qg_step_fp32_fallback_paths(cuda_ok, ny, nx, bc, method):
    grid, q = qg_setup_rect(ny, nx, 8, bc)
    lam, beta, dt = 1.0 / 4e4 ** 2, 1.7e-11, 0.5 * grid.dx
    m = QGModel(grid, beta, lam, method=method, bc=bc, dtype=torch.float32)
    ref = O.qg_step(q, grid.dx, grid.dy, beta, lam, dt, method, bc)
    assert rel_err(host(m.step(dev(q, torch.float32), dt)), ref) < 1e-5
    assert rel_err(host(m.step_unfused(dev(q, torch.float32), dt)), ref) < 1e-5


@pytest.mark.parametrize("n,method", [(256, "weno5"), (320, "wenoz5"), (256, "upwind3")])
def test_qg_step_fp32_forcing_drag_viscosity(cuda_ok, n, method):
    grid, q = qg_setup(n, torch.float32, 9)
    lam, beta, dt = 1.0 / 4e4 ** 2, 1.7e-11, 0.5 * (5.12e6 / n)
    forcing = np.zeros_like(q)
    forcing[1:-1, 1:-1] = 1e-12 * O.kminus3_field(n, n, 10)
    kw = dict(forcing=forcing, drag=1e-7, viscosity=50.0)
    m = QGModel(grid, beta, lam, method=method, dtype=torch.float32, **kw)
    ref = O.qg_step(q, grid.dx, grid.dy, beta, lam, dt, method, **kw)
    got = host(m.step(dev(q, torch.float32), dt))
    assert rel_err(got, ref) < 1e-5
    # the extra terms change the step by far more than the bar
    plain = O.qg_step(q, grid.dx, grid.dy, beta, lam, dt, method)
    assert rel_err(plain, ref) > 1e-4


def test_qg_step_fp32_2048_within_1e5(cuda_ok):
    # the benchmarked configuration: 2048^2 interior, Ld = 40 km, WENO5,
    # periodic q, DST psi, one rk3_ssp_step at CFL 0.5 for max|u| = 1 m/s;
    # 1e-5 relative on q_{n+1} against the FP64 oracle (about 10 s of CPU)
    n = 2048
    grid, q = qg_setup(n, torch.float32, 11)
    lam, beta, dt = 1.0 / 4e4 ** 2, 1.7e-11, 0.5 * (5.12e6 / n)
    m = QGModel(grid, beta, lam, method="weno5", dtype=torch.float32)
    from finitevolx_b200._lib import fn
    assert fn("fvx_dst_operand_layout")(m.plan.handle) == 1  # the even/odd tensor-core products
    got = host(m.step(dev(q, torch.float32), dt))
    m.plan.check_device()
    ref = O.qg_step(q, grid.dx, grid.dy, beta, lam, dt, "weno5")
    assert rel_err(got, ref) < 1e-5
    # and the step's increment itself is resolved (not hidden under q_n)
    assert rel_err(got - q, ref - q) < 1e-3


def test_qg_step_fp64_256_within_1e12(cuda_ok):
    # the metric's own configuration: 256^2 interior, FP64, Ld = 40 km, WENO5
    n = 256
    grid, q = qg_setup(n, torch.float64, 12)
    lam, beta, dt = 1.0 / 4e4 ** 2, 1.7e-11, 0.5 * (5.12e6 / n)
    m = QGModel(grid, beta, lam, method="weno5", dtype=torch.float64)
    ref = O.qg_step(q, grid.dx, grid.dy, beta, lam, dt, "weno5")
    got = host(m.step(dev(q), dt))
    assert rel_err(got, ref) < 1e-12
    assert rel_err(got - q, ref - q) < 1e-9


def test_qg_step_fp64_stage_writes_chain_input(cuda_ok):
    # FP64: the stage kernel writes its output's interior into the FP64
    # chain's input (no copy pass before the next solve); the same step as
    # with the copy pass, bit for bit, and across steps with presplit
    n = 256
    grid, q = qg_setup(n, torch.float64, 16)
    dt = 0.5 * (5.12e6 / n)
    m = QGModel(grid, 1.7e-11, 1.0 / 4e4 ** 2, method="weno5", dtype=torch.float64)
    assert m._fused_copy64
    fused = m.step(dev(q), dt)
    m.fuse_split = False
    plain = m.step(dev(q), dt)
    np.testing.assert_array_equal(host(fused), host(plain))
    m.fuse_split = True
    q1 = m.step(dev(q), dt)
    q2a = m.step(q1, dt, presplit=True)
    q2b = m.step(q1.clone(), dt, presplit=False)
    np.testing.assert_array_equal(host(q2a), host(q2b))


def test_qg_step_fp64_every_stage_tile(cuda_ok):
    # the FP64 stage tile is autotuned: every shape the tuner may pick meets
    # the FP64 bar at the metric's configuration
    from finitevolx_b200 import autotune
    n = 256
    grid, q = qg_setup(n, torch.float64, 14)
    lam, beta, dt = 1.0 / 4e4 ** 2, 1.7e-11, 0.5 * (5.12e6 / n)
    m = QGModel(grid, beta, lam, method="weno5", dtype=torch.float64)
    ref = O.qg_step(q, grid.dx, grid.dy, beta, lam, dt, "weno5")
    try:
        for cfg in range(len(autotune._TILES)):
            autotune.set_stage_tile("weno5", torch.float64, cfg)
            assert rel_err(host(m.step(dev(q), dt)), ref) < 1e-12, autotune._TILES[cfg]
    finally:
        autotune.set_stage_tile("weno5", torch.float64, 0)


@pytest.mark.parametrize("n,ld", [(128, 6.7e5), (512, 4.0e6)])
def test_qg_step_fp32_refined_weak_screening(cuda_ok, n, ld):
    # weakly screened fields (lambda dx^2 << 1): the plain split chain misses
    # the FP32 bar, one FP64-residual refinement pass per solve meets it
    grid, q = qg_setup(n, torch.float32, 13)
    lam, beta, dt = 1.0 / ld ** 2, 1.7e-11, 0.5 * (5.12e6 / n)
    ref = O.qg_step(q.astype(np.float32).astype(np.float64), grid.dx, grid.dy, beta, lam, dt, "weno5")
    plain = QGModel(grid, beta, lam, method="weno5", dtype=torch.float32)
    refined = QGModel(grid, beta, lam, method="weno5", dtype=torch.float32, dst_refine=1)
    assert rel_err(host(plain.step(dev(q, torch.float32), dt)), ref) > 1e-5
    assert rel_err(host(refined.step(dev(q, torch.float32), dt)), ref) < 1e-5
    # the refined unfused path (separate split pass) agrees
    refined.fuse_split = False
    assert rel_err(host(refined.step(dev(q, torch.float32), dt)), ref) < 1e-5
    refined.plan.check_device()


@pytest.mark.parametrize("lam", [0.0, 1.0 / 1e4 ** 2])
def test_dst_refinement_1024_batched(cuda_ok, lam):
    # config 3's size and batching (a 16-RHS slice of its 64): split chain +
    # FP64 refinement to a 1e-12 backward error; every result within 1e-10
    # of the FP64 DST oracle
    n, b = 1024, 16
    dx = 5.12e6 / n
    f = np.stack([O.kminus3_field(n, n, 40 + k, std=1e-5) for k in range(b)])
    plan = DSTHelmholtzPlan(n, n, dx, dx, (lam,), batch_max=b)
    psi, info = plan.solve_refined(dev(f), tol=1e-12)
    assert info["converged"] and info["backward_error"] <= 1e-12, info
    plan.check_device()
    ref = O.solve_helmholtz_dst(f, dx, dx, lam)
    got = host(psi)
    errs = [rel_err(got[k], ref[k]) for k in range(b)]
    assert max(errs) < 1e-10, errs
    # the FP32 chain on the same batch: the split chain's ~1e-5
    p32 = host(plan.solve(dev(f, torch.float32)))
    assert max(rel_err(p32[k], ref[k]) for k in range(b)) < 1e-4
