"""GPU parity of the ensemble of multi-layer QG members (uneven sizes and
layer counts, one persistent work-queue stage launch per RK stage, batched DST
per size group) against the FP64 multi-layer oracle, member by member; graph
replay equals eager steps.

Two bars:
* logic: single-layer members against QGModel.step, which runs the same DST
  plan type and fused stage kernel one field at a time -- 2e-5 relative (the
  batched products accumulate in a different K order per tile, which can
  flip a bf16 hi/lo rounding of an intermediate; an indexing or mixing error
  would show at O(1));
* precision: every member against the FP64 oracle -- 2e-4 relative after one
  FP32 step.  The FP32 DST chain carries its operands as hi + lo bf16 (16
  bits, psi error ~1e-5 relative to the largest mode); the velocity
  differentiation amplifies it (2.8e-5 in q for the 64^2, Rd ~ 670 km member,
  reproduced by tests/test_split_precision.py), and in multi-layer members the
  barotropic mode's error reaches the weaker layers through mode_to_layer.
  The 1.5-layer 2048^2 / Ld 40 km step meets 1e-5 (test_gpu_dst_qg.py)."""

import numpy as np
import pytest
import torch

import finitevolx_b200 as fvx
import oracle.fvx_oracle as O

pytestmark = pytest.mark.gpu

MEMBERS = [(64, 1), (128, 2), (256, 3), (64, 3), (256, 1)]


def init_state(ens, seed=0):
    qs = []
    for m, (n, nl) in enumerate(ens.members):
        q = np.zeros((nl, n + 2, n + 2))
        for k in range(nl):
            q[k, 1:-1, 1:-1] = O.kminus3_field(n, n, 100 * seed + 10 * m + k, std=1e-5)
            q[k] = O.enforce_periodic(q[k])
            ens.set_layer(m, k, torch.from_numpy(q[k]).float())
        qs.append(q)
    return qs


def test_ensemble_one_step_matches_oracle(cuda_ok):
    ens = fvx.QGEnsemble(MEMBERS)
    qs = init_state(ens)
    ens.step(1)
    torch.cuda.synchronize()
    errs = {}
    for m, (n, nl) in enumerate(ens.members):
        l2m, m2l, lam = ens.modes[m]
        q32 = np.stack([qs[m][k].astype(np.float32).astype(np.float64) for k in range(nl)])
        ref = O.mlqg_step(q32, l2m, m2l, lam, ens.dx[m], ens.dx[m], ens.beta, ens.dt[m], "weno5")
        for k in range(nl):
            got = ens.get_layer(m, k).double().cpu().numpy()
            errs[(m, k)] = np.abs(got - ref[k]).max() / np.abs(ref[k]).max()
    assert max(errs.values()) < 2e-4, sorted(errs.items(), key=lambda kv: -kv[1])


def test_ensemble_single_layer_matches_qgmodel(cuda_ok):
    members = [(64, 1), (128, 1), (256, 1), (128, 1)]
    ens = fvx.QGEnsemble(members)
    qs = init_state(ens, 2)
    ens.step(1)
    torch.cuda.synchronize()
    for m, (n, nl) in enumerate(members):
        grid = fvx.ArakawaCGrid2D.from_interior(n, n, ens.Lx, ens.Lx)
        lam = float(ens.modes[m][2][0])
        model = fvx.QGModel(grid, ens.beta, lam, method="weno5", dtype=torch.float32)
        ref = model.step(torch.from_numpy(qs[m][0]).float().cuda(), ens.dt[m]).double().cpu().numpy()
        got = ens.get_layer(m, 0).double().cpu().numpy()
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err < 2e-5, (m, err)


def test_ensemble_graph_replay_matches_eager(cuda_ok):
    a = fvx.QGEnsemble(MEMBERS[:3])
    b = fvx.QGEnsemble(MEMBERS[:3])
    init_state(a, 1)
    init_state(b, 1)
    g = a.capture(2)        # capture runs one eager step first
    g.replay()              # + 2 steps
    b.step(3)
    torch.cuda.synchronize()
    for m, (n, nl) in enumerate(a.members):
        for k in range(nl):
            assert torch.equal(a.get_layer(m, k), b.get_layer(m, k)), (m, k)
    assert a.launches_per_step == 3 * (len({n for n, _ in MEMBERS[:3]}) * 6 + 2)
