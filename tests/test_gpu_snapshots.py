"""GPU: QGSnapshotRecorder's planes (fused snapshot kernel after the
library's DST, velocity and vorticity kernels) and its Zarr v3 store against
the FP64 oracle's record_snapshot.  FP64 model: 1e-11 relative per plane;
FP32 model: 1e-4 (the split DST chain)."""

import numpy as np
import pytest
import torch

import finitevolx_b200 as fvx
import oracle.fvx_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 1e-4)])
def test_snapshots_match_oracle(cuda_ok, tmp_path, dtype, tol):
    n, Lx = 64, 5.12e6
    grid = fvx.ArakawaCGrid2D.from_interior(n, n, Lx, Lx)
    lam, beta, dt, eta_scale = 1.0 / 4e4 ** 2, 1.7e-11, 0.5 * Lx / n, 9.375e-5 / 9.81
    m = fvx.QGModel(grid, beta, lam, method="weno5", dtype=dtype)
    q = np.zeros((n + 2, n + 2))
    q[1:-1, 1:-1] = O.kminus3_field(n, n, 3, std=1e-5)
    q = O.enforce_periodic(q)
    qd = torch.as_tensor(q, dtype=dtype, device="cuda")
    rec = fvx.QGSnapshotRecorder(m, tmp_path / "qg.zarr", dt, eta_scale, attrs={"model": "1.5-layer QG"})
    states = []
    for k in range(5):
        if k % 2 == 0:
            rec.record(qd, k)
            states.append((k, qd.double().cpu().numpy()))
        qd = m.step(qd, dt)
    rec.close()
    got = fvx.read_zarr_v3(tmp_path / "qg.zarr")
    assert got["__attrs__"] == {"model": "1.5-layer QG"}
    np.testing.assert_allclose(got["time"][0], [k * dt for k, _ in states])
    for t, (k, qs) in enumerate(states):
        planes, ens = O.qg_snapshot(qs, grid.dx, grid.dy, lam, eta_scale)
        for p, (name, _, _) in enumerate(fvx.snapshots.VARIABLES):
            arr, dims, attrs = got[name]
            assert dims == ["time", "y", "x"] and arr.shape == (len(states), n, n)
            ref = planes[p]
            err = np.abs(arr[t] - ref).max() / max(np.abs(ref).max(), 1e-300)
            assert err < tol, (name, t, err)
        assert abs(got["pv_enstrophy"][0][t] - ens) <= tol * ens
