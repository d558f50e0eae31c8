"""GPU: QGPipeline (uploads, graph-replayed steps and downloads of a stream
of host states on three streams) gives the same states as QGModel.step."""

import numpy as np
import pytest
import torch

import finitevolx_b200 as fvx
import oracle.fvx_oracle as O

pytestmark = pytest.mark.gpu


def test_pipeline_matches_step(cuda_ok):
    n = 256
    Lx = 5.12e6
    grid = fvx.ArakawaCGrid2D.from_interior(n, n, Lx, Lx)
    m = fvx.QGModel(grid, 1.7e-11, 1.0 / 4e4 ** 2, method="weno5", dtype=torch.float32)
    dt = 0.5 * Lx / n
    states = []
    for seed in range(3):
        q = np.zeros((n + 2, n + 2))
        q[1:-1, 1:-1] = O.kminus3_field(n, n, seed, std=1e-5)
        states.append(O.enforce_periodic(q))
    host_in = torch.tensor(np.stack(states), dtype=torch.float32).pin_memory()
    host_out = torch.zeros_like(host_in).pin_memory()
    pipe = fvx.QGPipeline(m, dt)
    pipe.run(host_in, host_out, n=7)  # wraps around the three host states
    torch.cuda.synchronize()
    for k in range(3):
        ref = m.step(host_in[k].cuda(), dt).cpu()
        got = host_out[k]
        assert float((got - ref).abs().max() / ref.abs().max()) <= 1e-6
