"""CPU: the precision budget of the FP32 tensor-core DST chain.

NumPy emulation of the device's chain (4 products, each operand split into
bf16 hi + lo, 3 split products, FP32 outputs) on the ensemble's smallest,
weakly screened member (64^2 interior, one layer, Rd ~ 670 km).  It
reproduces the one-step q error the GPU shows there (~2.8e-5 relative) and
shows that adding the fourth split product (Xl Sl) does not remove it: the
floor is the 16-bit hi + lo representation of each FP32 intermediate.
"""

import numpy as np
import torch

import oracle.fvx_oracle as O


def _bf16(x):
    return torch.from_numpy(np.asarray(x, np.float32)).to(torch.bfloat16).double().numpy()


def _split(x):
    x32 = np.asarray(x, np.float32).astype(np.float64)
    h = _bf16(x32)
    return h, _bf16(x32 - h)


def _prod(X, S, terms):
    Xh, Xl = _split(X)
    Sh, Sl = _split(S)
    C = Xh @ Sh + Xh @ Sl + Xl @ Sh + (Xl @ Sl if terms == 4 else 0.0)
    return C.astype(np.float32).astype(np.float64)


def _dst_emulated(f, d, lam, terms):
    n = f.shape[0]
    S = np.sin(np.pi * np.outer(np.arange(1, n + 1), np.arange(1, n + 1)) / (n + 1))
    e = -4 / d ** 2 * np.sin(np.pi * np.arange(1, n + 1) / (2 * (n + 1))) ** 2
    inv = 1.0 / (e[:, None] + e[None, :] - lam)
    W = _prod(f, S, terms).T
    W = _prod(W, S, terms).T * inv
    W = _prod(W, S, terms).T
    return 4.0 / (n + 1) ** 2 * _prod(W, S, terms).T


def test_split_chain_precision_budget():
    n = 64
    rr, _, _ = O.decompose_vertical_modes(O.build_coupling_matrix([400.0], [9.81]), 9.375e-5)
    lam, dx = 1.0 / rr[0] ** 2, 5.12e6 / n
    q = np.zeros((n + 2, n + 2))
    q[1:-1, 1:-1] = O.kminus3_field(n, n, 0, std=1e-5)
    q = O.enforce_periodic(q)
    psi_ref = O.solve_helmholtz_dst(q[1:-1, 1:-1], dx, dx, lam)
    pr = np.zeros_like(q)
    pr[1:-1, 1:-1] = psi_ref
    t0 = O.qg_tendency_psi(q, pr, dx, dx, 1.7e-11, "weno5")
    dt = 0.5 * dx
    step_err = {}
    for terms in (3, 4):
        p = np.zeros_like(q)
        p[1:-1, 1:-1] = _dst_emulated(q[1:-1, 1:-1], dx, lam, terms)
        t1 = O.qg_tendency_psi(q, p, dx, dx, 1.7e-11, "weno5")
        step_err[terms] = np.abs(dt * (t1 - t0)).max() / np.abs(q + dt * t0).max()
    assert 1e-5 < step_err[3] < 5e-5, step_err
    assert step_err[4] > 0.5 * step_err[3], step_err  # the dropped product is not the floor
