"""Canonical 18x18 inputs of the reference's golden fixtures, restated.

Mirrors finitevolX tests/fixtures/inputs.py:47-58 (sizes), :141-184 (the
cross-island h-mask) and :245-287 (analytic fields) with NumPy.
"""

import numpy as np

NY_I = NX_I = 16
NY = NX = 18
LX = LY = 1.0
DX = LX / NX_I
DY = LY / NY_I


def h_mask_2d():
    h = np.zeros((NY, NX), dtype=bool)
    h[1:-1, 1:-1] = True
    h[1, :] = h[-2, :] = False
    h[:, 1] = h[:, -2] = False
    h[6:9, 6:11] = False
    h[5:10, 7:10] = False
    return h


def _xy():
    x = np.linspace(0.0, 1.0, NX)
    y = np.linspace(0.0, 1.0, NY)
    Y, X = np.meshgrid(y, x, indexing="ij")
    return X, Y


def fields_2d():
    X, Y = _xy()
    return dict(
        h=np.sin(2.0 * np.pi * X) * np.cos(np.pi * Y) + 0.5 * (X + Y),
        u=np.cos(np.pi * X) * np.sin(2.0 * np.pi * Y),
        v=-np.sin(np.pi * X) * np.cos(2.0 * np.pi * Y),
        q=np.sin(np.pi * X) * np.sin(np.pi * Y),
        f=1.0 + 0.1 * Y,
    )
