"""CPU: the threaded oracle step (bench's CPU legs) is bit-identical to the
single-threaded oracle step, with bands small enough that every band edge
falls inside the domain and the halo rows matter."""

import numpy as np
import pytest

import oracle.fvx_oracle as O
from oracle.threaded import qg_step_threaded


@pytest.mark.parametrize("method", ("weno5", "weno9", "van_leer"))
def test_threaded_step_bit_identical(method):
    n = 96
    dx = 5.12e6 / n
    q = np.zeros((n + 2, n + 2))
    q[1:-1, 1:-1] = O.kminus3_field(n, n, 3, std=1e-5)
    q = O.enforce_periodic(q)
    ref = O.qg_step(q, dx, dx, 1.7e-11, 1.0 / 4e4 ** 2, 0.5 * dx, method)
    got = qg_step_threaded(q, dx, dx, 1.7e-11, 1.0 / 4e4 ** 2, 0.5 * dx, method, workers=4, min_rows=16)
    np.testing.assert_array_equal(got, ref)
