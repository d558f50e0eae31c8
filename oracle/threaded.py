"""The oracle's QG step on all host cores -- TEST AND BENCH INFRASTRUCTURE ONLY.

``qg_step_threaded`` evaluates exactly ``fvx_oracle.qg_step`` (the FP64
restatement of finitevolX's QG 1.5-layer RK3 step,
scripts/qg_1p5_layer.py:420-497 with timestepping/explicit_rk.py:74-121),
spread over host threads: the DST Helmholtz solve runs its 1-D transforms
on SciPy's FFT workers, and the tendency (geostrophic velocity, WENO
advection, beta term) runs on bands of rows, each band computed with a halo
of ``HALO`` rows on both sides and only its own rows kept.  Every output
element is produced by the same NumPy operations on the same inputs as in
the single-threaded step, so the result is bit-identical to
``fvx_oracle.qg_step`` (tests/test_oracle_threaded.py).  Only ``bench.py``'s
CPU legs and the tests use it; the product never does.
"""

from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from oracle import fvx_oracle as O

# The tendency at row j reads u, v on rows j-4 .. j+4 (WENO9 reach 5 plus the
# flux divergence) and u, v read psi on rows j-1 .. j+1: 8 halo rows cover
# every scheme with margin.
HALO = 8


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover - non-Linux hosts
        return os.cpu_count() or 1


def _bands(ny: int, workers: int, min_rows: int = 64):
    nb = max(1, min(workers, ny // min_rows))
    edges = np.linspace(0, ny, nb + 1).astype(int)
    return [(int(edges[k]), int(edges[k + 1])) for k in range(nb)]


def qg_tendency_threaded(q, dx, dy, beta, lam, method, pool, workers, min_rows=64):
    """fvx_oracle.qg_tendency (periodic q, no forcing/drag/viscosity) on bands of rows."""
    import scipy.fft

    qb = O.enforce_periodic(q)
    psi = np.zeros_like(qb)
    with scipy.fft.set_workers(workers):
        psi[1:-1, 1:-1] = O.solve_helmholtz_dst(qb[1:-1, 1:-1], dx, dy, lam)
    ny = qb.shape[0]
    out = np.empty_like(qb)

    def band(r0, r1):
        a, b = max(0, r0 - HALO), min(ny, r1 + HALO)
        t = O.qg_tendency_psi(qb[a:b], psi[a:b], dx, dy, beta, method)
        out[r0:r1] = t[r0 - a:r1 - a]

    list(pool.map(lambda rb: band(*rb), _bands(ny, workers, min_rows)))
    return out


def qg_step_threaded(q, dx, dy, beta, lam, dt, method="weno5", workers=None, min_rows=64):
    """One rk3_ssp_step of the QG tendency, periodic ghost refill; the same
    result as ``fvx_oracle.qg_step(q, dx, dy, beta, lam, dt, method)``."""
    workers = workers or host_threads()
    with ThreadPoolExecutor(workers) as pool:
        f = lambda y: qg_tendency_threaded(y, dx, dy, beta, lam, method, pool, workers, min_rows)  # noqa: E731
        return O.enforce_periodic(O.rk3_ssp_step(q, f, dt))
