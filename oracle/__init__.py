"""CPU oracle for the finitevolx_b200 parity tests (test infrastructure only).

This package restates, in plain FP64 NumPy, the arithmetic of finitevolX's
explicit-step and elliptic-inversion hot path.  It is the checker the GPU
kernels are compared against.  Only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may
import it; the product library never calls it.
"""

from oracle.fvx_oracle import *  # noqa: F401,F403
