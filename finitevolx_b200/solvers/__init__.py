"""Elliptic solvers: DST Helmholtz, masked CG / multigrid, PV inversion."""

from finitevolx_b200.solvers.spectral import (
    DSTHelmholtzPlan,
    dst1_eigenvalues,
    solve_helmholtz_dst,
    solve_poisson_dst,
)
