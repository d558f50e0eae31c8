"""Elliptic solvers: DST Helmholtz, masked CG / multigrid, PV inversion."""

from finitevolx_b200.solvers.spectral import (
    DSTHelmholtzPlan,
    dst1_eigenvalues,
    solve_helmholtz_dst,
    solve_poisson_dst,
)
from finitevolx_b200.solvers.multigrid import (
    MultigridSolver,
    build_multigrid_solver,
    make_multigrid_preconditioner,
)
from finitevolx_b200.solvers.iterative import CGInfo, MaskedHelmholtzPCG, masked_laplacian, solve_cg
from finitevolx_b200.solvers.elliptic import pv_inversion, streamfunction_from_vorticity
