"""Elliptic solvers: spectral Helmholtz (DST / DCT / periodic), capacitance, masked CG / multigrid, PV inversion."""

from finitevolx_b200.solvers.spectral import (
    DSTHelmholtzPlan,
    SpectralHelmholtzPlan,
    dct2_eigenvalues,
    dst1_eigenvalues,
    fft_eigenvalues,
    make_spectral_preconditioner,
    solve_helmholtz_dct,
    solve_helmholtz_dst,
    solve_helmholtz_fft,
    solve_poisson_dct,
    solve_poisson_dst,
    solve_poisson_fft,
)
from finitevolx_b200.solvers.capacitance import CapacitanceSolver, build_capacitance_solver
from finitevolx_b200.solvers.multigrid import (
    MultigridSolver,
    build_multigrid_solver,
    make_multigrid_preconditioner,
)
from finitevolx_b200.solvers.iterative import CGInfo, MaskedHelmholtzPCG, masked_laplacian, solve_cg
from finitevolx_b200.solvers.elliptic import (
    pressure_from_divergence,
    pv_inversion,
    streamfunction_from_vorticity,
)
