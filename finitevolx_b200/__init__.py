"""finitevolx_b200: B200-native (sm_100a) drop-in for finitevolX's explicit-step
and elliptic-inversion hot path.

Public names mirror ``finitevolx`` (finitevolx/__init__.py).  Every operator
runs in libfvx.so, a C-ABI CUDA library built for sm_100a; arrays are CUDA
``torch.Tensor`` objects (NumPy inputs are copied to the device).
"""

from finitevolx_b200.grid import ArakawaCGrid2D, CartesianGrid2D
from finitevolx_b200.mask import (
    Mask2D,
    StencilCapability2D,
    count_contiguous,
    make_sponge,
    narrow_mask_hierarchy,
)
from finitevolx_b200.advection import (
    Advection2D,
    Reconstruction2D,
    upwind_flux,
    uv_center_flux,
    uv_node_flux,
)
from finitevolx_b200.operators import (
    Difference2D,
    Interpolation2D,
    arakawa_jacobian,
    divergence_2d,
)
from finitevolx_b200.diffusion import BiharmonicDiffusion2D, Diffusion2D, diffusion_2d
from finitevolx_b200.boundary import enforce_periodic, enforce_periodic_, pad_interior
from finitevolx_b200.timestepping import euler_step, heun_step, rk3_ssp_step
from finitevolx_b200.solvers import (
    CapacitanceSolver,
    CGInfo,
    DSTHelmholtzPlan,
    MaskedHelmholtzPCG,
    MultigridSolver,
    SpectralHelmholtzPlan,
    build_capacitance_solver,
    build_multigrid_solver,
    dct2_eigenvalues,
    dst1_eigenvalues,
    fft_eigenvalues,
    make_multigrid_preconditioner,
    make_spectral_preconditioner,
    masked_laplacian,
    pressure_from_divergence,
    pv_inversion,
    solve_cg,
    solve_helmholtz_dct,
    solve_helmholtz_dst,
    solve_helmholtz_fft,
    solve_poisson_dct,
    solve_poisson_dst,
    solve_poisson_fft,
    streamfunction_from_vorticity,
)
from finitevolx_b200.vertical import (
    build_coupling_matrix,
    decompose_vertical_modes,
    layer_to_mode,
    mode_to_layer,
)
from finitevolx_b200.qg import QGModel, QGPipeline
from finitevolx_b200.ensemble import QGEnsemble
from finitevolx_b200.swm import Coriolis2D, MomentumAdvection2D, Vorticity2D
from finitevolx_b200 import diagnostics
from finitevolx_b200.snapshots import QGSnapshotRecorder, read_zarr_v3

__all__ = [
    "ArakawaCGrid2D", "CartesianGrid2D", "Mask2D", "StencilCapability2D", "count_contiguous",
    "make_sponge", "narrow_mask_hierarchy", "Advection2D", "Reconstruction2D", "upwind_flux",
    "uv_center_flux", "uv_node_flux", "Difference2D", "Interpolation2D", "arakawa_jacobian",
    "divergence_2d", "BiharmonicDiffusion2D", "Diffusion2D", "diffusion_2d", "enforce_periodic",
    "enforce_periodic_", "pad_interior", "euler_step", "heun_step", "rk3_ssp_step", "CGInfo",
    "DSTHelmholtzPlan", "MaskedHelmholtzPCG", "MultigridSolver", "build_multigrid_solver",
    "make_multigrid_preconditioner", "masked_laplacian", "pv_inversion", "solve_cg", "solve_helmholtz_dst",
    "CapacitanceSolver", "SpectralHelmholtzPlan", "build_capacitance_solver", "dct2_eigenvalues",
    "dst1_eigenvalues", "fft_eigenvalues", "make_spectral_preconditioner", "pressure_from_divergence",
    "solve_helmholtz_dct", "solve_helmholtz_fft", "solve_poisson_dct", "solve_poisson_fft",
    "solve_poisson_dst", "streamfunction_from_vorticity", "build_coupling_matrix",
    "decompose_vertical_modes", "layer_to_mode", "mode_to_layer", "QGModel", "QGPipeline", "QGEnsemble", "QGSnapshotRecorder", "read_zarr_v3",
    "Coriolis2D", "MomentumAdvection2D", "Vorticity2D", "diagnostics",
]
