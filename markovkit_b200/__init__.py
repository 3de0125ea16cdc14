"""markovkit_b200: MarkovKit's RDME resolvent solve and Krylov FSP on NVIDIA B200.

The compute lives in libmarkovkit_b200.so (hand-written sm_100a CUDA behind the C ABI of
include/markovkit_b200.h). This package is the Python mirror of the reference API over it.
"""

from .api import (  # noqa: F401
    full_multigrid,
    generator,
    gmres,
    gmres_options,
    grid,
    host_preconditioner,
    ilu0_preconditioner,
    jacobi_preconditioner,
    jump,
    local_reaction,
    multigrid_options,
    population_box,
    population_sector,
    reaction_diffusion,
    sector_multigrid,
    shifted_generator,
    solver,
    batch_solver,
    set_row_path,
    voxel_domain,
)
from .inputs import dirichlet_rhs, uniform01, uniform_rhs  # noqa: F401
