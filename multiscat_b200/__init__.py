"""B200-native close-coupling atom-surface scattering solver.

Public entry points:

- :func:`run_multiscat_fortran` -- drop-in for the reference's f2py solve
  (same arguments, returns psi[nkx, nky, nz]).
- :func:`get_scattering_matrix` / :func:`get_scattering_matrices` -- the
  reference-shaped API on slate-free condition objects.
- :class:`ScatteringPlan` -- batched, device-resident solves.

The solve runs in hand-written CUDA (``libmultiscat_b200.so``); there is no
CPU fallback.
"""

from .api import (
    OptimizationConfig,
    ScatteringCondition,
    ScatteringMetadata,
    UnitSystem,
    get_scattering_matrices,
    get_scattering_matrix,
    get_scattering_matrix_from_state,
    get_scattering_matrix_von_neumann,
    get_scattering_state,
    momentum_from_angles,
    natural_arrays,
)
from .solver import (
    ScatteringPlan,
    SolveResult,
    SystemSpec,
    channel_subset_system,
    full_grid_system,
    release_cached_memory,
    run_multiscat_fortran,
)

__all__ = [
    "OptimizationConfig", "ScatteringCondition", "ScatteringMetadata", "UnitSystem",
    "get_scattering_matrices", "get_scattering_matrix", "get_scattering_matrix_von_neumann",
    "get_scattering_state", "get_scattering_matrix_from_state",
    "momentum_from_angles", "natural_arrays",
    "ScatteringPlan", "SolveResult", "SystemSpec", "channel_subset_system", "full_grid_system",
    "release_cached_memory", "run_multiscat_fortran",
]
