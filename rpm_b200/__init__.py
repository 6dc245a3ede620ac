"""rpm_b200: B200-native engine for the radical-pair matrix-free Krylov hot path.

Drop-in for ``rpm_statevector_engine`` (Hamiltonian action, adaptive Lanczos
propagation, singlet observable) plus the production assembly helpers, backed
by hand-written sm_100a kernels in ``lib/librpm_b200.so`` (C ABI:
``include/rpm_b200.h``).  The batched mixed-precision propagator lives in
:mod:`rpm_b200.batched`.
"""

from .engine import (  # noqa: F401
    AdaptiveLanczosPropagator,
    CompiledFullPairHamiltonian,
    LocalTerm,
    MatrixFreeHamiltonian,
    PropagationResult,
    PropagationStats,
    SingletPopulationObservable,
    random_phase_nuclear_state,
    singlet_initial_state,
    singlet_population,
    state_error_to_population_bound,
)
from .model import (  # noqa: F401
    efimova_hore_electron_coupling_operator,
    field_vector_mT,
    quadrupole_operator,
    spin_operators,
    two_spin_coupling_operator,
)
from .production import (  # noqa: F401
    build_hamiltonian,
    build_quantum_needle_hamiltonian,
    coarse_grid_indices,
    integrate_yield,
    make_propagator,
    random_phase_initial_state,
)

__version__ = "0.1.0"
